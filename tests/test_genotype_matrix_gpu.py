"""GenotypeMatrix half-passes (multiply_Zt_v / multiply_Z_v) and the record-level PCG.

* cs_genotype_multiply_zt / _z against the oracle's dense Z (the standardised genotypes the
  reference's PlinkReader::multiply_Z_v / multiply_Zt_v apply, libCosmicCore/src/
  plink_reader.cpp:241-438) over a sample subset and a variant selection that includes
  monomorphic and all-missing SNPs: FP64 within 1e-12 and the tensor-core form within 1e-6
  relative (max-norm per column); Z (Z^T X) / M equals the kinship apply.
* cs_pcg_solve_records against a dense solve of STCG_VCE's record-level covariance
  V = sg Zr K Zr^T + spe Zr Zr^T + se I (libCosmicCore/src/stcg_vce.cpp:80-126), 1e-9.
* A C++ program drives the reference's STCG solve (STCG_VCE::apply_G = Z (Z^T v) / M through
  the facade's GenotypeMatrix, then MatrixFreePCG with the scalar Jacobi preconditioner, as
  stcg_vce.cpp:80-126 and matrix_free_pcg.h:20-68 write them) and must reproduce the library's
  block PCG solution.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")
from cosmicscanner_b200 import _abi  # noqa: E402


def colwise_rel(Y, E):
    scale = np.maximum(np.abs(E).max(axis=0), 1e-300)
    return (np.abs(Y - E).max(axis=0) / scale)


@pytest.fixture(scope="module")
def data():
    d = synth.cohort(1900, 2300, 71, missing=0.02, n_causal=20)
    n, m = d["n"], d["m"]
    bed = d["bed"].copy()
    stride = (n + 3) // 4
    rows = bed[3:].reshape(m, stride)
    rows[5, :] = 0xFF      # monomorphic (all 11)
    rows[17, :] = 0x55     # all missing
    ref = oracle.Bed(rows, n)
    g = cs.Genotypes.from_bed_bytes(bed, n, m)
    return d, bed, ref, g


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
@pytest.mark.parametrize("selection", ["all", "subset"])
def test_half_passes_match_dense_z(data, precision, tol, selection):
    d, bed, ref, g = data
    n, m = d["n"], d["m"]
    rng = np.random.default_rng(3)
    if selection == "all":
        keep, variants = None, None
    else:
        keep = rng.choice(n, 1500, replace=False).astype(np.int32)
        variants = np.sort(np.concatenate([[5, 17], rng.choice(np.arange(20, m), 1400,
                                                               replace=False)])).astype(np.int32)
    op = cs.createKinshipOperator(g, keep, variants)
    Z = ref.dense_z(keep, variants)
    assert Z.shape == (op.rows(), op.numVariants())
    for k in (1, 7, 40):
        X = rng.standard_normal((op.rows(), k))
        V = rng.standard_normal((op.numVariants(), k))
        U = op.multiply_Zt_v(X, precision=precision)
        Y = op.multiply_Z_v(V, precision=precision)
        assert U.shape == (op.numVariants(), k) and Y.shape == (op.rows(), k)
        assert colwise_rel(U, Z.T @ X).max() < tol
        assert colwise_rel(Y, Z @ V).max() < tol
        if selection == "subset":
            pos5 = int(np.nonzero(variants == 5)[0][0])
            assert np.all(U[pos5] == 0.0)
    X = rng.standard_normal((op.rows(), 3))
    KX = op.multiply_Z_v(op.multiply_Zt_v(X)) / op.numVariants()
    assert colwise_rel(KX, op.apply(X)).max() < 1e-12
    with pytest.raises(cs.InvalidArgument):
        op.multiply_Z_v(np.zeros(op.numVariants() + 1))
    op.close()


def test_pcg_records_matches_dense_solve(data):
    torch = pytest.importorskip("torch")
    d, bed, ref, g = data
    n, m = d["n"], d["m"]
    rng = np.random.default_rng(9)
    counts = rng.integers(1, 4, size=n)
    rec = np.repeat(np.arange(n, dtype=np.int32), counts)
    rec[::97] = -1                               # records without a genotype row
    n_rec = len(rec)
    op = cs.createKinshipOperator(g)
    Z = ref.dense_z()
    K = Z @ Z.T / m
    Zr = np.zeros((n_rec, n))
    ok = rec >= 0
    Zr[np.nonzero(ok)[0], rec[ok]] = 1.0
    sg, spe, se = 0.6, 0.25, 0.4
    V = sg * Zr @ K @ Zr.T + spe * Zr @ Zr.T + se * np.eye(n_rec)
    B = rng.standard_normal((n_rec, 4))
    for precision, tol in (("fp64", 1e-9), ("mixed", 1e-6)):
        pcg = cs.MatrixFreePCG(op, sg, se, precision=precision, kinship_divisor=m,
                               rec_to_row=rec, with_pe=True, sigma2_pe=spe)
        X = pcg.solve(B, tol=1e-11, max_iter=3000)
        E = np.linalg.solve(V, B)
        assert colwise_rel(X, E).max() < tol, precision
        assert np.all(pcg.iterations > 0)
    op.close()


def test_facade_genotype_matrix_drives_stcg_solve(data, tmp_path):
    """The reference's STCG solve_V written against the facade's GenotypeMatrix."""
    torch = pytest.importorskip("torch")
    d, bed, ref, g = data
    n, m = d["n"], d["m"]
    bed_path = tmp_path / "g.bed"
    bed.tofile(bed_path)
    y = d["y"]
    y_path = tmp_path / "y.bin"
    y.astype(np.float64).tofile(y_path)
    out_path = tmp_path / "x.bin"
    sg, se = 0.55, 0.45
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "stcg_solve.cpp"
    src.write_text(r'''
#include "cosmicscanner_b200.hpp"
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iterator>
#include <vector>
static double dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}
int main(int argc, char** argv) {
    const long n = std::atol(argv[3]), m = std::atol(argv[4]);
    const double vg = std::atof(argv[5]), ve = std::atof(argv[6]);
    std::ifstream fb(argv[1], std::ios::binary);
    std::vector<unsigned char> bed((std::istreambuf_iterator<char>(fb)), {});
    std::ifstream fy(argv[2], std::ios::binary);
    std::vector<double> y(n);
    fy.read(reinterpret_cast<char*>(y.data()), 8 * n);
    auto g = cs::Genotypes::from_bed(bed.data(), bed.size(), n, m);
    cs::KinshipOperator op(g);
    cs::GenotypeMatrix geno(op);
    // STCG_VCE::apply_G (stcg_vce.cpp:80-87): Z (Z^T u) / cols
    auto apply_V = [&](const std::vector<double>& v, std::vector<double>& out) {
        std::vector<double> t, gu;
        geno.multiply_Zt_v(v, t);
        geno.multiply_Z_v(t, gu);
        out.resize(n);
        for (long i = 0; i < n; ++i) out[i] = vg * gu[i] / (double)geno.cols() + ve * v[i];
    };
    // MatrixFreePCG::solve (matrix_free_pcg.h:20-68), Jacobi 1/(vg + ve), absolute stop
    const double diag = vg + ve, tol = 1e-10;
    std::vector<double> x(n, 0.0), r(y), z(n), p(n), ap;
    for (long i = 0; i < n; ++i) z[i] = r[i] / diag;
    p = z;
    double rz = dot(r, z);
    int it = 0;
    for (; it < 2000; ++it) {
        apply_V(p, ap);
        const double alpha = rz / dot(p, ap);
        for (long i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * ap[i]; }
        if (std::sqrt(dot(r, r)) < tol) break;
        for (long i = 0; i < n; ++i) z[i] = r[i] / diag;
        const double rz2 = dot(r, z);
        for (long i = 0; i < n; ++i) p[i] = z[i] + (rz2 / rz) * p[i];
        rz = rz2;
    }
    std::ofstream fo(argv[7], std::ios::binary);
    fo.write(reinterpret_cast<const char*>(x.data()), 8 * n);
    std::printf("%d\n", it + 1);
    return 0;
}
''')
    exe = tmp_path / "stcg_solve"
    lib_dir = os.path.dirname(_abi.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(root, "include"), str(src),
                    "-o", str(exe), "-L", lib_dir, "-lcosmicscanner_b200",
                    f"-Wl,-rpath,{lib_dir}"], check=True)
    res = subprocess.run([str(exe), str(bed_path), str(y_path), str(n), str(m), str(sg), str(se),
                          str(out_path)], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    x_cpp = np.fromfile(out_path, dtype=np.float64)
    op = cs.createKinshipOperator(g)
    x_lib = cs.MatrixFreePCG(op, sg, se, kinship_divisor=m).solve(y, tol=1e-10, max_iter=2000)
    assert np.abs(x_cpp - x_lib).max() < 1e-9 * np.abs(x_lib).max()
    op.close()
