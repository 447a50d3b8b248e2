"""Edge cases across the GPU paths: a sample count that is not a multiple of 4 (a ragged last
byte per SNP), SNPs that are all missing or monomorphic (the GRM skips them, the scans report
no row), empty and single-SNP scan windows, and an empty apply.  Compared with the oracle
at the tolerances of the main parity tests."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


def set_row(bed, n, j, code):
    """Sets every sample of SNP j to one 2-bit code (1 = missing)."""
    stride = (n + 3) // 4
    byte = code | (code << 2) | (code << 4) | (code << 6)
    bed[3 + j * stride:3 + (j + 1) * stride] = byte


@pytest.fixture(scope="module")
def ragged():
    n, m = 403, 1200
    d = synth.cohort(n, m, 77, missing=0.03, n_causal=20, h2=0.5)
    bed = d["bed"].copy()
    set_row(bed, n, 5, 1)     # all missing
    set_row(bed, n, 17, 0)    # monomorphic: every sample hom A1
    set_row(bed, n, 600, 3)   # monomorphic: every sample hom A2
    ref = oracle.Bed(bed[3:].reshape(m, -1), n)
    g = cs.Genotypes.from_bed_bytes(bed, n, m)
    return d, bed, ref, g


def test_ragged_grm_and_exact_scan(ragged):
    d, bed, ref, g = ragged
    n = d["n"]
    G_o, nv, s2 = oracle.grm_dense(ref)
    b = cs.GrmBuilder().compute(g)
    assert b.getTotalSnps() == nv == d["m"] - 3
    G = b.getGrm()
    assert np.abs(G - G_o).max() < 1e-12 * np.abs(G_o).max()
    keep = np.arange(n, dtype=np.int32)
    y, X = d["y"], d["X"].astype(np.float32).astype(np.float64)
    v = cs.EigenVce().prepare(y, X, b)
    v.runNullModel()
    eng = cs.LmmEngine()
    eng.prepareFromVce(v)
    for prec, tol in (("fp64", 1e-6), ("mixed", 1e-3)):
        out = eng.scan(g, keep, precision=prec)
        exp = oracle.scan_exact(ref, keep, v.getProjectedW(), v.getEigenvalues(), v.getUty(),
                                v.getUtX(), v.getSigma2g(), v.getSigma2e())
        t = exp["tested"]
        assert np.array_equal(out["tested"], t)
        assert not t[[5, 17, 600]].any()
        assert np.isnan(out["p"][[5, 17, 600]]).all()
        assert np.abs(out["log10p"][t] - exp["log10p"][t]).max() < tol
    # empty and single-SNP windows
    w = eng.scan_window(g, keep, 40, 40, precision="mixed")
    assert all(len(w[k]) == 0 for k in ("beta", "p", "tested"))
    w1 = eng.scan_window(g, keep, 41, 42, precision="fp64")
    full = eng.scan(g, keep, precision="fp64")
    assert w1["tested"][0] == full["tested"][41]
    assert abs(w1["beta"][0] - full["beta"][41]) <= 1e-12 * abs(full["beta"][41])


def test_ragged_lowrank_scan(ragged):
    d, bed, ref, g = ragged
    n = d["n"]
    y, X = d["y"], d["X"].astype(np.float32).astype(np.float64)
    op = cs.createKinshipOperator(g)
    eng = cs.LmmEngine()
    eng.prepareLowRankMatrixFree(y, X, op, rank=25, precision="mixed")
    U, lam, res = ref.lowrank_prepare(y, X, 25)
    keep = np.arange(n)
    out = eng.scan(g, keep, precision="mixed")
    exp = ref.scan_lowrank(keep, U, lam, res.residual_eigenvalue, res.sigma2_g, res.sigma2_e, y, X)
    t = exp["tested"]
    assert np.array_equal(out["tested"], t) and not t[[5, 17, 600]].any()
    assert np.abs(out["log10p"][t] - exp["log10p"][t]).max() < 1e-3
    w = eng.scan_window(g, keep.astype(np.int32), 7, 7, precision="mixed")
    assert len(w["tested"]) == 0


def test_empty_apply(ragged):
    d, bed, ref, g = ragged
    op = cs.createKinshipOperator(g)
    out = op.apply(np.zeros((d["n"], 0)))
    assert out.shape == (d["n"], 0)
