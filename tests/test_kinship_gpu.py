"""GPU kinship operator against the CPU oracle (the reference's batch-equivalence checks).

Mirrors tests/test_kinship_batch.cpp of the reference: the regenerated 37 x 1031 fixture,
six selections, RHS widths 1/7/41, relative error < 1e-10 against the dense Z Z^T / M,
transpose == apply, aliasing, bitwise repeatability, trace, empty RHS, bad dimensions.
"""
import ctypes

import numpy as np
import pytest

import oracle
from tests.test_oracle import M, N, compare, selections

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")


@pytest.fixture(scope="module")
def fixture():
    sels = selections()
    rows = [N if k is None else len(k) for k, _ in sels]
    bed, omega = oracle.kinship_batch_fixture(N, M, 8128, rows=rows)
    ref = oracle.Bed(bed[3:].reshape(M, -1), N)
    g = cs.Genotypes.from_bed_bytes(bed, N, M)
    return bed, omega, sels, rows, ref, g


def test_stats_bit_exact(fixture):
    *_, ref, g = fixture
    st = g.stats()
    assert np.array_equal(st["mean"], ref.mean)
    assert np.array_equal(st["inv_std"], ref.inv_std)
    assert np.array_equal(st["count"], ref.count)
    assert np.array_equal(st["sum"], ref.sum)


def test_batch_equivalence(fixture):
    bed, omega, sels, rows, ref, g = fixture
    off = 0
    for (keep, snps), r in zip(sels, rows):
        op = cs.createKinshipOperator(g, keep, snps)
        assert op.rows() == r and op.cols() == r
        assert op.numVariants() == (M if snps is None else len(snps))
        z = ref.dense_z(keep, snps)
        K = z @ z.T / z.shape[1]
        assert abs(op.trace() - np.trace(K)) < 1e-10
        compare(op.getDiagonal(), np.diag(K))
        for w in (1, 7, 41):
            om = omega[off:off + r * w].reshape(w, r).T
            off += r * w
            res = op.apply(om)
            compare(res, K @ om)
            compare(res, ref.apply_block(om, keep, snps))
            vec = op.apply(om[:, 0])
            compare(vec, K @ om[:, 0])
            compare(op.applyTranspose(om[:, 0]), vec)
            again = op.apply(om)
            assert np.array_equal(again, res), "repeat is not bitwise deterministic"
        empty = op.apply(np.zeros((r, 0)))
        assert empty.shape == (r, 0)
        with pytest.raises(cs.InvalidArgument):
            op.apply(np.zeros((r + 1, 1)))


def test_device_alias_and_wide_rhs(fixture):
    torch = pytest.importorskip("torch")
    bed, omega, sels, rows, ref, g = fixture
    op = cs.createKinshipOperator(g)
    rng = np.random.default_rng(7)
    for k in (1, 3, 8, 20, 33, 64, 65, 130, 266):
        X = rng.standard_normal((N, k))
        expect = ref.apply_block(X)
        t = torch.tensor(X.T.copy(), device="cuda")  # row-major (k, N) == column-major (N, k)
        op.apply_device(t.data_ptr(), N, k, t.data_ptr(), N)  # Y aliases X
        torch.cuda.synchronize()
        compare(t.cpu().numpy().T, expect)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_f32(fixture, precision):
    """cs_kinship_apply_f32: float X / Y (Y aliasing X) against the FP64 oracle rounded to
    float: within 1e-6 of the largest entry (float rounding plus the mixed form's bound)."""
    torch = pytest.importorskip("torch")
    bed, omega, sels, rows, ref, g = fixture
    op = cs.createKinshipOperator(g)
    rng = np.random.default_rng(11)
    for k in (1, 7, 41, 130):
        X = rng.standard_normal((N, k)).astype(np.float32)
        expect = ref.apply_block(X.astype(np.float64))
        t = torch.tensor(X.T.copy(), device="cuda")
        op.apply_device_f32(t.data_ptr(), N, k, t.data_ptr(), N, precision)
        torch.cuda.synchronize()
        got = t.cpu().numpy().T.astype(np.float64)
        assert np.abs(got - expect).max() <= 1e-6 * np.abs(expect).max(), (k, precision)


def test_selection_errors(fixture):
    *_, g = fixture
    with pytest.raises(cs.InvalidArgument):
        cs.createKinshipOperator(g, [0, N])
    with pytest.raises(cs.InvalidArgument):
        cs.createKinshipOperator(g, None, [M])
    with pytest.raises(cs.InvalidArgument):
        cs.createKinshipOperator(g, None, [-1])


def test_larger_random_matrix():
    synth = pytest.importorskip("cosmicscanner_b200.synth")
    d = synth.cohort(1500, 4000, 11, missing=0.02)
    ref = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    rng = np.random.default_rng(3)
    keep = np.sort(rng.choice(d["n"], 1100, replace=False))
    variants = np.arange(0, d["m"], 2)
    for kp, vp in ((None, None), (keep, variants)):
        op = cs.createKinshipOperator(g, kp, vp)
        X = rng.standard_normal((op.rows(), 70))
        compare(op.apply(X), ref.apply_block(X, kp, vp, n_threads=8))
        assert abs(op.trace() - ref.trace(kp, vp)) < 1e-9 * abs(ref.trace(kp, vp))


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_narrow_fp64_apply(k):
    """One to four right-hand sides take the decode-GEMV passes (every thread keeps its run of
    samples' values in registers): same result as the oracle, ragged sample counts across
    CTA chunks, a sample subset and a variant selection, bitwise repeatable."""
    synth = pytest.importorskip("cosmicscanner_b200.synth")
    d = synth.cohort(9000, 2100, 91, missing=0.02, n_causal=10)
    ref = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    rng = np.random.default_rng(k)
    keep = np.sort(rng.choice(d["n"], 8301, replace=False)).astype(np.int32)
    variants = np.sort(rng.choice(d["m"], 1900, replace=False)).astype(np.int32)
    for kp, vs in ((None, None), (keep, variants)):
        op = cs.createKinshipOperator(g, kp, vs)
        X = rng.standard_normal((op.rows(), k))
        E = ref.apply_block(X, kp, vs, n_threads=8)
        Y = op.apply(X)
        assert (np.abs(Y - E).max(axis=0) / np.abs(E).max(axis=0)).max() < 1e-12
        assert np.array_equal(op.apply(X), Y)
        op.close()


@pytest.mark.parametrize("k", [1, 16, 40])
def test_mixed_small_cohort_many_slices(k):
    """A small cohort against many SNPs: the tensor-core passes split the SNP contraction into
    many K slices to fill the GPU (300 samples are 3 tiles, 60,000 SNPs 469 K-blocks), with
    none left empty; the result equals the FP64 form to the mixed tolerance."""
    synth = pytest.importorskip("cosmicscanner_b200.synth")
    d = synth.cohort(300, 60000, 29, missing=0.02, n_causal=10)
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    op = cs.createKinshipOperator(g)
    rng = np.random.default_rng(k)
    X = rng.standard_normal((op.rows(), k))
    E = op.apply(X, precision="fp64")
    Y = op.apply(X, precision="mixed")
    assert (np.abs(Y - E).max(axis=0) / np.abs(E).max(axis=0)).max() < 1e-6
    assert np.array_equal(op.apply(X, precision="mixed"), Y)
    op.close()
