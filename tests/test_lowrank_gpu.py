"""Low-rank matrix-free null model + scan on the GPU against the CPU oracle.

Both follow LmmEngine::prepareLowRankMatrixFree / scanLowRank (src/lmm_engine.cpp:
897-1361) on the same inputs: the same Omega (mt19937_64 seed 42 through libstdc++'s
normal_distribution), the same rank selection and REML search.  Tolerances: eigenvalues
and trace 1e-8 relative, variance components 1e-6 relative, BETA/SE 1e-6 relative,
-log10 P 1e-6 absolute, FREQ and the tested set exact.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def data():
    d = synth.cohort(700, 3000, 5, missing=0.02, n_causal=50, h2=0.5)
    ref = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    return d, ref, g


@pytest.mark.parametrize("subset", [False, True])
def test_prepare_and_scan_match_oracle(data, subset):
    d, ref, g = data
    n = d["n"]
    if subset:
        rng = np.random.default_rng(9)
        keep = np.sort(rng.choice(n, 520, replace=False)).astype(np.int32)
        variants = np.arange(0, d["m"], 3, dtype=np.int32)
    else:
        keep = np.arange(n, dtype=np.int32)
        variants = None
    y = d["y"][keep]
    X = d["X"][keep].astype(np.float32).astype(np.float64)
    rank = 40
    U_o, lam_o, res = ref.lowrank_prepare(y, X, rank, keep=None if not subset else keep,
                                          variants=variants, n_threads=8)
    op = cs.createKinshipOperator(g, None if not subset else keep, variants)
    eng = cs.LmmEngine()
    diag = eng.prepareLowRankMatrixFree(y, X, op, rank=rank)
    assert diag["effective_rank"] == res.rank
    assert diag["sketch_size"] == res.sketch_size
    assert diag["trace_threshold_met"] == res.trace_threshold_met
    assert abs(diag["trace"] - res.trace) <= 1e-10 * res.trace
    U_g, lam_g = eng.lowrank_basis()
    assert rel(lam_g, lam_o) < 1e-8
    assert abs(diag["residual_eigenvalue"] - res.residual_eigenvalue) <= 1e-8 * res.residual_eigenvalue
    # same low-rank operator: U diag(l) U^T v
    v = np.random.default_rng(1).standard_normal(len(y))
    assert rel(U_g @ (lam_g * (U_g.T @ v)), U_o @ (lam_o * (U_o.T @ v))) < 1e-7
    for key in ("sigma2_g", "sigma2_e", "delta"):
        assert abs(diag[key] - getattr(res, key)) <= 1e-5 * abs(getattr(res, key)), key
    # scan (all SNPs, analysed samples = keep)
    out = eng.scan(g, keep, min_maf=0.01)
    exp = ref.scan_lowrank(keep, U_o, lam_o, res.residual_eigenvalue, res.sigma2_g,
                           res.sigma2_e, y, X, min_maf=0.01)
    assert np.array_equal(out["tested"], exp["tested"])
    t = exp["tested"]
    assert t.sum() > 0.9 * d["m"]
    assert np.array_equal(out["freq"][t], exp["freq"][t])
    assert rel(out["beta"][t], exp["beta"][t]) < 1e-5
    assert rel(out["se"][t], exp["se"][t]) < 1e-5
    assert np.abs(out["log10p"][t] - exp["log10p"][t]).max() < 1e-4


def test_invalid_rank(data):
    d, ref, g = data
    op = cs.createKinshipOperator(g)
    eng = cs.LmmEngine()
    with pytest.raises(cs.InvalidArgument):
        eng.prepareLowRankMatrixFree(d["y"], d["X"], op, rank=d["n"])
    with pytest.raises(cs.InvalidArgument):
        eng.prepareLowRankMatrixFree(d["y"], d["X"], op, rank=0)


@pytest.mark.parametrize("n,cols", [(37, 1), (1000, 7), (20000, 13), (2, 1)])
def test_device_normal_stream_matches_libstdcxx(n, cols):
    """The device engine + polar transform reproduce std::normal_distribution over
    std::mt19937_64 (uniforms and acceptance bit-exact; log/sqrt within an ulp or two)."""
    for seed in (42, 8128, 20250101):
        got = cs.normal_matrix(seed, n, cols)
        ref = oracle.normal_matrix(seed, n, cols)
        assert np.abs(got - ref).max() <= 4e-16 * np.abs(ref).max()


@pytest.mark.parametrize("n,cols,seed", [(50000, 40, 42), (100000, 266, 8128), (200000, 266, 42)])
def test_device_normal_stream_parallel_chunks(n, cols, seed):
    """Streams longer than one chunk of the engine (1,048,320 draws) are drawn in parallel from
    jumped windows: 3, 33 and 66 chunks (the last beyond the 64-chunk table, finished
    sequentially) must still equal std::normal_distribution over std::mt19937_64."""
    got = cs.normal_matrix(seed, n, cols)
    ref = oracle.normal_matrix(seed, n, cols)
    assert np.abs(got - ref).max() <= 4e-16 * np.abs(ref).max()
