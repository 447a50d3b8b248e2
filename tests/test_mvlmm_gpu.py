"""Multi-trait LMM scan with a fixed null (MvLmmEngine::scan(PlinkReader),
src/mvlmm_engine.cpp:756-931) on the GPU against the oracle restatement, given the same
eigenbasis, eigenvalues, rotated phenotypes / covariates and Vg, Ve.  FP64 rotation: beta,
Var(beta) and Wald within 1e-8 relative, P within 1e-10, statuses and FREQ exact; the
tensor-core rotation: Wald and beta within 1e-5 relative."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


@pytest.fixture(scope="module")
def setup():
    d = synth.cohort(400, 900, 61, missing=0.02, n_causal=40)
    n, m = d["n"], d["m"]
    ref = oracle.Bed(d["bed"][3:].reshape(m, -1), n)
    Zs = ref.dense_z()
    K = Zs @ Zs.T / m
    D, W = np.linalg.eigh(K)
    keep_r = D > 1e-8          # the projected basis (W has fewer columns than rows)
    D, W = D[keep_r], W[:, keep_r]
    rng = np.random.default_rng(9)
    t = 3
    Y = np.column_stack([d["y"] + 0.4 * rng.standard_normal(n) for _ in range(t)])
    X = d["X"]
    A = rng.standard_normal((t, t))
    Vg = A @ A.T / t + 0.2 * np.eye(t)
    B = rng.standard_normal((t, t))
    Ve = B @ B.T / t + 0.5 * np.eye(t)
    g = cs.Genotypes.from_bed_bytes(d["bed"], n, m)
    args = (np.arange(n, dtype=np.int32), W, D, W.T @ Y, W.T @ X, Vg, Ve)
    return d, ref, g, args


@pytest.mark.parametrize("window", [(0, 900), (100, 357)])
def test_mvlmm_fp64_matches_oracle(setup, window):
    d, ref, g, args = setup
    b, e = window
    o = oracle.mvlmm_scan(ref, *args, snp_begin=b, snp_end=e)
    out = cs.mvlmm_scan(g, *args, snp_begin=b, snp_end=e, precision="fp64")
    assert np.array_equal(out["status"], o["status"])
    assert np.array_equal(out["freq"], o["freq"])
    ok = o["status"] < 3
    assert ok.sum() > 0.9 * (e - b)
    sc = np.abs(o["beta"][ok]).max()
    assert np.abs(out["beta"][ok] - o["beta"][ok]).max() <= 1e-8 * sc
    assert np.abs(out["cov"][ok] - o["cov"][ok]).max() <= 1e-8 * np.abs(o["cov"][ok]).max()
    assert np.abs(out["wald"][ok] - o["wald"][ok]).max() <= 1e-8 * o["wald"][ok].max()
    assert np.abs(out["p"][ok] - o["p"][ok]).max() < 1e-10


def test_mvlmm_mixed_rotation(setup):
    d, ref, g, args = setup
    o = cs.mvlmm_scan(g, *args, precision="fp64")
    out = cs.mvlmm_scan(g, *args, precision="mixed")
    ok = o["status"] < 3
    assert np.array_equal(out["status"][ok] < 3, np.ones(ok.sum(), bool))
    assert np.abs(out["wald"][ok] - o["wald"][ok]).max() <= 1e-5 * o["wald"][ok].max()
    assert np.abs(out["beta"][ok] - o["beta"][ok]).max() <= 1e-5 * np.abs(o["beta"][ok]).max()
