"""Serving loop: requests on cohort subsets with continuous batching of kinship applies.

Each request is the matrix-free LMM job on its subset (low-rank sketch of the subset's
kinship, REML per trait, scan of a SNP window).  Checks: one request against the CPU oracle
of the same job (src/lmm_engine.cpp:897-1361 restated; variance components 1e-5 relative, BETA 1e-5, -log10 P
1e-4); every request of a concurrent mix
against the same request run alone (the stacked applies keep columns independent, so the
results agree to FP64 rounding: 1e-9); the batcher really stacked requests; cohorts below
half the resident samples run on their own repacked subset operator; bad requests fail
before any work.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def data():
    d = synth.cohort(900, 2500, 41, missing=0.02, n_causal=60, h2=0.5)
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    variants = cs.grm_variant_selection(g.stats(), 0.01)
    ref = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    return d, g, variants, ref


def make_request(d, seed, n_sub, traits):
    rng = np.random.default_rng(seed)
    S = np.sort(rng.choice(d["n"], n_sub, replace=False)).astype(np.int32)
    Y = np.column_stack([d["y"][S] + 0.3 * t * rng.standard_normal(n_sub) for t in range(traits)])
    X = np.column_stack([np.ones(n_sub), rng.standard_normal(n_sub)]).astype(np.float32).astype(np.float64)
    b = int(rng.integers(0, d["m"] - 600))
    return S, Y, X, b, b + 600


@pytest.mark.parametrize("n_sub", [640, 300])
def test_request_matches_oracle(data, n_sub):
    """640 of 900 samples share the full-space applies; 300 (below half) run on their own
    repacked subset operator."""
    d, g, variants, ref = data
    S, Y, X, b, e = make_request(d, 1, n_sub, 2)
    srv = cs.Server(g, variants, rank=40, precision="fp64", max_active=2)
    rid = srv.submit(S, Y, X, b, e)
    st = srv.wait(rid)
    assert st["state"] == 2 and st["latency_s"] > 0
    assert srv.stats()["own_view_requests"] == (1 if n_sub < 450 else 0)
    wbed = oracle.Bed(d["bed"][3:].reshape(d["m"], -1)[b:e], d["n"])
    for t in range(2):
        U, lam, res = ref.lowrank_prepare(Y[:, t], X, 40, keep=S, variants=variants, n_threads=8)
        out = srv.result(rid, t)
        assert abs(out["sigma2_g"] - res.sigma2_g) <= 1e-5 * res.sigma2_g
        assert abs(out["sigma2_e"] - res.sigma2_e) <= 1e-5 * res.sigma2_e
        o = wbed.scan_lowrank(S, U, lam, res.residual_eigenvalue, res.sigma2_g, res.sigma2_e,
                              Y[:, t], X)
        assert np.array_equal(out["tested"], o["tested"])
        m = o["tested"]
        assert np.array_equal(out["freq"][m], o["freq"][m])
        assert rel(out["beta"][m], o["beta"][m]) < 1e-5
        assert np.abs(out["log10p"][m] - o["log10p"][m]).max() < 1e-4
    srv.release(rid)
    srv.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mix_equals_alone(data, precision):
    d, g, variants, ref = data
    reqs = [make_request(d, 10 + i, n, t) for i, (n, t) in
            enumerate([(700, 1), (450, 3), (880, 2), (300, 1), (520, 2)])]
    alone = cs.Server(g, variants, rank=30, precision=precision, max_active=1)
    solo = []
    for S, Y, X, b, e in reqs:
        rid = alone.submit(S, Y, X, b, e)
        alone.wait(rid)
        solo.append([alone.result(rid, t) for t in range(Y.shape[1])])
    alone.close()
    # a batching window holds each stack open until every running request waits on an apply
    mix = cs.Server(g, variants, rank=30, precision=precision, max_active=5, batch_window_ms=50.0)
    ids = [mix.submit(S, Y, X, b, e) for S, Y, X, b, e in reqs]
    for rid in ids:
        assert mix.wait(rid)["state"] == 2
    stats = mix.stats()
    assert stats["completed"] == len(reqs) and stats["failed"] == 0
    assert stats["max_requests_per_apply"] >= 2  # applies of different requests were stacked
    assert stats["own_view_requests"] == 1      # the 300-sample cohort (< N / 2)
    assert stats["memory_budget_gb"] > 0
    assert 0 < stats["p50_s"] <= stats["p99_s"]
    for rid, (S, Y, X, b, e), ref_out in zip(ids, reqs, solo):
        for t in range(Y.shape[1]):
            out = mix.result(rid, t)
            assert abs(out["sigma2_g"] - ref_out[t]["sigma2_g"]) <= 1e-9 * ref_out[t]["sigma2_g"]
            m = ref_out[t]["tested"]
            assert np.array_equal(out["tested"], m)
            assert np.abs(out["log10p"][m] - ref_out[t]["log10p"][m]).max() < 1e-9
    mix.close()


def test_bad_requests_rejected(data):
    d, g, variants, ref = data
    srv = cs.Server(g, variants, rank=20)
    S = np.arange(100, dtype=np.int32)
    Y = np.random.default_rng(0).standard_normal(100)
    X = np.ones((100, 1))
    with pytest.raises(cs.InvalidArgument):
        srv.submit(np.r_[S[:-1], 0], Y, X)  # duplicate sample
    with pytest.raises(cs.InvalidArgument):
        srv.submit(S, Y, X, 0, d["m"] + 1)  # window out of range
    with pytest.raises(cs.InvalidArgument):
        srv.submit(np.r_[S[:-1], d["n"]], Y, X)  # sample out of range
    srv.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_multi_trait_shares_projection(data, precision, tol):
    """A request's later traits take their py column from the first scan's projection of
    every trait's y; each agrees with the same trait requested alone (its own projection)."""
    d, g, variants, ref = data
    S, Y, X, b, e = make_request(d, 99, 600, 4)
    srv = cs.Server(g, variants, rank=30, precision=precision, max_active=1)
    rid = srv.submit(S, Y, X, b, e)
    assert srv.wait(rid)["state"] == 2
    multi = [srv.result(rid, t) for t in range(4)]
    for t in range(4):
        one = srv.submit(S, Y[:, t:t + 1].copy(), X, b, e)
        assert srv.wait(one)["state"] == 2
        alone = srv.result(one, 0)
        m = alone["tested"]
        assert np.array_equal(multi[t]["tested"], m)
        assert abs(multi[t]["sigma2_g"] - alone["sigma2_g"]) <= 1e-12 * alone["sigma2_g"]
        assert rel(multi[t]["beta"][m], alone["beta"][m]) < tol
        assert np.abs(multi[t]["log10p"][m] - alone["log10p"][m]).max() < 10 * tol
    srv.close()
