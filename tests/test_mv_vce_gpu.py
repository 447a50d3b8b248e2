"""Multi-trait dense null on the GPU against the numpy oracle: MvEigenVce::prepare, the EM and
AI-REML null models (libCosmicCore/src/eigen_vce.cpp:496-911, 1031-1065) and the mvLMM scan
from its device eigenbasis (src/mvlmm_engine.cpp:195-207, 756-931).

Tolerances: eigenvalues 1e-10 of the largest; the EM estimate Vg / Ve 1e-7 relative to their
largest entry with the same iteration count; the log-likelihood 1e-9 relative; AI-REML Vg / Ve
1e-6 and SEs 1e-5; the scan from the handle equal to cs_mvlmm_scan on the same null to 1e-12,
and to the oracle's scan as the existing mvLMM tests (1e-8 relative Wald)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


@pytest.fixture(scope="module")
def data():
    d = synth.cohort(360, 1800, 23, missing=0.02, n_causal=25, h2=0.5)
    bed = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    rng = np.random.default_rng(8)
    n = d["n"]
    Y = np.column_stack([d["y"], 0.5 * d["y"] + rng.standard_normal(n),
                         rng.standard_normal(n)])
    X = d["X"].astype(np.float32).astype(np.float64)
    keep = np.sort(rng.choice(n, 330, replace=False)).astype(np.int32)
    return d, bed, g, Y, X, keep


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("aireml", [False, True])
def test_mv_null_matches_oracle(data, aireml):
    d, bed, g, Y, X, keep = data
    G, _, _ = oracle.grm_dense(bed)
    Gk = G[np.ix_(keep, keep)]
    D_o, W_o, UtY_o, UtX_o, Vg0, Ve0 = oracle.mv_eigen_vce_prepare(Gk, Y[keep], X[keep])
    conv, it, Vg_o, Ve_o, sg_o, se_o, ll_o = oracle.mv_run_null(D_o, UtY_o, Vg0, Ve0,
                                                               aireml=aireml)
    b = cs.GrmBuilder().compute(g)
    v = cs.MvEigenVce(aireml=aireml).prepare(Y[keep], X[keep], b, keep)
    assert v.n_eig == len(D_o) and v.d == 3
    assert np.abs(v.getEigenvalues() - D_o).max() < 1e-10 * D_o.max()
    assert v.runNullModel() == conv
    assert v.iterations == it
    tol = 1e-6 if aireml else 1e-7
    assert rel(v.getVg(), Vg_o) < tol and rel(v.getVe(), Ve_o) < tol
    assert abs(v.logl - ll_o) <= 1e-9 * abs(ll_o)
    if aireml:
        assert rel(v.getVgSE(), sg_o) < 1e-5 and rel(v.getVeSE(), se_o) < 1e-5
    v.close()
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mv_scan_from_vce(data, precision):
    d, bed, g, Y, X, keep = data
    b = cs.GrmBuilder().compute(g)
    v = cs.MvEigenVce().prepare(Y[keep], X[keep], b, keep)
    assert v.runNullModel()
    out = v.scan(g, keep, 200, 1500, precision=precision)
    # the same null handed over as host arrays
    e = cs.EigenVce()  # only for the basis: W is the multi-trait basis of the same G
    e.prepare(Y[keep, 0], X[keep], b, keep)
    W = e.getProjectedW()
    ref = cs.mvlmm_scan(g, keep, W, v.getEigenvalues(), v.getUty(), np.zeros((v.n_eig, 0)),
                        v.getVg(), v.getVe(), 200, 1500, precision=precision)
    assert np.array_equal(out["status"], ref["status"])
    ok = out["status"] != 3
    assert rel(out["wald"][ok], ref["wald"][ok]) < 1e-12
    exp = oracle.mvlmm_scan(bed, keep, W, v.getEigenvalues(), v.getUty(),
                            np.zeros((v.n_eig, 0)), v.getVg(), v.getVe(), 200, 1500)
    ok = exp["status"] != 3
    tol = 1e-8 if precision == "fp64" else 1e-5
    assert rel(out["wald"][ok], exp["wald"][ok]) < tol
    assert rel(out["beta"][ok], exp["beta"][ok]) < tol
    v.close()
    e.close()
    b.close()


def test_mv_errors(data):
    d, bed, g, Y, X, keep = data
    b = cs.GrmBuilder().compute(g)
    with pytest.raises(cs.CosmicError, match="traits"):
        cs.MvEigenVce().prepare(np.ones((len(keep), 9)), X[keep], b, keep)
    with pytest.raises(cs.CosmicError, match="projection"):
        cs.MvEigenVce(use_projection=False).prepare(Y[keep], X[keep], b, keep)
    v = cs.MvEigenVce(max_iter=3).prepare(Y[keep], X[keep], b, keep)
    assert not v.runNullModel() and v.iterations == 3
