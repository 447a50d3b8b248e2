"""Multi-trait matrix-free REML (cs_mv_stcg_solve) against the oracle.

* Same probes: the oracle's dense restatement of the algorithm (oracle.mv_stcg_em: the EM update
  of MvEigenVce::updateEM, libCosmicCore/src/eigen_vce.cpp:551-604, written for V = Vg (x) K +
  Ve (x) I with the REML projection P, Hutchinson traces from the same mt19937_64 probe stream)
  must agree with the GPU's CG form to CG accuracy: Vg and Ve within 1e-7 of their largest entry
  (FP64 kinship applies), 1e-5 (tensor-core applies).
* The oracle's general form with exact traces equals the reference's eigenbasis EM to rounding
  (checked here too), and the stochastic GPU run stays near it: after the same number of EM
  iterations with 32 probes, every entry within 0.03 (about five times the spread of the trace
  noise observed at this size).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


@pytest.fixture(scope="module")
def data():
    d = synth.cohort(600, 2000, 15, missing=0.02, n_causal=100, h2=0.5)
    n, m = d["n"], d["m"]
    ref = oracle.Bed(d["bed"][3:].reshape(m, -1), n)
    Z = ref.dense_z()
    K = Z @ Z.T / m
    rng = np.random.default_rng(2)
    Y = np.column_stack([d["y"], 0.7 * d["y"] + 0.7 * rng.standard_normal(n),
                         rng.standard_normal(n)])
    X = d["X"].astype(np.float32).astype(np.float64)
    g = cs.Genotypes.from_bed_bytes(d["bed"], n, m)
    op = cs.createKinshipOperator(g)
    return d, K, Y, X, g, op


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-7), ("mixed", 1e-5)])
def test_same_probes_match_oracle(data, precision, tol):
    d, K, Y, X, g, op = data
    kw = dict(max_iter=4, tol=0.0, mc_samples=6, probe_seed=777)
    Vg_o, Ve_o, it, _ = oracle.mv_stcg_em(K, Y, X, **kw)
    Vg, Ve, r = cs.mv_stcg_solve(op, Y, X, kinship_divisor=d["m"], pcg_tol=1e-12,
                                 precision=precision, **kw)
    assert r["iterations"] == it == 4
    assert r["operator_columns"] >= r["operator_applies"] * 3 * (1 + 6) - 1
    scale = max(np.abs(Vg_o).max(), np.abs(Ve_o).max())
    assert np.abs(Vg - Vg_o).max() < tol * scale, (Vg, Vg_o)
    assert np.abs(Ve - Ve_o).max() < tol * scale, (Ve, Ve_o)
    assert np.allclose(Vg, Vg.T) and np.allclose(Ve, Ve.T)


def test_exact_form_equals_eigenbasis_em(data):
    d, K, Y, X, g, op = data
    Vg, Ve, _, _ = oracle.mv_stcg_em(K, Y[:, :2], X, max_iter=5, tol=0.0, exact_traces=True)
    D, W, UtY, UtX, Vg2, Ve2 = oracle.mv_eigen_vce_prepare(K, Y[:, :2], X, projection=True)
    for _ in range(5):
        Vg2, Ve2 = oracle.mv_em_step(D, UtY, Vg2, Ve2)
    assert np.abs(Vg - Vg2).max() < 1e-12 and np.abs(Ve - Ve2).max() < 1e-12


def test_stochastic_run_tracks_exact_em(data):
    d, K, Y, X, g, op = data
    Yt = Y[:, :2]
    Vg_x, Ve_x, _, _ = oracle.mv_stcg_em(K, Yt, X, max_iter=40, tol=0.0, exact_traces=True)
    Vg, Ve, r = cs.mv_stcg_solve(op, Yt, X, kinship_divisor=d["m"], max_iter=40, tol=0.0,
                                 mc_samples=32, precision="mixed")
    assert np.abs(Vg - Vg_x).max() < 0.03, (Vg, Vg_x)
    assert np.abs(Ve - Ve_x).max() < 0.03, (Ve, Ve_x)
    assert r["operator_applies"] > 40 and r["pcg_iterations"] > 0
