"""The dense-tier oracle checked against independent formulas, on the CPU: the GRM against a
vectorised VanRaden / Yang restatement, the Brent null model of the covariate-projected
eigenbasis against the one that keeps X (the two REML objectives differ by a constant), and
the exact scan against the dense GLS projection P = V^-1 - V^-1 X (X^T V^-1 X)^-1 X^T V^-1."""
import numpy as np
import pytest

import oracle

synth = pytest.importorskip("cosmicscanner_b200.synth")


@pytest.fixture(scope="module")
def small():
    d = synth.cohort(120, 400, 23, missing=0.04, n_causal=8, h2=0.6)
    bed = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    return d, bed


def dosages(bed):
    codes = oracle._codes(bed.rows, bed.n)
    x = np.array([2.0, np.nan, 1.0, 0.0])[codes]  # SNP x sample
    return x


@pytest.mark.parametrize("algorithm", [1, 0])
def test_grm_oracle_vs_formula(small, algorithm):
    d, bed = small
    x = dosages(bed)
    obs = ~np.isnan(x)
    f = np.nansum(x, axis=1) / (2.0 * obs.sum(axis=1))
    maf = np.minimum(f, 1 - f)
    ok = (maf >= np.float32(0.01)) & (maf > 1e-8)
    mean = (2 * f).astype(np.float32).astype(np.float64)
    Z = np.where(obs, x - mean[:, None], 0.0)[ok]
    if algorithm == 0:
        s = (1.0 / np.sqrt(2 * f * (1 - f))).astype(np.float32).astype(np.float64)
        Z = Z * s[ok][:, None]
        G = Z.T @ Z / ok.sum()
    else:
        G = Z.T @ Z / (2 * f * (1 - f)).astype(np.float32)[ok].astype(np.float64).sum()
    G_o, nv, s2 = oracle.grm_dense(bed, algorithm=algorithm)
    assert nv == ok.sum()
    assert np.abs(G_o - G).max() < 1e-12 * np.abs(G).max()


def test_projection_and_gls_routes_agree(small):
    d, bed = small
    G, _, _ = oracle.grm_dense(bed)
    y, X = d["y"], d["X"].astype(np.float32).astype(np.float64)
    Dp, _, Utyp, UtXp = oracle.eigen_vce_prepare(G, y, X, True)
    a = oracle.solve_diagonal(Dp, Utyp, UtXp)
    D, W, Uty, UtX = oracle.eigen_vce_prepare(G, y, X, False)
    b = oracle.solve_diagonal(D, Uty, UtX)
    # the golden search stops within 1e-5 in log10 delta
    assert abs(np.log10(a["delta"]) - np.log10(b["delta"])) < 2e-5
    assert abs(a["sigma2_g"] - b["sigma2_g"]) < 1e-4 * b["sigma2_g"]


def test_exact_scan_oracle_vs_dense_gls(small):
    d, bed = small
    n = d["n"]
    G, _, _ = oracle.grm_dense(bed)
    y, X = d["y"], d["X"].astype(np.float32).astype(np.float64)
    D, W, Uty, UtX = oracle.eigen_vce_prepare(G, y, X, True)
    r = oracle.solve_diagonal(D, Uty, UtX)
    sg, se = r["sigma2_g"], r["sigma2_e"]
    out = oracle.scan_exact(bed, np.arange(n), W, D, Uty, UtX, sg, se)
    V = sg * G + se * np.eye(n)
    Vi = np.linalg.inv(V)
    P = Vi - Vi @ X @ np.linalg.inv(X.T @ Vi @ X) @ X.T @ Vi
    x = dosages(bed)
    obs = ~np.isnan(x)
    mean = np.nansum(x, axis=1) / obs.sum(axis=1)
    g = np.where(obs, x - mean[:, None], 0.0).T  # sample x SNP
    score = g.T @ (P @ y)
    var = np.einsum("ij,ij->j", g, P @ g)
    t = out["tested"]
    assert t.sum() > 300
    np.testing.assert_allclose(out["beta"][t], (score / var)[t], rtol=1e-8, atol=1e-12)
    np.testing.assert_allclose(out["se"][t], (1 / np.sqrt(var))[t], rtol=1e-8)


def test_mv_em_oracle_properties(small):
    """MvEigenVce's EM restatement: the REML log-likelihood never decreases along the EM
    iterations, AI-REML ends at least as high, and with one trait the EM fixed point is the
    single-trait Brent REML estimate."""
    d, bed = small
    G, _, _ = oracle.grm_dense(bed)
    rng = np.random.default_rng(5)
    Y = np.column_stack([d["y"], 0.3 * d["y"] + rng.standard_normal(len(d["y"]))])
    X = d["X"].astype(np.float32).astype(np.float64)
    D, W, UtY, UtX, Vg, Ve = oracle.mv_eigen_vce_prepare(G, Y, X)
    ll = [oracle.mv_loglik(D, UtY, Vg, Ve)]
    for _ in range(30):
        Vg, Ve = oracle.mv_em_step(D, UtY, Vg, Ve)
        ll.append(oracle.mv_loglik(D, UtY, Vg, Ve))
    assert all(b >= a - 1e-9 for a, b in zip(ll, ll[1:]))
    D, W, UtY, UtX, Vg0, Ve0 = oracle.mv_eigen_vce_prepare(G, Y, X)
    em = oracle.mv_run_null(D, UtY, Vg0, Ve0)
    ai = oracle.mv_run_null(D, UtY, Vg0, Ve0, aireml=True)
    assert em[0] and ai[6] >= em[6] - 1e-6
    # one trait: EM -> the Brent REML estimate
    D1, _, Uty1, UtX1, vg, ve = oracle.mv_eigen_vce_prepare(G, Y[:, :1], X)
    r = oracle.mv_run_null(D1, Uty1, vg, ve, max_iter=20000, tol=1e-16)
    b = oracle.solve_diagonal(D1, Uty1[:, 0], UtX1)
    assert abs(r[2][0, 0] - b["sigma2_g"]) < 1e-3 * b["sigma2_g"]
    assert abs(r[3][0, 0] - b["sigma2_e"]) < 1e-3 * b["sigma2_e"]
