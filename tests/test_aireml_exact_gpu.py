"""The matrix-free AI-REML (PCG + Hutchinson, STCG_VCE with one record per sample) against
exact REML.

The exact reference is EigenVce::runIterativeReml (libCosmicCore/src/eigen_vce.cpp:155-252),
restated in the oracle: AI-REML in the eigenbasis of the covariate-projected dense kinship
A'KA with K = Z Z^T / M, the same K the matrix-free operator applies.  The matrix-free route
estimates tr(P dV) with Rademacher probes, so its variance components differ from the exact
ones by a stochastic error.  Its size is predicted from the exact solution: the trace
estimates' covariance 2/S sum_{i!=j} A_ij B_ij (S probes, A and B the symmetrised P K and P)
mapped through the inverse expected information (oracle.hutchinson_vc_sd).  The route runs the
reference's default 50 iterations (probes are redrawn every iteration and the AI step is
blended by 0.35, so the iterate settles around the exact solution) with 30 and 64 probes; each
variance component must lie within 4 predicted standard deviations of exact REML, and the
predicted deviation must shrink with the probe count.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


@pytest.fixture(scope="module")
def exact():
    d = synth.cohort(2000, 6000, 61, missing=0.01, n_causal=200, h2=0.5)
    n, m = d["n"], d["m"]
    ref = oracle.Bed(d["bed"][3:].reshape(m, -1), n)
    Z = ref.dense_z()
    K = Z @ Z.T / m
    X = d["X"].astype(np.float32).astype(np.float64)
    D, W, Uty, UtX = oracle.eigen_vce_prepare(K, d["y"], X, projection=True)
    ex = oracle.eigen_vce_iterative_reml(D, Uty, UtX, average_information=True)
    assert ex["converged"]
    g = cs.Genotypes.from_bed_bytes(d["bed"], n, m)
    return d, K, X, ex, g


def test_exact_reml_oracle_is_a_stationary_point(exact):
    d, K, X, ex, g = exact
    # the score at the exact solution vanishes relative to the information
    step = np.linalg.solve(ex["ai"], ex["score"])
    assert np.abs(step).max() < 1e-6 * max(ex["sigma2_g"], ex["sigma2_e"])


@pytest.mark.parametrize("probes", [30, 64])
def test_matrix_free_aireml_within_stochastic_error(exact, probes):
    d, K, X, ex, g = exact
    sd = oracle.hutchinson_vc_sd(K, X, ex["sigma2_g"], ex["sigma2_e"], probes)
    op = cs.createKinshipOperator(g)
    vce = cs.StcgVce()
    r = vce.solve(op, d["y"], X, kinship_divisor=d["m"], max_iter=50, mc_samples=probes,
                  slq_probes=0)
    err = np.array([r["sigma2_g"] - ex["sigma2_g"], r["sigma2_e"] - ex["sigma2_e"]])
    assert np.all(np.abs(err) <= 4.0 * sd), (probes, err, sd)
    vce.close()
    op.close()


def test_predicted_error_shrinks_with_probes(exact):
    d, K, X, ex, g = exact
    s30 = oracle.hutchinson_vc_sd(K, X, ex["sigma2_g"], ex["sigma2_e"], 30)
    s64 = oracle.hutchinson_vc_sd(K, X, ex["sigma2_g"], ex["sigma2_e"], 64)
    assert np.allclose(s64, s30 * np.sqrt(30 / 64), rtol=1e-12)
