"""The small single-trait configuration end to end on the GPU against the oracle.

Cohort: N=2,000 samples, M=10,000 SNPs, MAF ~ U(0.05, 0.5), 1% missing calls,
X = [intercept, N(0,1)], 100 causal SNPs, h2 = 0.5 (``synth.config1``).

* Decode and statistics: per-SNP means, 1/sd, observed counts and allele sums bit-exact.
* Low-rank matrix-free route (`gwas --model lmm --fastlmm --fastlmm-matrix-free`, rank 256 +
  10 oversampling, seed 42): the FP64 and the mixed (tensor-core) forms against the oracle's
  restatement of prepareLowRankMatrixFree + scanLowRank on the same inputs.  Tolerances: rank
  equal; variance components, BETA and SE within 1e-5 relative (BETA / SE as max |delta| over
  max |value|); -log10 P within 1e-4 absolute (FP64) and 1e-3 (mixed); the tested set and FREQ
  identical.
* PCG + Hutchinson AI-REML (STCG_VCE with one record per sample, 30 Rademacher probes, SLQ
  log-likelihood with 30 probes x 15 steps, six iterations: four EM warm-up steps and two AI
  steps): the FP64 and mixed forms against the oracle's restatement with the same probe streams
  (the oracle applies K as a dense Z Z^T / M to keep its CG steps fast).  Variance components
  and fixed effects within 1e-5 relative, the log-likelihood within 1e-6 relative.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


@pytest.fixture(scope="module")
def cfg1():
    d = synth.config1()
    n, m = d["n"], d["m"]
    ref = oracle.Bed(d["bed"][3:].reshape(m, -1), n)
    g = cs.Genotypes.from_bed_bytes(d["bed"], n, m)
    X = d["X"].astype(np.float32).astype(np.float64)
    return d, ref, g, X


def test_config1_stats_bit_exact(cfg1):
    d, ref, g, X = cfg1
    st = g.stats()
    assert np.array_equal(st["mean"], ref.mean)
    assert np.array_equal(st["inv_std"], ref.inv_std)
    assert np.array_equal(st["count"], ref.count)
    assert np.array_equal(st["sum"], ref.sum)


@pytest.fixture(scope="module")
def lowrank_oracle(cfg1):
    d, ref, g, X = cfg1
    variants = cs.grm_variant_selection(g.stats(), 0.01)
    exp = oracle.lowrank_job_blas(ref, d["y"], X, variants=variants, rank=256, oversample=10)
    return variants, exp


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config1_lowrank_route(cfg1, lowrank_oracle, precision):
    d, ref, g, X = cfg1
    variants, exp = lowrank_oracle
    n = d["n"]
    op = cs.KinshipOperator(g, None, variants)
    eng = cs.LmmEngine()
    diag = eng.prepareLowRankMatrixFree(d["y"], X, op, rank=256, oversample=10,
                                        precision=precision)
    assert diag["effective_rank"] == exp["rank"]
    for key in ("sigma2_g", "sigma2_e"):
        assert abs(diag[key] - exp[key]) <= 1e-5 * abs(exp[key]), (key, diag[key], exp[key])
    out = eng.scan(g, np.arange(n), min_maf=0.01, precision=precision)
    t = exp["tested"]
    assert np.array_equal(out["tested"], t)
    assert np.array_equal(out["freq"][t], exp["freq"][t])
    for key in ("beta", "se"):
        err = np.abs(out[key][t] - exp[key][t]).max() / np.abs(exp[key][t]).max()
        assert err < 1e-5, (key, err)
    tol = 1e-4 if precision == "fp64" else 1e-3
    assert np.abs(out["log10p"][t] - exp["log10p"][t]).max() < tol
    eng.close()
    op.close()


@pytest.fixture(scope="module")
def aireml_oracle(cfg1):
    d, ref, g, X = cfg1
    Z = ref.dense_z()
    K = Z @ Z.T / d["m"]
    kw = dict(max_iter=6, mc_samples=30, slq_probes=30, slq_steps=15)
    ro, beta_o, a_o, _ = oracle.stcg_vce(ref, d["y"], X, dense_k=K, **kw)
    return kw, ro, beta_o, a_o


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config1_aireml_route(cfg1, aireml_oracle, precision):
    d, ref, g, X = cfg1
    kw, ro, beta_o, a_o = aireml_oracle
    op = cs.createKinshipOperator(g)
    vce = cs.StcgVce()
    r = vce.solve(op, d["y"], X, kinship_divisor=d["m"], precision=precision, **kw)
    assert r["iterations"] == ro["iterations"]
    for key in ("sigma2_g", "sigma2_e"):
        assert abs(r[key] - ro[key]) <= 1e-5 * ro[key], (key, r[key], ro[key])
    assert abs(r["logl"] - ro["logl"]) <= 1e-6 * abs(ro["logl"])
    beta, a, _ = vce.solution()
    assert np.abs(beta - beta_o).max() <= 1e-5 * np.abs(beta_o).max()
    assert np.abs(a - a_o).max() <= 1e-5 * np.abs(a_o).max()
    vce.close()
    op.close()
