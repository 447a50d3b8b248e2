"""Leave-one-chromosome-out matrix-free LMM (the reference's default when the .bim holds more
than one chromosome, src/gwas_scanner.cpp:299-314, 464-472) against the oracle: per
chromosome, the operator drops that chromosome's GRM variants, fits its own low-rank null
model and scans that chromosome's SNPs.  Tolerances as the single-null path."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


def test_loco_matches_oracle_per_chromosome():
    d = synth.cohort(600, 2400, 77, missing=0.02, n_causal=60, h2=0.5)
    n, m = d["n"], d["m"]
    chrom = np.array(["1"] * 900 + ["2"] * 700 + ["10"] * 800)
    X = d["X"].astype(np.float32).astype(np.float64)
    res, diags = cs.run_lmm_matrix_free(d["bed"], n, m, d["y"], X, rank=30, chrom=chrom)
    assert list(diags) == ["1", "2", "10"]
    rows = d["bed"][3:].reshape(m, -1)
    ref = oracle.Bed(rows, n)
    g_stats = cs.Genotypes.from_bed_bytes(d["bed"], n, m)
    variants = cs.grm_variant_selection(g_stats.stats(), 0.01)
    keep = np.arange(n, dtype=np.int32)
    for c in ["1", "2", "10"]:
        loco = variants[chrom[variants] != c]
        U, lam, r = ref.lowrank_prepare(d["y"], X, 30, variants=loco, n_threads=8)
        assert abs(diags[c]["sigma2_g"] - r.sigma2_g) <= 1e-5 * r.sigma2_g
        assert abs(diags[c]["sigma2_e"] - r.sigma2_e) <= 1e-5 * r.sigma2_e
        idx = np.flatnonzero(chrom == c)
        sub = oracle.Bed(rows[idx[0]:idx[-1] + 1], n)
        o = sub.scan_lowrank(keep, U, lam, r.residual_eigenvalue, r.sigma2_g, r.sigma2_e,
                             d["y"], X)
        t = res["tested"][idx]
        assert np.array_equal(t, o["tested"])
        assert np.array_equal(res["freq"][idx][t], o["freq"][t])
        assert np.abs(res["log10p"][idx][t] - o["log10p"][t]).max() < 1e-4
        assert np.abs(res["beta"][idx][t] - o["beta"][t]).max() <= 1e-5 * np.abs(o["beta"][t]).max()
