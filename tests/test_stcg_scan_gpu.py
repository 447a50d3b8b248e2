"""Repeatability scan after the STCG null model (RepeatabilityModel::scanSTCG,
src/models/repeatability_scan_stcg.cpp:42-140) on the GPU against the oracle's
one-LDLT-solve-per-SNP restatement, given the same subject GRM and variance components.
Tolerances: BETA and SE 1e-6 relative, -log10 P 1e-6 absolute, MAF and tested set exact."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


@pytest.mark.parametrize("window", [(0, 700), (250, 333)])
def test_stcg_scan_matches_oracle(window):
    d = synth.repeatability_cohort(300, 700, 91, max_records=4, missing=0.03)
    n, m = d["n"], d["m"]
    rows = d["bed"][3:].reshape(m, -1)
    ref = oracle.Bed(rows, n)
    # subjects: every other genotype row (a kept subset), records of those subjects only
    subjects = np.arange(0, n, 2, dtype=np.int32)
    rank = -np.ones(n, dtype=np.int32)
    rank[subjects] = np.arange(len(subjects), dtype=np.int32)
    keep = rank[d["rec_to_row"]] >= 0
    o2s = rank[d["rec_to_row"][keep]]
    y = d["y"][keep]
    X = d["X"][keep].astype(np.float32).astype(np.float64)
    # a subject GRM: Z Z^T / M over the subjects (any SPD-ish GRM serves the scan)
    Z = ref.dense_z(subjects, None)
    G = Z @ Z.T / Z.shape[1]
    vg, vpe, ve = 0.3, 0.2, 0.5
    b, e = window
    o = oracle.stcg_scan(ref, G, subjects, o2s, y, X, vg, vpe, ve, 0.01, b, e)
    g = cs.Genotypes.from_bed_bytes(d["bed"], n, m)
    out = cs.stcg_scan(g, G, subjects, o2s, y, X, vg, vpe, ve, 0.01, b, e)
    assert np.array_equal(out["tested"], o["tested"])
    assert np.array_equal(out["maf"], o["maf"])
    t = o["tested"]
    assert t.sum() > 0.8 * (e - b)
    assert np.abs(out["beta"][t] - o["beta"][t]).max() <= 1e-6 * np.abs(o["beta"][t]).max()
    assert np.abs(out["se"][t] - o["se"][t]).max() <= 1e-6 * np.abs(o["se"][t]).max()
    assert np.abs(out["log10p"][t] - o["log10p"][t]).max() < 1e-6


def test_stcg_scan_rejects_bad_input():
    d = synth.repeatability_cohort(60, 100, 5, max_records=2)
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    G = np.eye(60)
    subj = np.arange(60, dtype=np.int32)
    with pytest.raises(cs.InvalidArgument):
        cs.stcg_scan(g, G, subj, d["rec_to_row"] + 60, d["y"], d["X"], 0.3, 0.2, 0.5)
    with pytest.raises(cs.InvalidArgument):
        cs.stcg_scan(g, G, subj, d["rec_to_row"], d["y"], d["X"], 0.3, 0.2, 0.5, snp_end=101)
