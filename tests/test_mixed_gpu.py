"""Tensor-core (int8 tcgen05) form of the kinship operator and of the low-rank LMM.

Tolerances are those stated for the mixed form against the FP64 oracle: every operator
apply within 1e-6 relative error (max-norm per column), variance components and BETA/SE
within 1e-5 relative, -log10 P within 1e-3 absolute.  Cases cover the reference's
partial-byte fixture (N=37), sample subsets, repeated / permuted rows, LOCO-like variant
masks, intercept-like columns and column counts that span several column tiles.
"""
import numpy as np
import pytest

import oracle
from tests.test_oracle import M, N, selections

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


def colwise_rel(Y, E):
    scale = np.maximum(np.abs(E).max(axis=0), 1e-300)
    return (np.abs(Y - E).max(axis=0) / scale)


def test_batch_fixture_mixed():
    sels = selections()
    rows = [N if k is None else len(k) for k, _ in sels]
    bed, omega = oracle.kinship_batch_fixture(N, M, 8128, rows=rows)
    ref = oracle.Bed(bed[3:].reshape(M, -1), N)
    g = cs.Genotypes.from_bed_bytes(bed, N, M)
    off = 0
    for (keep, snps), r in zip(sels, rows):
        op = cs.createKinshipOperator(g, keep, snps)
        for w in (1, 7, 41):
            om = omega[off:off + r * w].reshape(w, r).T
            off += r * w
            E = ref.apply_block(om, keep, snps)
            Y = op.apply(om, precision="mixed")
            assert colwise_rel(Y, E).max() < 1e-6
            again = op.apply(om, precision="mixed")
            assert np.array_equal(again, Y), "mixed apply is not bitwise repeatable"


@pytest.mark.parametrize("k", [1, 5, 16, 65, 68, 81, 170, 240, 266])
def test_operator_mixed_random(k):
    d = synth.cohort(2600, 3000, 17, missing=0.02, n_causal=10)
    ref = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    op = cs.createKinshipOperator(g)
    rng = np.random.default_rng(k)
    X = rng.standard_normal((d["n"], k))
    if k > 2:
        X[:, 0] = 1.0           # intercept: K 1 ~ 0, compared in absolute terms below
        X[:, 1] += 25.0         # large column mean
    E = ref.apply_block(X, n_threads=8)
    Y = op.apply(X, precision="mixed")
    rel = colwise_rel(Y, E)
    if k > 2:
        assert np.abs(Y[:, 0] - E[:, 0]).max() < 1e-6 * np.abs(E[:, 2:]).max()
        assert rel[1:].max() < 1e-6, rel.max()
    else:
        assert rel.max() < 1e-6


def test_operator_mixed_selection():
    d = synth.cohort(3000, 2500, 23, missing=0.03, n_causal=10)
    ref = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    rng = np.random.default_rng(4)
    keep = rng.choice(d["n"], 2100, replace=False).astype(np.int32)     # unsorted subset
    variants = np.sort(rng.choice(d["m"], 1700, replace=False)).astype(np.int32)
    op = cs.createKinshipOperator(g, keep, variants)
    X = rng.standard_normal((len(keep), 33))
    E = ref.apply_block(X, keep, variants, n_threads=8)
    assert colwise_rel(op.apply(X, precision="mixed"), E).max() < 1e-6


def test_lowrank_mixed_matches_oracle():
    d = synth.cohort(1500, 4000, 29, missing=0.02, n_causal=60, h2=0.5)
    n = d["n"]
    ref = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), n)
    g = cs.Genotypes.from_bed_bytes(d["bed"], n, d["m"])
    y = d["y"]
    X = d["X"].astype(np.float32).astype(np.float64)
    U_o, lam_o, res = ref.lowrank_prepare(y, X, 60, n_threads=8)
    op = cs.createKinshipOperator(g)
    eng = cs.LmmEngine()
    diag = eng.prepareLowRankMatrixFree(y, X, op, rank=60, precision="mixed")
    assert diag["effective_rank"] == res.rank
    for key in ("sigma2_g", "sigma2_e"):
        assert abs(diag[key] - getattr(res, key)) <= 1e-5 * abs(getattr(res, key)), key
    keep = np.arange(n)
    out = eng.scan(g, keep, precision="mixed")
    exp = ref.scan_lowrank(keep, U_o, lam_o, res.residual_eigenvalue, res.sigma2_g,
                           res.sigma2_e, y, X)
    t = exp["tested"]
    assert np.array_equal(out["tested"], t)
    assert np.array_equal(out["freq"][t], exp["freq"][t])
    for key in ("beta", "se"):
        err = np.abs(out[key][t] - exp[key][t]).max() / np.abs(exp[key][t]).max()
        assert err < 1e-5, (key, err)
    assert np.abs(out["log10p"][t] - exp["log10p"][t]).max() < 1e-3


def test_lowrank_scan_reuses_sketch_rows(monkeypatch):
    """With every sample analysed, the mixed scan takes its U block from the last sketch
    apply ((Z^T Q) W_sel) and projects only X and Py through the genotypes; the result agrees
    with the full projection (CS_B200_SCAN_REUSE=0) within the mixed tolerance, and the
    LOCO-style operator (SNPs missing from it) falls back to the full projection."""
    d = synth.cohort(1200, 3000, 41, missing=0.02, n_causal=40, h2=0.5)
    n = d["n"]
    g = cs.Genotypes.from_bed_bytes(d["bed"], n, d["m"])
    y = d["y"]
    X = d["X"].astype(np.float32).astype(np.float64)
    keep = np.arange(n)
    for variants in (None, np.arange(0, 2000, dtype=np.int32)):
        op = cs.createKinshipOperator(g, None, variants)
        eng = cs.LmmEngine()
        eng.prepareLowRankMatrixFree(y, X, op, rank=50, precision="mixed")
        a = eng.scan(g, keep, precision="mixed")
        monkeypatch.setenv("CS_B200_SCAN_REUSE", "0")
        b = eng.scan(g, keep, precision="mixed")
        monkeypatch.delenv("CS_B200_SCAN_REUSE")
        t = b["tested"]
        assert np.array_equal(a["tested"], t) and t.sum() > 0.9 * d["m"]
        assert np.array_equal(a["freq"][t], b["freq"][t])
        for key in ("beta", "se"):
            err = np.abs(a[key][t] - b[key][t]).max() / np.abs(b[key][t]).max()
            assert err < 1e-6, (key, err)
        assert np.abs(a["log10p"][t] - b["log10p"][t]).max() < 1e-4


@pytest.mark.parametrize("mode", [
    {"CS_B200_CTA_PAIRS": "0"},                                  # single CTAs, every width
    {"CS_B200_CTA_PAIRS": "1"},                                  # CTA pairs, every width
    {"CS_B200_TMEM_A": "0", "CS_B200_TMEM_A_PAIRS": "0"},        # A in shared memory
    {"CS_B200_CTA_PAIRS": "1", "CS_B200_TMEM_A_PAIRS": "1"},     # pairs: rows in TMEM only
    {"CS_B200_TMEM_A": "1"},                                     # the 32-wide TMEM form only
    {"CS_B200_CTA_PAIRS": "1", "CS_B200_TMEM_A_PAIRS": "3"},     # pairs: five-set TMEM samples
    {"CS_B200_DECODE_ALT": "0"},                                 # all decoders on every K-block
    {"CS_B200_DECODE_ALT": "1"},                                 # decoder groups alternate
], ids=["single", "pairs", "smem-a", "pairs-rows-tmem", "tmem32", "pairs-five-set-tmem",
        "decode-shared", "decode-alternate"])
def test_operator_mixed_forced_cta_mode(mode):
    """Forced plan families (single CTAs or CTA pairs for every width, the A operand in shared
    memory or in tensor memory, five- or six-set samples passes) give the same operator as the
    oracle within the mixed tolerance; the switches are read once per process, so each runs in
    a child interpreter."""
    import json
    import os
    import subprocess
    import sys

    code = r'''
import json, sys, numpy as np
sys.path.insert(0, sys.argv[1])
import cosmicscanner_b200 as cs
from cosmicscanner_b200 import synth
d = synth.cohort(2600, 3000, 17, missing=0.02, n_causal=10)
g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
op = cs.createKinshipOperator(g)
out = {}
for k in (16, 40, 68):
    X = np.random.default_rng(k).standard_normal((d["n"], k))
    out[k] = op.apply(X, precision="mixed").tolist()
print(json.dumps(out))
'''
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, **mode)
    res = subprocess.run([sys.executable, "-c", code, root], env=env, capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    forced = json.loads(res.stdout.strip().splitlines()[-1])
    d = synth.cohort(2600, 3000, 17, missing=0.02, n_causal=10)
    ref = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    for k in (16, 40, 68):
        X = np.random.default_rng(k).standard_normal((d["n"], k))
        E = ref.apply_block(X, n_threads=8)
        Y = np.array(forced[str(k)])
        assert colwise_rel(Y, E).max() < 1e-6


def test_tensor_memory_forms_bitwise():
    """The five-set samples pass over the sample-major copy (A in tensor memory, each SNP's
    imputed code put in along K under the missing-call mask) forms the same int32 sums as the
    shared-memory form, and so does the rows pass: on CTA pairs with the same K slices the two
    plan families return the same bits (64- or 80-wide column tiles; k = 16 and 96)."""
    import json
    import os
    import subprocess
    import sys

    code = r'''
import json, sys, numpy as np
sys.path.insert(0, sys.argv[1])
import cosmicscanner_b200 as cs
from cosmicscanner_b200 import synth
d = synth.cohort(2600, 3000, 23, missing=0.03, n_causal=10)
g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
op = cs.createKinshipOperator(g)
out = {}
for k in (16, 96):
    X = np.random.default_rng(k).standard_normal((d["n"], k))
    out[k] = op.apply(X, precision="mixed").tobytes().hex()
print(json.dumps(out))
'''
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    runs = []
    for mode in ({"CS_B200_CTA_PAIRS": "1", "CS_B200_TMEM_A_PAIRS": "3"},
                 {"CS_B200_CTA_PAIRS": "1", "CS_B200_TMEM_A_PAIRS": "0"}):
        env = dict(os.environ, CS_B200_AUTOTUNE="0", **mode)
        res = subprocess.run([sys.executable, "-c", code, root], env=env, capture_output=True,
                             text=True, timeout=600)
        assert res.returncode == 0, res.stderr[-2000:]
        runs.append(json.loads(res.stdout.strip().splitlines()[-1]))
    for k in ("16", "96"):
        assert runs[0][k] == runs[1][k], f"k={k}: tensor-memory and shared-memory forms differ"


def test_decoder_groups_bitwise():
    """Whether the decoder warps share every K-block or split into two groups that take
    alternate K-blocks changes only who writes which part of the tensor-memory tiles, so the
    applies are bitwise equal (narrow and 64-wide single-CTA plans, CTA pairs in both forms)."""
    import json
    import os
    import subprocess
    import sys

    code = r'''
import json, sys, numpy as np
sys.path.insert(0, sys.argv[1])
import cosmicscanner_b200 as cs
from cosmicscanner_b200 import synth
d = synth.cohort(2600, 3000, 29, missing=0.02, n_causal=10)
g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
op = cs.createKinshipOperator(g)
out = {}
for k in (16, 48, 96):
    X = np.random.default_rng(k).standard_normal((d["n"], k))
    out[k] = op.apply(X, precision="mixed").tobytes().hex()
print(json.dumps(out))
'''
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for extra in ({}, {"CS_B200_CTA_PAIRS": "1", "CS_B200_TMEM_A_PAIRS": "3"}):
        runs = []
        for alt in ("0", "1"):
            env = dict(os.environ, CS_B200_AUTOTUNE="0", CS_B200_DECODE_ALT=alt, **extra)
            res = subprocess.run([sys.executable, "-c", code, root], env=env, capture_output=True,
                                 text=True, timeout=600)
            assert res.returncode == 0, res.stderr[-2000:]
            runs.append(json.loads(res.stdout.strip().splitlines()[-1]))
        for k in ("16", "48", "96"):
            assert runs[0][k] == runs[1][k], f"k={k} {extra}: decoder groups changed the result"
