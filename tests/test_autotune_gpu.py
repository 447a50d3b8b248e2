"""The tensor-core passes' autotuner.

On a shape large enough to be tuned (2 R n k >= 2e10), the first mixed apply times the
candidate plans (CTA pairs or single CTAs x column-tile widths) of both passes and keeps the
fastest per shape bucket.  The tuner never changes the number of K slices, the only plan
parameter that changes floating-point results, so the tuned apply returns exactly the bits of
the default plan (the same apply in a process with CS_B200_AUTOTUNE=0), and it stays within the
mixed tolerance of the FP64 apply.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N, M, K = 10000, 12000, 96

SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import cosmicscanner_b200 as cs
from cosmicscanner_b200 import synth
d = synth.cohort(%d, %d, 77, missing=0.02, n_causal=20)
g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
op = cs.createKinshipOperator(g)
X = np.random.default_rng(1).standard_normal((d["n"], %d))
np.save(sys.argv[2], op.apply(X, precision="mixed"))
""" % (N, M, K)


def test_tuned_apply_matches_default_bitwise(tmp_path):
    d = synth.cohort(N, M, 77, missing=0.02, n_causal=20)
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    op = cs.createKinshipOperator(g)
    X = np.random.default_rng(1).standard_normal((d["n"], K))
    cs.profile_enable(True)
    Y = op.apply(X, precision="mixed")   # tunes both passes on first use
    again = op.apply(X, precision="mixed")
    table = cs.profile_summary()["autotune"]
    cs.profile_enable(False)
    assert np.array_equal(Y, again)
    passes = {(e["pass"], e["k"]) for e in table}
    assert ("rows", K) in passes and ("samples", K) in passes
    for e in table:
        assert e["candidates"] >= 2 and 0 < e["ms_best"] <= e["ms_default"] * 1.0001
    out = tmp_path / "default.npy"
    env = dict(os.environ, CS_B200_AUTOTUNE="0")
    res = subprocess.run([sys.executable, "-c", SCRIPT, ROOT, str(out)], env=env,
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    assert np.array_equal(np.load(out), Y), "a tuned plan changed the result"
    E = op.apply(X, precision="fp64")
    err = (np.abs(Y - E).max(axis=0) / np.abs(E).max(axis=0)).max()
    assert err < 1e-6, err
    op.close()
