"""The committed golden fixtures (tests/golden/, written by tests/golden/make_golden.py).

CPU: the oracle reproduces them (the known-answer recipe of the reference's
tests/test_kinship_batch.cpp with dense expected outputs; the low-rank null model and scan).
GPU: the CUDA library matches them — FP64 operator 1e-10, mixed operator 1e-6, variance
components 1e-5 relative, -log10 P 1e-4 absolute, statistics and tested set exact."""
import os

import numpy as np
import pytest

import oracle

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
N, M = 37, 1031
WIDTHS = (1, 7, 41)


def load(name):
    return dict(np.load(os.path.join(HERE, name)))


def sel(g, s):
    keep = g[f"keep_{s}"]
    var = g[f"variants_{s}"]
    return (None if len(keep) == 0 else keep), (None if len(var) == 0 else var)


def close(a, b, tol):
    assert np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max()), np.abs(a - b).max()


def test_oracle_reproduces_kinship_golden():
    g = load("kinship_batch_37x1031.npz")
    B = oracle.Bed(g["bed"][3:].reshape(M, -1), N)
    assert np.array_equal(B.mean, g["mean"]) and np.array_equal(B.inv_std, g["inv_std"])
    assert np.array_equal(B.count, g["count"]) and np.array_equal(B.sum, g["sum"])
    for s in range(6):
        keep, var = sel(g, s)
        assert abs(B.trace(keep, var) - g[f"trace_{s}"]) < 1e-10
        for w in WIDTHS:
            close(B.apply_block(g[f"x_{s}_{w}"], keep, var), g[f"kx_{s}_{w}"], 1e-10)


def test_oracle_reproduces_lowrank_golden():
    g = load("lowrank_200x600.npz")
    n, m = 200, 600
    B = oracle.Bed(g["bed"][3:].reshape(m, -1), n)
    U, lam, r = B.lowrank_prepare(g["y"], g["X"], 20, variants=g["variants"], n_threads=1)
    assert r.rank == int(g["rank"])
    close(lam, g["lam"], 1e-12)
    assert abs(r.sigma2_g - g["sigma2_g"]) <= 1e-12 * g["sigma2_g"]
    o = B.scan_lowrank(np.arange(n, dtype=np.int32), U, lam, r.residual_eigenvalue, r.sigma2_g,
                       r.sigma2_e, g["y"], g["X"])
    assert np.array_equal(o["tested"], g["tested"])
    t = g["tested"]
    close(o["log10p"][t], g["log10p"][t], 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_gpu_matches_kinship_golden(precision, tol):
    cs = pytest.importorskip("cosmicscanner_b200")
    g = load("kinship_batch_37x1031.npz")
    gen = cs.Genotypes.from_bed_bytes(g["bed"], N, M)
    st = gen.stats()
    assert np.array_equal(st["mean"], g["mean"]) and np.array_equal(st["inv_std"], g["inv_std"])
    assert np.array_equal(st["count"], g["count"]) and np.array_equal(st["sum"], g["sum"])
    for s in range(6):
        keep, var = sel(g, s)
        op = cs.createKinshipOperator(gen, keep, var)
        assert abs(op.trace() - g[f"trace_{s}"]) < 1e-10
        close(op.getDiagonal(), g[f"diag_{s}"], 1e-10)
        for w in WIDTHS:
            close(op.apply(g[f"x_{s}_{w}"], precision=precision), g[f"kx_{s}_{w}"], tol)


@pytest.mark.gpu
def test_gpu_matches_lowrank_golden():
    cs = pytest.importorskip("cosmicscanner_b200")
    g = load("lowrank_200x600.npz")
    n, m = 200, 600
    gen = cs.Genotypes.from_bed_bytes(g["bed"], n, m)
    op = cs.createKinshipOperator(gen, None, g["variants"])
    eng = cs.LmmEngine()
    d = eng.prepareLowRankMatrixFree(g["y"], g["X"], op, rank=20)
    assert d["effective_rank"] == int(g["rank"])
    assert abs(d["sigma2_g"] - g["sigma2_g"]) <= 1e-5 * g["sigma2_g"]
    assert abs(d["sigma2_e"] - g["sigma2_e"]) <= 1e-5 * g["sigma2_e"]
    out = eng.scan(gen, np.arange(n, dtype=np.int32))
    assert np.array_equal(out["tested"], g["tested"])
    t = g["tested"]
    assert np.array_equal(out["freq"][t], g["freq"][t])
    assert np.abs(out["log10p"][t] - g["log10p"][t]).max() < 1e-4
