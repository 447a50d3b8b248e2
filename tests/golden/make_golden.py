"""Writes the golden fixtures under tests/golden/ (run from the repository root:
``python tests/golden/make_golden.py``).

kinship_batch_37x1031.npz
    The reference's known-answer recipe (tests/test_kinship_batch.cpp of the reference):
    the 37 x 1031 BED bytes and omega draws regenerated from mt19937_64(8128), the six
    sample / variant selections, and the expected outputs computed DENSELY in FP64 from the
    float dosages exactly as that test builds them (z = (dosage - mean) * inv_std, NaN -> 0,
    K = z z^T / M): K @ omega per selection and width, trace and diagonal; plus the
    per-SNP statistics of PlinkReader::computeStats.
lowrank_200x600.npz
    A seeded synthetic cohort with the CPU oracle's low-rank null model (rank 20) and
    scanLowRank outputs: a regression pin for the restatement and a fixed target for the
    CUDA path.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from cosmicscanner_b200 import synth  # noqa: E402

N, M = 37, 1031
SUBSET = [35, 1, 20, 3, 4, 31, 7, 8, 10, 12, 14, 16, 18, 22, 24, 26, 28, 30, 32, 34]
WIDTHS = (1, 7, 41)


def selections():
    identity = list(range(N))
    permuted = [N - 1 - i for i in range(N)]
    repeated = [i // 2 for i in range(N)]
    variants = [j for j in range(M) if j % 3 != 1]
    out = []
    for s in range(6):
        keep = SUBSET if s == 1 else identity if s == 3 else permuted if s == 4 else \
            repeated if s == 5 else None
        out.append((keep, None if s == 0 else variants))
    return out


def kinship_batch():
    sels = selections()
    rows = [N if k is None else len(k) for k, _ in sels]
    bed, omega = oracle.kinship_batch_fixture(N, M, 8128, rows=rows)
    B = oracle.Bed(bed[3:].reshape(M, -1), N)
    out = {"bed": bed, "omega": omega, "mean": B.mean, "inv_std": B.inv_std,
           "count": B.count, "sum": B.sum}
    off = 0
    for s, ((keep, snps), r) in enumerate(zip(sels, rows)):
        z = B.dense_z(keep, snps)
        K = z @ z.T / z.shape[1]
        out[f"trace_{s}"] = np.array(np.trace(K))
        out[f"diag_{s}"] = np.diag(K).copy()
        out[f"keep_{s}"] = np.array([] if keep is None else keep, dtype=np.int32)
        out[f"variants_{s}"] = np.array([] if snps is None else snps, dtype=np.int32)
        for w in WIDTHS:
            X = omega[off:off + r * w].reshape(w, r).T  # column by column
            off += r * w
            out[f"x_{s}_{w}"] = np.asfortranarray(X)
            out[f"kx_{s}_{w}"] = K @ X
    np.savez_compressed(os.path.join(HERE, "kinship_batch_37x1031.npz"), **out)


def lowrank():
    d = synth.cohort(200, 600, 4242, missing=0.02, n_causal=30, h2=0.5)
    n, m = d["n"], d["m"]
    B = oracle.Bed(d["bed"][3:].reshape(m, -1), n)
    X = d["X"].astype(np.float32).astype(np.float64)
    variants = np.flatnonzero((B.inv_std != 0) & (np.minimum(B.mean / 2, 1 - B.mean / 2) >= 0.01)).astype(np.int32)
    U, lam, r = B.lowrank_prepare(d["y"], X, 20, variants=variants, n_threads=1)
    keep = np.arange(n, dtype=np.int32)
    o = B.scan_lowrank(keep, U, lam, r.residual_eigenvalue, r.sigma2_g, r.sigma2_e, d["y"], X)
    np.savez_compressed(
        os.path.join(HERE, "lowrank_200x600.npz"), bed=d["bed"], y=d["y"], X=X,
        variants=variants, lam=lam, sigma2_g=r.sigma2_g, sigma2_e=r.sigma2_e,
        r0=r.residual_eigenvalue, rank=r.rank, beta=o["beta"], se=o["se"], p=o["p"],
        log10p=o["log10p"], freq=o["freq"], tested=o["tested"])


if __name__ == "__main__":
    kinship_batch()
    lowrank()
    print("golden fixtures written to", HERE)
