"""Deterministic synthetic cohorts for tests and benchmarks.

Genotypes come from the counter-based generator in synth.cpp (host, OpenMP); per-SNP
frequencies, population labels, covariates and phenotypes from numpy with fixed seeds.
The workload shapes follow the benchmark configurations:

* ``config1``: N=2,000, M=10,000, MAF ~ U(0.05, 0.5), 1% missing, X = [1, N(0,1)],
  beta = (0, 0.5), 100 causal SNPs, h2 = 0.5.
* ``config2``: N=50,000, M=100,000, two Balding-Nichols populations (Fst 0.01, 50/50),
  2% missing, X = [1, N(0,1), Bernoulli(0.5)], h2 = 0.4 from 1,000 causal SNPs.
* ``config3``: N=100,000, M=500,000, MAF ~ U(0.01, 0.5), 8 traits with LKJ(2) genetic
  correlation, h2 ~ U(0.2, 0.6), exchangeable residual correlation 0.3.
* ``config4``: N=100,000 individuals with 1..5 records each, M=300,000 (repeatability).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "libcs_synth.so")
_SRC = os.path.join(HERE, "synth.cpp")
_lib = None


def build() -> str:
    if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
        subprocess.run([cxx, "-O2", "-fopenmp", "-fPIC", "-shared", "-o", _LIB, _SRC], check=True)
    return _LIB


def _l():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB)
        L.cs_synth_bed.argtypes = [C.c_int64, C.c_int64, C.c_uint64, C.c_void_p, C.c_int32,
                                   C.c_void_p, C.c_double, C.c_void_p]
        L.cs_synth_decode.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p]
        _lib = L
    return _lib


def allele_frequencies(m, maf_lo, n_pops, fst, rng):
    p = rng.uniform(maf_lo, 0.5, size=m)
    if n_pops <= 1 or fst <= 0:
        return p[:, None].copy()
    a = p * (1 - fst) / fst
    b = (1 - p) * (1 - fst) / fst
    f = rng.beta(a[:, None], b[:, None], size=(m, n_pops))
    return np.clip(f, 1e-6, 1 - 1e-6)


def genotype_bed(n, m, seed, freq, pop, missing_rate) -> np.ndarray:
    freq = np.ascontiguousarray(freq, dtype=np.float64)
    pop = np.ascontiguousarray(pop, dtype=np.int32)
    out = np.empty(3 + m * ((n + 3) // 4), dtype=np.uint8)
    _l().cs_synth_bed(n, m, seed, freq.ctypes.data, freq.shape[1], pop.ctypes.data,
                      float(missing_rate), out.ctypes.data)
    return out


def decode(bed, n, snps) -> np.ndarray:
    snps = np.ascontiguousarray(snps, dtype=np.int32)
    out = np.empty((n, len(snps)), order="F")
    _l().cs_synth_decode(bed.ctypes.data, n, snps.ctypes.data, len(snps), out.ctypes.data)
    return out


def cohort(n, m, seed, maf_lo=0.05, n_pops=1, fst=0.0, missing=0.01, n_causal=100, h2=0.5,
           covariates="intercept+normal", beta_x=None):
    """Returns dict(bed, n, m, y, X, pop, causal)."""
    rng = np.random.default_rng(seed)
    freq = allele_frequencies(m, maf_lo, n_pops, fst, rng)
    pop = rng.integers(0, max(n_pops, 1), size=n).astype(np.int32) if n_pops > 1 else np.zeros(n, np.int32)
    bed = genotype_bed(n, m, seed, freq, pop, missing)
    causal = np.sort(rng.choice(m, size=min(n_causal, m), replace=False)).astype(np.int32)
    G = decode(bed, n, causal)
    mu = np.nanmean(G, axis=0)
    sd = np.nanstd(G, axis=0)
    sd[sd == 0] = 1.0
    Z = np.where(np.isnan(G), 0.0, (G - mu) / sd)
    g = Z @ rng.standard_normal(len(causal))
    g = (g - g.mean()) / (g.std() or 1.0) * np.sqrt(h2)
    cols = [np.ones(n)]
    if "normal" in covariates:
        cols.append(rng.standard_normal(n))
    if "bernoulli" in covariates:
        cols.append(rng.integers(0, 2, size=n).astype(np.float64))
    X = np.column_stack(cols)
    if beta_x is None:
        beta_x = np.zeros(X.shape[1])
        if X.shape[1] > 1:
            beta_x[1] = 0.5
    y = X @ np.asarray(beta_x, dtype=np.float64) + g + rng.standard_normal(n) * np.sqrt(1 - h2)
    return {"bed": bed, "n": n, "m": m, "y": y, "X": X, "pop": pop, "causal": causal}


def config1(seed=20261203 + 1):
    return cohort(2000, 10000, seed, maf_lo=0.05, missing=0.01, n_causal=100, h2=0.5)


def config2(seed=20261203 + 2, n=50000, m=100000):
    return cohort(n, m, seed, maf_lo=0.05, n_pops=2, fst=0.01, missing=0.02, n_causal=1000,
                  h2=0.4, covariates="intercept+normal+bernoulli")


def lkj_correlation(d, eta, rng):
    """A d x d correlation matrix from the LKJ(eta) distribution by the C-vine construction of
    Lewandowski, Kurowicka and Joe (2009): partial correlations drawn as 2 Beta(b, b) - 1 with b
    starting at eta + (d - 1) / 2 and lowered by 1/2 per vine level, then turned into
    correlations along the vine."""
    b = eta + (d - 1) / 2.0
    P = np.zeros((d, d))
    R = np.eye(d)
    for k in range(d - 1):
        b -= 0.5
        for i in range(k + 1, d):
            P[k, i] = 2.0 * rng.beta(b, b) - 1.0
            r = P[k, i]
            for l in range(k - 1, -1, -1):
                r = r * np.sqrt((1.0 - P[l, i] ** 2) * (1.0 - P[l, k] ** 2)) + P[l, i] * P[l, k]
            R[k, i] = R[i, k] = r
    return R


def multi_trait_cohort(n, m, seed, d=8, eta=2.0, h2_range=(0.2, 0.6), resid_corr=0.3,
                       maf_lo=0.01, missing=0.01, n_causal=200):
    """d correlated traits: genetic correlation ~ LKJ(eta), h2_t ~ U(h2_range), exchangeable
    residual correlation resid_corr; each trait's polygenic score from its own n_causal SNPs
    (N(0,1) effects on standardised genotypes), mixed by the genetic correlation's Cholesky
    factor.  X = [1, N(0,1)].  Returns dict(bed, n, m, Y, X, Rg, h2)."""
    rng = np.random.default_rng(seed)
    freq = allele_frequencies(m, maf_lo, 1, 0.0, rng)
    pop = np.zeros(n, np.int32)
    bed = genotype_bed(n, m, seed, freq, pop, missing)
    causal = rng.choice(m, size=min(d * n_causal, m), replace=False).astype(np.int32)
    scores = np.zeros((n, d))
    for t in range(d):
        snps = np.sort(causal[t * n_causal:(t + 1) * n_causal])
        G = decode(bed, n, snps)
        mu = np.nanmean(G, axis=0)
        sd = np.nanstd(G, axis=0)
        sd[sd == 0] = 1.0
        s = np.where(np.isnan(G), 0.0, (G - mu) / sd) @ rng.standard_normal(len(snps))
        scores[:, t] = (s - s.mean()) / (s.std() or 1.0)
    Rg = lkj_correlation(d, eta, rng)
    Re = np.full((d, d), resid_corr) + (1.0 - resid_corr) * np.eye(d)
    h2 = rng.uniform(h2_range[0], h2_range[1], size=d)
    g = scores @ np.linalg.cholesky(Rg).T
    e = rng.standard_normal((n, d)) @ np.linalg.cholesky(Re).T
    X = np.column_stack([np.ones(n), rng.standard_normal(n)])
    Y = X @ np.vstack([np.zeros(d), np.full(d, 0.5)]) + g * np.sqrt(h2) + e * np.sqrt(1.0 - h2)
    return {"bed": bed, "n": n, "m": m, "Y": Y, "X": X, "Rg": Rg, "h2": h2}


def config3(seed=20261203 + 3, n=100000, m=500000):
    return multi_trait_cohort(n, m, seed)


def repeatability_cohort(n, m, seed, max_records=5, h2=0.3, repeatability=0.5, maf_lo=0.01,
                         missing=0.01, n_causal=100):
    """Record-level repeatability data: records per individual ~ U{1..max_records};
    y = X beta + Zr (g + pe) + e with var(g) = h2, var(pe) = repeatability - h2,
    var(e) = 1 - repeatability; fixed effects intercept, N(0,1) and a 4-level factor
    (three indicator columns).  Returns dict(bed, n, m, rec_to_row, y, X)."""
    base = cohort(n, m, seed, maf_lo=maf_lo, missing=missing, n_causal=n_causal, h2=1.0,
                  covariates="intercept")
    rng = np.random.default_rng(seed + 7)
    g = (base["y"] - base["y"].mean()) / (base["y"].std() or 1.0) * np.sqrt(h2)
    pe = rng.standard_normal(n) * np.sqrt(max(repeatability - h2, 0.0))
    counts = rng.integers(1, max_records + 1, size=n)
    rec_to_row = np.repeat(np.arange(n, dtype=np.int32), counts)
    n_rec = len(rec_to_row)
    level = rng.integers(0, 4, size=n_rec)
    X = np.column_stack([np.ones(n_rec), rng.standard_normal(n_rec)] +
                        [(level == q).astype(np.float64) for q in range(1, 4)])
    beta = np.array([0.0, 0.5, 0.2, -0.1, 0.3])
    y = X @ beta + g[rec_to_row] + pe[rec_to_row] + rng.standard_normal(n_rec) * np.sqrt(1 - repeatability)
    return {"bed": base["bed"], "n": n, "m": m, "rec_to_row": rec_to_row, "y": y, "X": X}


def config4(seed=20261203 + 4, n=100000, m=300000):
    return repeatability_cohort(n, m, seed)
