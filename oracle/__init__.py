"""ctypes loader for the CPU oracle — TEST INFRASTRUCTURE ONLY.

The oracle restates the reference CosmicScanner algorithms on the CPU in FP64
(oracle.cpp cites the reference file:line of every function).  Only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it, and
only as the checker: the product library never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build() -> str:
    """Compile liboracle.so in place (make); returns its path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class StcgOptions(C.Structure):
    _fields_ = [
        ("max_iter", C.c_int32), ("tol", C.c_double), ("mc_samples", C.c_int32),
        ("pcg_tol", C.c_double), ("pcg_max_iter", C.c_int32), ("slq_probes", C.c_int32),
        ("slq_steps", C.c_int32), ("probe_seed", C.c_uint64),
    ]


class StcgResult(C.Structure):
    _fields_ = [
        ("sigma2_g", C.c_double), ("sigma2_pe", C.c_double), ("sigma2_e", C.c_double),
        ("logl", C.c_double), ("iterations", C.c_int32), ("converged", C.c_int32),
        ("pcg_iterations", C.c_int64),
    ]


class LowRankResult(C.Structure):
    _fields_ = [
        ("rank", C.c_int32), ("sketch_size", C.c_int32),
        ("residual_eigenvalue", C.c_double), ("relative_frobenius_error", C.c_double),
        ("trace", C.c_double), ("trace_fraction", C.c_double),
        ("trace_threshold_met", C.c_int32),
        ("sigma2_g", C.c_double), ("sigma2_e", C.c_double), ("delta", C.c_double),
        ("best_log_eta", C.c_double), ("best_objective", C.c_double),
    ]


_P = C.c_void_p
_I64 = C.c_int64


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "oracle.cpp"))
        ):
            build()
        L = C.CDLL(_LIB_PATH)
        sel = [_P, _I64, _P, _I64]  # keep, n_keep, variants, n_var
        L.orc_compute_stats.argtypes = [_P, _I64, _I64, _I64, _P, _P, _P, _P]
        L.orc_kinship_apply_vector.argtypes = [_P, _I64, _I64, _P, _P] + sel + [_P, _P, C.c_int]
        L.orc_kinship_apply_vector.restype = C.c_int
        L.orc_kinship_apply_block.argtypes = [_P, _I64, _I64, _P, _P] + sel + [_P, _I64, _I64, _P, _I64, C.c_int]
        L.orc_kinship_apply_block.restype = C.c_int
        L.orc_kinship_trace.argtypes = [_P, _I64, _I64, _P, _P] + sel
        L.orc_kinship_trace.restype = C.c_double
        L.orc_kinship_diagonal.argtypes = [_P, _I64, _I64, _P, _P] + sel + [_P]
        L.orc_dense_z.argtypes = [_P, _I64, _I64, _P, _P] + sel + [_P, _I64]
        L.orc_kinship_batch_fixture.argtypes = [C.c_int, C.c_int, C.c_uint64, _P, C.c_int, _P, C.c_int, _P, _P]
        L.orc_normal_matrix.argtypes = [C.c_uint64, _I64, _I64, _P]
        L.orc_prepare_marker.argtypes = [_P, _I64, C.c_double, _P, _P, _P]
        L.orc_prepare_marker.restype = C.c_int
        L.orc_chisq_prob.argtypes = [C.c_double, C.c_int]
        L.orc_chisq_prob.restype = C.c_double
        L.orc_lowrank_prepare.argtypes = [_P, _I64, _I64, _P, _P] + sel + [
            _P, _P, _I64, C.c_int, C.c_int, C.c_uint64, C.c_double, C.c_int, C.c_int, _P, _P, _P]
        L.orc_lowrank_prepare.restype = C.c_int
        L.orc_lowrank_reml.argtypes = [_P, _P, _I64, _I64, C.c_double, _P, _P, _I64, _P]
        L.orc_lowrank_reml.restype = C.c_int
        L.orc_scan_lowrank.argtypes = [_P, _I64, _I64, _I64, _P, _I64, _P, _P, _I64, C.c_double,
                                       C.c_double, C.c_double, _P, _P, _I64, C.c_double,
                                       _P, _P, _P, _P, _P, _P]
        L.orc_scan_lowrank.restype = C.c_int
        L.orc_pcg_solve.argtypes = [_P, _I64, _I64, _P, _P] + sel + [
            C.c_double, C.c_double, _P, C.c_double, C.c_int, _P]
        L.orc_pcg_solve.restype = C.c_int
        L.orc_stcg_vce.argtypes = [_P, _I64, _I64, _I64, _P, _P, _P, _I64, C.c_int, _P, _P, _I64,
                                   _P, _P, _P, _P, _P]
        L.orc_stcg_vce.restype = C.c_int
        L.orc_stcg_vce_dense.argtypes = [_P, _I64, _P, _I64, C.c_int, _P, _P, _I64, _P, _P, _P,
                                         _P, _P]
        L.orc_stcg_vce_dense.restype = C.c_int
        L.orc_stcg_scan.argtypes = [_P, _I64, _I64, _P, _I64, _P, _P, _I64, _P, _P, _I64,
                                    C.c_double, C.c_double, C.c_double, C.c_double, _I64, _I64,
                                    _P, _P, _P, _P, _P, _P]
        L.orc_stcg_scan.restype = C.c_int
        L.orc_mvlmm_scan.argtypes = [_P, _I64, _I64, _P, _I64, _P, _I64, _P, _P, _I64, _P, _I64,
                                     _P, _P, _I64, _I64, _P, _P, _P, _P, _P, _P]
        L.orc_mvlmm_scan.restype = C.c_int
        L.orc_decode_z_cols.argtypes = [_P, _I64, _P, _P, _P, _I64, _I64, _P, _I64, C.c_int]
        L.orc_scan_encode_cols.argtypes = [_P, _I64, _I64, _I64, _I64, C.c_double, _P, _I64, _P,
                                           _P, _P, C.c_int]
        L.orc_chisq_prob_vec.argtypes = [_P, _I64, C.c_int, _P, C.c_int]
        L.orc_rademacher.argtypes = [C.c_uint64, _I64, _I64, _I64, _P]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


class Bed:
    """Packed SNP-major BED rows (magic skipped) with the reference's per-SNP stats."""

    def __init__(self, rows: np.ndarray, n_samples: int):
        self.rows = np.ascontiguousarray(rows, dtype=np.uint8)
        self.n = int(n_samples)
        self.m = int(self.rows.shape[0])
        self.stride = int(self.rows.shape[1])
        self.mean = np.zeros(self.m)
        self.inv_std = np.zeros(self.m)
        self.count = np.zeros(self.m, dtype=np.int32)
        self.sum = np.zeros(self.m)
        lib().orc_compute_stats(_ptr(self.rows), self.n, self.m, self.stride, _ptr(self.mean),
                                _ptr(self.inv_std), _ptr(self.count), _ptr(self.sum))

    def _sel(self, keep, variants):
        keep = _i32(keep)
        variants = _i32(variants)
        args = [_ptr(keep), 0 if keep is None else len(keep),
                _ptr(variants), self.m if variants is None else len(variants)]
        return args, (keep, variants)

    def rows_for(self, keep):
        return self.n if keep is None else len(keep)

    def apply_vector(self, v, keep=None, variants=None, n_threads=1):
        args, hold = self._sel(keep, variants)
        v = np.ascontiguousarray(v, dtype=np.float64)
        out = np.zeros(self.rows_for(keep))
        rc = lib().orc_kinship_apply_vector(_ptr(self.rows), self.n, self.stride, _ptr(self.mean),
                                            _ptr(self.inv_std), *args, _ptr(v), _ptr(out), n_threads)
        if rc != 0:
            raise RuntimeError("oracle apply_vector failed")
        return out

    def apply_block(self, X, keep=None, variants=None, n_threads=1):
        args, hold = self._sel(keep, variants)
        X = np.asfortranarray(X, dtype=np.float64)
        n, k = X.shape
        out = np.zeros((n, k), order="F")
        rc = lib().orc_kinship_apply_block(_ptr(self.rows), self.n, self.stride, _ptr(self.mean),
                                           _ptr(self.inv_std), *args, _ptr(X), n, k, _ptr(out), n,
                                           n_threads)
        if rc != 0:
            raise RuntimeError("oracle apply_block failed")
        return out

    def trace(self, keep=None, variants=None):
        args, hold = self._sel(keep, variants)
        return lib().orc_kinship_trace(_ptr(self.rows), self.n, self.stride, _ptr(self.mean),
                                       _ptr(self.inv_std), *args)

    def diagonal(self, keep=None, variants=None):
        args, hold = self._sel(keep, variants)
        out = np.zeros(self.rows_for(keep))
        lib().orc_kinship_diagonal(_ptr(self.rows), self.n, self.stride, _ptr(self.mean),
                                   _ptr(self.inv_std), *args, _ptr(out))
        return out

    def dense_z(self, keep=None, variants=None):
        args, hold = self._sel(keep, variants)
        nr = self.rows_for(keep)
        nv = self.m if variants is None else len(variants)
        z = np.zeros((nr, nv), order="F")
        lib().orc_dense_z(_ptr(self.rows), self.n, self.stride, _ptr(self.mean),
                          _ptr(self.inv_std), *args, _ptr(z), nr)
        return z

    def lowrank_prepare(self, y, X, rank, keep=None, variants=None, oversample=10, seed=42,
                        trace_threshold=0.95, min_rank=1, n_threads=1):
        args, hold = self._sel(keep, variants)
        y = np.ascontiguousarray(y, dtype=np.float64)
        X = np.asfortranarray(X, dtype=np.float64)
        n, p = X.shape
        U = np.zeros((n, rank), order="F")
        lam = np.zeros(rank)
        res = LowRankResult()
        rc = lib().orc_lowrank_prepare(_ptr(self.rows), self.n, self.stride, _ptr(self.mean),
                                       _ptr(self.inv_std), *args, _ptr(y), _ptr(X), p, rank,
                                       oversample, seed, trace_threshold, min_rank, n_threads,
                                       _ptr(U), _ptr(lam), C.byref(res))
        if rc != 0:
            raise RuntimeError(f"oracle lowrank_prepare failed ({rc})")
        r = res.rank
        return np.asfortranarray(U[:, :r]), lam[:r].copy(), res

    def scan_lowrank(self, keep, U, lam, r0, sigma2_g, sigma2_e, y, X, min_maf=0.01):
        keep = _i32(keep)
        U = np.asfortranarray(U, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        X = np.asfortranarray(X, dtype=np.float64)
        n, p = X.shape
        out = {k: np.full(self.m, np.nan) for k in ("beta", "se", "p", "log10p", "freq")}
        tested = np.zeros(self.m, dtype=np.int32)
        rc = lib().orc_scan_lowrank(_ptr(self.rows), self.n, self.stride, self.m, _ptr(keep), n,
                                    _ptr(U), _ptr(lam), U.shape[1], r0, sigma2_g, sigma2_e,
                                    _ptr(y), _ptr(X), p, min_maf, _ptr(out["beta"]),
                                    _ptr(out["se"]), _ptr(out["p"]), _ptr(out["log10p"]),
                                    _ptr(out["freq"]), _ptr(tested))
        if rc != 0:
            raise RuntimeError("oracle scan_lowrank failed")
        out["tested"] = tested.astype(bool)
        return out

    def pcg_solve(self, b, sg2, se2, tol, max_iter, keep=None, variants=None):
        args, hold = self._sel(keep, variants)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        it = lib().orc_pcg_solve(_ptr(self.rows), self.n, self.stride, _ptr(self.mean),
                                 _ptr(self.inv_std), *args, sg2, se2, _ptr(b), tol, max_iter, _ptr(x))
        return x, it


def stcg_vce(bed: "Bed", y, X, rec_to_row=None, with_pe=False, max_iter=50, tol=1e-6,
             mc_samples=20, pcg_tol=1e-10, pcg_max_iter=2000, slq_probes=30, slq_steps=15,
             probe_seed=20250101, dense_k=None):
    """STCG_VCE::solve restated (libCosmicCore/src/stcg_vce.cpp:157-407); returns
    (result dict, beta, a_rows, pe_rows).  dense_k: the kinship operator as a dense
    K = Z Z^T / M (bed.n x bed.n), applied as one matrix-vector product per CG step."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    X = np.asfortranarray(np.asarray(X, dtype=np.float64).reshape(len(y), -1))
    rmap = None if rec_to_row is None else np.ascontiguousarray(rec_to_row, dtype=np.int32)
    opt = StcgOptions(max_iter, tol, mc_samples, pcg_tol, pcg_max_iter, slq_probes, slq_steps,
                      probe_seed)
    res = StcgResult()
    beta = np.zeros(X.shape[1])
    a = np.zeros(bed.n)
    pe = np.zeros(bed.n)
    if dense_k is not None:
        K = np.asfortranarray(dense_k, dtype=np.float64)
        rc = lib().orc_stcg_vce_dense(_ptr(K), bed.n, _ptr(rmap), len(y), int(bool(with_pe)),
                                      _ptr(y), _ptr(X), X.shape[1], C.byref(opt), C.byref(res),
                                      _ptr(beta), _ptr(a), _ptr(pe))
    else:
        rc = lib().orc_stcg_vce(_ptr(bed.rows), bed.n, bed.stride, bed.m, _ptr(bed.mean),
                                _ptr(bed.inv_std), _ptr(rmap), len(y), int(bool(with_pe)), _ptr(y),
                                _ptr(X), X.shape[1], C.byref(opt), C.byref(res), _ptr(beta),
                                _ptr(a), _ptr(pe))
    if rc != 0:
        raise RuntimeError("oracle stcg_vce failed")
    out = {name: getattr(res, name) for name, _ in res._fields_}
    return out, beta, a, pe


def stcg_scan(bed: "Bed", G, subject_rows, obs_to_subject, y, X, vg, vpe, ve, min_maf=0.01,
              snp_begin=0, snp_end=None):
    """scan_stcg_with_grm restated (src/models/repeatability_scan_stcg.cpp:42-140)."""
    G = np.asfortranarray(G, dtype=np.float64)
    subj = np.ascontiguousarray(subject_rows, dtype=np.int32)
    o2s = np.ascontiguousarray(obs_to_subject, dtype=np.int32)
    y = np.ascontiguousarray(y, dtype=np.float64)
    X = np.asfortranarray(np.asarray(X, dtype=np.float64).reshape(len(y), -1))
    end = bed.m if snp_end is None else int(snp_end)
    w = end - int(snp_begin)
    out = {k: np.zeros(w) for k in ("beta", "se", "p", "log10p", "maf")}
    tested = np.zeros(w, dtype=np.int32)
    rc = lib().orc_stcg_scan(_ptr(bed.rows), bed.n, bed.stride, _ptr(G), G.shape[0], _ptr(subj),
                             _ptr(o2s), len(y), _ptr(y), _ptr(X), X.shape[1], vg, vpe, ve,
                             min_maf, int(snp_begin), end, _ptr(out["beta"]), _ptr(out["se"]),
                             _ptr(out["p"]), _ptr(out["log10p"]), _ptr(out["maf"]), _ptr(tested))
    if rc != 0:
        raise RuntimeError(f"oracle stcg_scan failed ({rc})")
    out["tested"] = tested.astype(bool)
    return out


def mvlmm_scan(bed: "Bed", keep, W, D, Uty, UtX, Vg, Ve, snp_begin=0, snp_end=None):
    """MvLmmEngine::scan(PlinkReader) restated (src/mvlmm_engine.cpp:756-931)."""
    keep = np.ascontiguousarray(keep, dtype=np.int32)
    W = np.asfortranarray(W, dtype=np.float64)
    n, r = W.shape
    D = np.ascontiguousarray(D, dtype=np.float64)
    Uty = np.asfortranarray(np.asarray(Uty, dtype=np.float64).reshape(r, -1))
    d = Uty.shape[1]
    UtX = np.asfortranarray(np.asarray(UtX, dtype=np.float64).reshape(r, -1))
    Vg = np.asfortranarray(Vg, dtype=np.float64)
    Ve = np.asfortranarray(Ve, dtype=np.float64)
    end = bed.m if snp_end is None else int(snp_end)
    m = end - int(snp_begin)
    beta, cov = np.zeros((m, d)), np.zeros((m, d, d))
    wald, pv, fr = np.zeros(m), np.zeros(m), np.zeros(m)
    st = np.zeros(m, dtype=np.int32)
    lib().orc_mvlmm_scan(_ptr(bed.rows), bed.n, bed.stride, _ptr(keep), n, _ptr(W), r, _ptr(D),
                         _ptr(Uty), d, _ptr(UtX), UtX.shape[1], _ptr(Vg), _ptr(Ve),
                         int(snp_begin), end, _ptr(beta), _ptr(cov), _ptr(wald), _ptr(pv),
                         _ptr(fr), _ptr(st))
    return {"beta": beta, "cov": cov, "wald": wald, "p": pv, "freq": fr, "status": st}


def kinship_batch_fixture(n=37, m=1031, seed=8128, rows=None, widths=(1, 7, 41)):
    """Regenerates tests/test_kinship_batch.cpp's BED bytes and omega draws exactly."""
    rows = np.asarray(rows if rows is not None else [], dtype=np.int32)
    widths = np.asarray(widths, dtype=np.int32)
    stride = (n + 3) // 4
    bed = np.zeros(3 + m * stride, dtype=np.uint8)
    total = int(sum(int(r) * int(w) for r in rows for w in widths))
    omega = np.zeros(max(total, 1))
    lib().orc_kinship_batch_fixture(n, m, seed, _ptr(bed), len(rows), _ptr(rows), len(widths),
                                    _ptr(widths), _ptr(omega) if total else None)
    return bed, omega[:total]


def normal_matrix(seed, n, cols):
    out = np.zeros((n, cols), order="F")
    lib().orc_normal_matrix(seed, n, cols, _ptr(out))
    return out


def rademacher(seed, skip, n, cols):
    """n x cols +-1 block from mt19937_64(seed) + uniform_int_distribution<int>(0, 1) after
    `skip` draws, column by column (the probe stream of the matrix-free REML estimators)."""
    out = np.zeros((n, cols), order="F")
    lib().orc_rademacher(int(seed), int(skip), int(n), int(cols), _ptr(out))
    return out


def chisq_prob(stat, df=1):
    return lib().orc_chisq_prob(float(stat), int(df))


def prepare_marker(raw, min_maf=0.01):
    raw = np.ascontiguousarray(raw, dtype=np.float64)
    vals = np.zeros_like(raw)
    f = C.c_double()
    obs = C.c_int32()
    ok = lib().orc_prepare_marker(_ptr(raw), len(raw), min_maf, _ptr(vals), C.byref(f), C.byref(obs))
    return bool(ok), vals, f.value, obs.value


# ---------------------------------------------------------------- BLAS restatements
# Timed CPU baseline: the whole low-rank job with numpy's multithreaded BLAS/LAPACK standing in
# for Eigen's GEMMs, Householder QR and eigensolver, and OpenMP table decodes in liboracle.
# Decode tables follow src/kinship_operator.cpp:276-283.

def _decode_block(rows, n, values):
    """rows: (b, stride) packed bytes; values: (b, 4) per-row code values -> (n, b) FP64."""
    codes = np.stack([(rows >> (2 * q)) & 3 for q in range(4)], axis=2).reshape(rows.shape[0], -1)[:, :n]
    return np.take_along_axis(values, codes.astype(np.int64), axis=1).T.copy()


def _threads(n_threads):
    if n_threads:
        return int(n_threads)
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _reml_search(lam, r0, n, p, yty, Xty, XtX, Uty, UtX, y, X):
    """The low-rank REML objective and search of src/lmm_engine.cpp:1010-1073 (81-point grid
    on log eta in [-12, 12], then at most 80 golden-section steps to 1e-8), with the
    projections U^T y, U^T X precomputed so that each evaluation is O(rank p^2)."""
    df = n - p
    rank = len(lam)

    def objective(log_eta, want_q=False):
        eta = np.exp(log_eta)
        base = 1.0 / (1.0 + eta * r0)
        c = 1.0 / (1.0 + eta * lam) - base
        info = base * XtX + UtX.T @ (c[:, None] * UtX)
        rhs = base * Xty + UtX.T @ (c * Uty)
        try:
            L = np.linalg.cholesky(info)
        except np.linalg.LinAlgError:
            return (np.inf, None) if want_q else np.inf
        beta = np.linalg.solve(info, rhs)
        r = y - X @ beta
        Utr = Uty - UtX @ beta
        q = base * float(r @ r) + float(Utr @ (c * Utr))
        if not (q > 0.0) or not np.isfinite(q):
            return (np.inf, None) if want_q else np.inf
        logdet = (n - rank) * np.log1p(eta * r0) + np.log1p(eta * lam).sum()
        logdet += 2.0 * np.log(np.abs(np.diag(L))).sum()
        v = logdet + df * np.log(q / df)
        return (v, q) if want_q else v

    grid = 81
    vals = [objective(-12.0 + 24.0 * i / (grid - 1)) for i in range(grid)]
    best = int(np.argmin(vals))
    left = -12.0 + 24.0 * max(0, best - 1) / (grid - 1)
    right = -12.0 + 24.0 * min(grid - 1, best + 1) / (grid - 1)
    golden = (np.sqrt(5.0) - 1.0) / 2.0
    c = right - golden * (right - left)
    d = left + golden * (right - left)
    fc, fd = objective(c), objective(d)
    for _ in range(80):
        if right - left <= 1e-8:
            break
        if fc < fd:
            right, d, fd = d, c, fc
            c = right - golden * (right - left)
            fc = objective(c)
        else:
            left, c, fc = c, d, fd
            d = left + golden * (right - left)
            fd = objective(d)
    log_eta = 0.5 * (left + right)
    _, q = objective(log_eta, want_q=True)
    se2 = q / df
    return {"log_eta": log_eta, "sigma2_e": se2, "sigma2_g": np.exp(log_eta) * se2,
            "delta": np.exp(-log_eta)}


def lowrank_job_blas(bed: "Bed", y, X, variants=None, rank=256, oversample=10, seed=42,
                     min_maf=0.01, trace_threshold=0.95, min_rank=1, block=512, n_threads=None):
    """The whole `gwas --model lmm --fastlmm --fastlmm-matrix-free --no-loco` job on the CPU for
    every sample in .fam order: LmmEngine::prepareLowRankMatrixFree (src/lmm_engine.cpp:897-1095:
    Omega from mt19937_64 + normal_distribution, K Omega, two power iterations with QR, a final
    QR, B = Q^T K Q, its eigendecomposition, trace-fraction rank selection, tail-mean residual
    eigenvalue, REML grid + golden search) and LmmEngine::scanLowRank over every SNP of the file
    (src/lmm_engine.cpp:1269-1361), with Eigen's dense kernels as numpy BLAS/LAPACK calls.

    Each kinship apply is apply_block (src/kinship_operator.cpp:225-302): per block of 512
    selected SNPs, decode Z (n x 512) once and accumulate Z (Z^T V).  The scan forms, per block of
    512 SNPs, G^T [U | X | Py] with one GEMM and reads V^-1 g's quadratic forms from it
    (g^T V^-1 g = base g^T g + sum_j c_j (u_j^T g)^2), the same quantities as the reference's
    V^-1 G block without materialising it.  Returns a dict with sigma2_g / sigma2_e, the rank,
    per-SNP beta / se / log10p / freq / tested, and per-stage seconds."""
    import time

    threads = _threads(n_threads)
    y = np.ascontiguousarray(y, dtype=np.float64)
    X = np.asfortranarray(np.asarray(X, dtype=np.float64).reshape(len(y), -1))
    n, p = X.shape
    if n != bed.n:
        raise ValueError("lowrank_job_blas: every sample in .fam order is required")
    sel = (np.arange(bed.m, dtype=np.int32) if variants is None
           else np.ascontiguousarray(variants, dtype=np.int32))
    m_sel = len(sel)
    sk = min(n, rank + max(0, oversample))
    t = {}
    t0 = time.perf_counter()
    omega = normal_matrix(seed, n, sk)
    t["omega"] = time.perf_counter() - t0
    L = lib()
    zbuf = np.empty((n, block), order="F")
    trace_acc = [0.0]

    def apply(V, want_trace=False):
        out = np.zeros((n, V.shape[1]), order="F")
        for first in range(0, m_sel, block):
            cnt = min(block, m_sel - first)
            snps = sel[first:first + cnt]
            z = zbuf[:, :cnt]
            L.orc_decode_z_cols(_ptr(bed.rows), bed.stride, _ptr(bed.mean), _ptr(bed.inv_std),
                                _ptr(snps), cnt, n, z.ctypes.data, n, threads)
            proj = z.T @ V
            out += z @ proj
            if want_trace:
                trace_acc[0] += float(np.einsum("ij,ij->", z, z))
        out *= 1.0 / m_sel
        return out

    t0 = time.perf_counter()
    sample = apply(omega, want_trace=True)
    total_trace = trace_acc[0] / m_sel
    for _ in range(2):
        q, _ = np.linalg.qr(sample)
        sample = apply(q)
    q, _ = np.linalg.qr(sample)
    kq = apply(q)
    t["applies_qr"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    small = q.T @ kq
    small = 0.5 * (small + small.T)
    evals, evecs = np.linalg.eigh(small)
    lead = np.maximum(0.0, evals[::-1][:rank])
    selected = rank
    met = trace_threshold <= 0.0
    if trace_threshold > 0.0 and total_trace > 0.0:
        retained = np.cumsum(lead) / total_trace
        first_allowed = min(rank, max(1, min_rank))
        ok = np.nonzero((np.arange(1, rank + 1) >= first_allowed) & (retained >= trace_threshold))[0]
        if len(ok):
            selected = int(ok[0]) + 1
            met = True
    lam = lead[:selected].copy()
    U = np.asfortranarray(q @ evecs[:, ::-1][:, :selected])
    r0 = max(0.0, (total_trace - lam.sum()) / (n - selected))
    UtX = U.T @ X
    Uty = U.T @ y
    reml = _reml_search(lam, r0, n, p, float(y @ y), X.T @ y, X.T @ X, Uty, UtX, y, X)
    t["eigh_reml"] = time.perf_counter() - t0

    # ---- scanLowRank (src/lmm_engine.cpp:1269-1361)
    t0 = time.perf_counter()
    sg2, se2 = reml["sigma2_g"], reml["sigma2_e"]
    base = 1.0 / max(1e-12, sg2 * r0 + se2)
    c = 1.0 / (sg2 * lam + se2) - base
    info = base * (X.T @ X) + UtX.T @ (c[:, None] * UtX)
    info_inv = np.linalg.inv(info)
    vy = base * (X.T @ y) + UtX.T @ (c * Uty)
    beta_x = info_inv @ vy
    resid = y - X @ beta_x
    py = base * resid + U @ (c * (U.T @ resid))
    B = np.asfortranarray(np.column_stack([U, X, py]))
    m = bed.m
    out = {k: np.full(m, np.nan) for k in ("beta", "se", "log10p", "freq")}
    tested = np.zeros(m, dtype=bool)
    gbuf = np.empty((n, block), order="F")
    freq = np.empty(block)
    passed = np.empty(block, dtype=np.int32)
    gsq = np.empty(block)
    for first in range(0, m, block):
        cnt = min(block, m - first)
        G = gbuf[:, :cnt]
        L.orc_scan_encode_cols(_ptr(bed.rows), bed.stride, first, cnt, n, float(min_maf),
                               G.ctypes.data, n, _ptr(freq), _ptr(passed), _ptr(gsq), threads)
        A = G.T @ B                                  # cnt x (r + p + 1)
        UtG = A[:, :selected]
        XtG = A[:, selected:selected + p]
        score = A[:, selected + p]
        XtVG = base * XtG + UtG @ (c[:, None] * UtX)
        var = base * gsq[:cnt] + (UtG * UtG) @ c - np.einsum("ja,ab,jb->j", XtVG, info_inv, XtVG)
        ok = (passed[:cnt] != 0) & (var > 1e-12) & np.isfinite(var)
        sl = slice(first, first + cnt)
        out["freq"][sl] = np.where(ok, freq[:cnt], np.nan)
        with np.errstate(invalid="ignore", divide="ignore"):
            out["beta"][sl] = np.where(ok, score / var, np.nan)
            out["se"][sl] = np.where(ok, 1.0 / np.sqrt(var), np.nan)
            stat = np.where(ok, score * score / var, 0.0)
        pv = np.empty(cnt)
        L.orc_chisq_prob_vec(_ptr(np.ascontiguousarray(stat)), cnt, 1, _ptr(pv), threads)
        with np.errstate(divide="ignore"):
            out["log10p"][sl] = np.where(ok, np.where(pv > 0.0, -np.log10(np.maximum(pv, 1e-300)), 300.0), np.nan)
        tested[sl] = ok
    t["scan"] = time.perf_counter() - t0
    out["tested"] = tested
    out.update({"sigma2_g": sg2, "sigma2_e": se2, "rank": selected, "sketch": sk,
                "residual_eigenvalue": r0, "trace": total_trace, "trace_threshold_met": bool(met),
                "seconds": t, "threads": threads})
    return out


# ---------------------------------------------------------------- dense exact tier (numpy)
# Restatements of the default `gwas --model lmm` route for small n: GrmBuilder::compute,
# EigenVce::prepare / runNullModel (Brent) / updateRemlDiagnostics and LmmEngine::scan's exact
# branch.  Float roundings are taken where the reference stores floats.

def _codes(rows, n):
    """(b, stride) packed rows -> (b, n) 2-bit codes."""
    return np.stack([(rows >> (2 * q)) & 3 for q in range(4)], axis=2).reshape(rows.shape[0], -1)[:, :n]


def grm_snp(c00, c10, c11, algorithm=1, min_maf=0.01):
    """One SNP of GrmBuilder::compute (libCosmicCore/src/grm_builder.cpp:187-312): None when
    filtered, else (value map for codes 0..3, float 2pq)."""
    import math
    f32 = lambda x: float(np.float32(x))
    n_obs = c00 + c10 + c11
    if n_obs == 0:
        return None
    freq = float(2 * c00 + c10) / (2.0 * n_obs)
    maf = min(freq, 1.0 - freq)
    if maf < f32(min_maf) or abs(maf) < 1e-8:
        return None
    weight = 1.0
    p1, p2 = float(c10) / n_obs, float(c00) / n_obs
    if algorithm == 4:
        two_pq = f32(weight * 4.0 * freq * freq * (1.0 - freq) * (1.0 - freq))
    elif algorithm == 5:
        mu = p1 + 2.0 * p2
        two_pq = f32(weight * (p1 + 4.0 * p2 - mu * mu))
    else:
        two_pq = f32(weight * 2.0 * freq * (1.0 - freq))
    mean = f32(freq * 2.0)
    scale = 1.0
    if algorithm in (0, 3):
        pq2 = 2.0 * freq * (1.0 - freq)
        scale = f32(1.0 / math.sqrt(pq2) if pq2 > 1e-9 else 0.0)
    elif algorithm == 5:
        mu = p1 + 2.0 * p2
        var = p1 + 4.0 * p2 - mu * mu
        scale = f32(1.0 / math.sqrt(var) if var > 1e-9 else 0.0)
    if algorithm == 4:
        fp = mean / 2.0
        fq = 1.0 - fp
        vals = [(-2.0 * fq * fq) * scale, 0.0, (2.0 * fp * fq) * scale, (-2.0 * fp * fp) * scale]
    elif algorithm == 2:
        fp = mean / 2.0
        vals = [(1.0 - fp) * scale, 0.0, (1.0 - 2.0 * fp) * scale, (-fp) * scale]
    else:
        vals = [(2.0 - mean) * scale, 0.0, (1.0 - mean) * scale, (0.0 - mean) * scale]
    return vals, two_pq


def grm_dense(bed: "Bed", min_maf=0.01, algorithm=1, variants=None, block_size=2048,
              raw=False):
    """GrmBuilder::compute (grm_builder.cpp:140-394), one population, unit weights, no HWE:
    G = sum over 2048-SNP .bed blocks of Z Z^T, normalised (:383-391) unless raw (the
    per-chromosome sums of GrmBuilder::computeSplit, :687-712).  Returns (G, n_valid,
    sum_2pq)."""
    n, m = bed.n, bed.m
    sel = np.arange(m) if variants is None else np.asarray(variants, dtype=np.int64)
    G = np.zeros((n, n))
    total_2pq, total_valid = 0.0, 0
    for b0 in range(0, m, block_size):
        idx = sel[(sel >= b0) & (sel < b0 + block_size)]
        if len(idx) == 0:
            continue
        codes = _codes(bed.rows[idx], n)
        block_2pq, valid, vals = 0.0, [], []
        for r, j in enumerate(idx):
            c = np.bincount(codes[r], minlength=4)
            st = grm_snp(int(c[0]), int(c[2]), int(c[3]), algorithm, min_maf)
            if st is None:
                continue
            block_2pq += st[1]
            valid.append(j)
            vals.append(st[0])
        if not valid:
            continue
        Z = _decode_block(bed.rows[np.asarray(valid)], n, np.asarray(vals))
        G += Z @ Z.T
        total_2pq += block_2pq
        total_valid += len(valid)
    if raw:
        return G, total_valid, total_2pq
    if algorithm in (0, 3):
        if total_valid > 0:
            G /= float(total_valid)
    elif algorithm == 2:
        tr = np.trace(G)
        if tr > 0:
            G /= tr / n
    elif total_2pq > 0:
        G /= total_2pq
    return G, total_valid, total_2pq


def grm_loco(G, n_valid, sum_2pq, raw_chr, n_chr, sum_chr, algorithm=1):
    """The LOCO GRM of src/gwas_scanner.cpp:476-491."""
    by_count = algorithm in (0, 3)
    s = float(n_valid) if by_count else sum_2pq
    s_chr = float(n_chr) if by_count else sum_chr
    s_loco = s - s_chr
    if s_chr > 0.0 and s_loco > 1e-6:
        return G * (s / s_loco) - raw_chr / s_loco
    return G.copy()


def eigen_vce_prepare(G, y, X, projection=True):
    """EigenVce::prepare (libCosmicCore/src/eigen_vce.cpp:19-63): Householder QR of X, its
    complement A, eigh(A^T G A) with negative eigenvalues set to 0, W_proj = A U."""
    y = np.asarray(y, dtype=np.float64)
    X = np.asarray(X, dtype=np.float64).reshape(len(y), -1)
    n, p = X.shape
    if projection and p > 0:
        Q, _ = np.linalg.qr(X, mode="complete")
        A = Q[:, p:]
        D, U = np.linalg.eigh(A.T @ G @ A)
        D = np.maximum(D, 0.0)
        return D, A @ U, U.T @ (A.T @ y), np.zeros((n - p, 0))
    D, U = np.linalg.eigh(G)
    D = np.maximum(D, 0.0)
    return D, U, U.T @ y, U.T @ X


def solve_diagonal(D, Uty, UtX):
    """VCESolver::solveDiagonal (libCosmicCore/src/vce.cpp:3073-3175): golden-section search
    of the REML objective over log10 delta in [-5, 5], tol 1e-5."""
    import math
    n, p = len(D), UtX.shape[1]
    n_eff = float(n - p)

    def fit(delta):
        vd = D + delta
        vinv = 1.0 / vd
        xvx = UtX.T @ (vinv[:, None] * UtX)
        xvy = UtX.T @ (vinv * Uty)
        beta = np.linalg.solve(xvx, xvy) if p else np.zeros(0)
        logdet_xvx = np.linalg.slogdet(xvx)[1] if p else 0.0
        resid = Uty - UtX @ beta
        return float((resid ** 2 * vinv).sum()), float(np.log(vd).sum()), logdet_xvx, beta

    def neg(delta):
        quad, ldv, ldx, _ = fit(delta)
        return 0.5 * (ldv + ldx + n_eff * math.log(quad / n_eff) + n_eff)

    lo, hi = -5.0, 5.0
    gr = (math.sqrt(5.0) + 1.0) / 2.0
    c, d = hi - (hi - lo) / gr, lo + (hi - lo) / gr
    fc, fd = neg(10.0 ** c), neg(10.0 ** d)
    while abs(c - d) > 1e-5:
        if fc < fd:
            hi, d, fd = d, c, fc
            c = hi - (hi - lo) / gr
            fc = neg(10.0 ** c)
        else:
            lo, c, fc = c, d, fd
            d = lo + (hi - lo) / gr
            fd = neg(10.0 ** d)
    best = 10.0 ** ((lo + hi) / 2.0)
    quad, _, _, beta = fit(best)
    vg = quad / n_eff
    ve = vg * best
    return {"sigma2_g": vg, "sigma2_e": ve, "delta": ve / vg, "beta": beta,
            "sigma2_g_se": vg * math.sqrt(2.0 / n_eff), "sigma2_e_se": ve * math.sqrt(2.0 / n_eff)}


def reml_diagnostics(D, Uty, UtX, sg, se):
    """EigenVce::updateRemlDiagnostics (eigen_vce.cpp:114-153) with the dense P."""
    import math
    n, p = len(D), UtX.shape[1]
    cov = np.maximum(sg * D + se, 1e-12)
    inv = 1.0 / cov
    P = np.diag(inv)
    log_det_fixed = 0.0
    if p:
        info = UtX.T @ (inv[:, None] * UtX)
        P -= (inv[:, None] * UtX) @ np.linalg.inv(info) @ (UtX.T * inv[None, :])
        log_det_fixed = np.linalg.slogdet(info)[1]
    py = P @ Uty
    kpy = D * py
    score = [0.5 * (py @ kpy - (np.diag(P) * D).sum()), 0.5 * (py @ py - np.trace(P))]
    ai = 0.5 * np.array([[kpy @ P @ kpy, kpy @ P @ py], [kpy @ P @ py, py @ P @ py]])
    cinv = np.linalg.inv(ai)
    return {"sigma2_g_se": math.sqrt(max(0.0, cinv[0, 0])),
            "sigma2_e_se": math.sqrt(max(0.0, cinv[1, 1])),
            "max_score": max(abs(score[0]), abs(score[1])),
            "log_likelihood": -0.5 * (np.log(cov).sum() + log_det_fixed + Uty @ py +
                                      (n - p) * math.log(2.0 * math.pi))}


def eigen_vce_iterative_reml(D, Uty, UtX, average_information=True, max_iter=100, tol=1e-6):
    """EigenVce::runIterativeReml (libCosmicCore/src/eigen_vce.cpp:155-252): exact FP64 REML
    in the eigenbasis from theta = (var/2, var/2), var = |U'y|^2 / df; AI steps with up to 40
    halvings while the log-likelihood drops by more than 1e-10 (EM: the 0.5-blended ratio
    update), stopping when the largest relative change < tol.  Returns sigma2_g, sigma2_e,
    their AI standard errors, the log-likelihood, the score, iterations and converged."""
    import math
    D = np.asarray(D, dtype=np.float64)
    Uty = np.asarray(Uty, dtype=np.float64)
    UtX = np.asarray(UtX, dtype=np.float64).reshape(len(D), -1)
    n, p = len(D), UtX.shape[1]
    df = n - p
    if df < 2:
        raise ValueError("EigenVce REML requires residual degrees of freedom")
    pvar = max(1e-10, float(Uty @ Uty) / df)
    lower = pvar * 1e-10

    def evaluate(theta):
        cov = np.maximum(theta[0] * D + theta[1], lower)
        inv = 1.0 / cov
        if p:
            info = UtX.T @ (inv[:, None] * UtX)
            info_inv = np.linalg.inv(info)
            log_det_fixed = float(np.linalg.slogdet(info)[1])
            B = inv[:, None] * UtX              # diag(inv) U'X

            def P(v):
                return inv * v - B @ (info_inv @ (B.T @ v))
            pdiag = inv - np.einsum("ia,ab,ib->i", B, info_inv, B)
        else:
            log_det_fixed = 0.0

            def P(v):
                return inv * v
            pdiag = inv
        py = P(Uty)
        kpy = D * py
        t = {"trace_g": float((pdiag * D).sum()), "trace_e": float(pdiag.sum()),
             "quad_g": float(py @ kpy), "quad_e": float(py @ py)}
        t["score"] = np.array([0.5 * (t["quad_g"] - t["trace_g"]), 0.5 * (t["quad_e"] - t["trace_e"])])
        pk, pp = P(kpy), P(py)
        t["ai"] = 0.5 * np.array([[kpy @ pk, kpy @ pp], [kpy @ pp, py @ pp]])
        t["logl"] = -0.5 * (float(np.log(cov).sum()) + log_det_fixed + float(Uty @ py) +
                            df * math.log(2.0 * math.pi))
        return t

    theta = np.array([0.5 * pvar, 0.5 * pvar])
    cur = evaluate(theta)
    converged, iterations = False, 0
    for it in range(max_iter):
        prop = theta.copy()
        if average_information:
            try:
                step = np.linalg.solve(cur["ai"], cur["score"])
            except np.linalg.LinAlgError:
                break
            frac = 1.0
            for _ in range(40):
                prop = np.maximum(theta + frac * step, lower)
                if evaluate(prop)["logl"] >= cur["logl"] - 1e-10:
                    break
                frac *= 0.5
        else:
            prop = np.array([theta[0] * cur["quad_g"] / max(1e-12, cur["trace_g"]),
                             theta[1] * cur["quad_e"] / max(1e-12, cur["trace_e"])])
            prop = np.maximum(0.5 * theta + 0.5 * prop, lower)
        change = float((np.abs(prop - theta) / (np.abs(theta) + pvar * 1e-8)).max())
        theta = prop
        cur = evaluate(theta)
        iterations = it + 1
        if change < tol:
            converged = True
            break
    sg = max(0.0, 0.0 if theta[0] <= 1.01 * lower else theta[0])
    se = max(0.0, 0.0 if theta[1] <= 1.01 * lower else theta[1])
    cinv = np.linalg.inv(cur["ai"])
    return {"sigma2_g": sg, "sigma2_e": se, "logl": cur["logl"],
            "sigma2_g_se": math.sqrt(max(0.0, cinv[0, 0])),
            "sigma2_e_se": math.sqrt(max(0.0, cinv[1, 1])),
            "score": cur["score"], "ai": cur["ai"], "iterations": iterations,
            "converged": converged}


def hutchinson_vc_sd(K, X, sigma2_g, sigma2_e, probes):
    """Predicted standard deviation of the variance components that a REML fit with
    Hutchinson trace estimates (Rademacher probes, `probes` per trace) settles on, around the
    exact REML solution: the trace estimates z'P K z / S and z'P z / S carry the covariance
    2/S sum_{i!=j} A_ij B_ij of their symmetrised matrices A = (PK + KP)/2, B = P, the score
    error is -1/2 of it, and the fitted components move by AI^-1 times the score error
    (AI the exact average information, P = V^-1 - V^-1 X (X'V^-1 X)^-1 X'V^-1 at the solution).
    Dense n x n algebra: for n of a few thousand."""
    n = K.shape[0]
    X = np.asarray(X, dtype=np.float64).reshape(n, -1)
    V = sigma2_g * K + sigma2_e * np.eye(n)
    Vi = np.linalg.inv(V)
    ViX = Vi @ X
    P = Vi - ViX @ np.linalg.solve(X.T @ ViX, ViX.T)
    PK = P @ K
    A = 0.5 * (PK + PK.T)
    mats = [A, P]
    cov = np.zeros((2, 2))
    for a in range(2):
        for b in range(2):
            Ma, Mb = mats[a], mats[b]
            cov[a, b] = 2.0 * ((Ma * Mb).sum() - (np.diag(Ma) * np.diag(Mb)).sum()) / probes
    score_cov = 0.25 * cov
    ai = 0.5 * np.array([[np.sum(PK * PK.T), np.sum(PK * P.T)], [np.sum(PK * P.T), np.sum(P * P)]])
    aiinv = np.linalg.inv(ai)
    vc_cov = aiinv @ score_cov @ aiinv.T
    return np.sqrt(np.maximum(np.diag(vc_cov), 0.0))


def scan_exact(bed: "Bed", keep, W, D, Uty, UtX, sg, se, min_maf=0.01, use_residuals=False,
               block=512):
    """LmmEngine::scan's exact branch (src/lmm_engine.cpp:1363-1474) over every SNP."""
    keep = np.asarray(keep, dtype=np.int64)
    n = len(keep)
    p = UtX.shape[1]
    vinv = 1.0 / (sg * D + se)
    wutx = UtX * vinv[:, None]
    inv = np.linalg.inv(UtX.T @ wutx) if p else np.zeros((0, 0))
    bx = inv @ (UtX.T @ (vinv * Uty)) if p else np.zeros(0)
    py = (Uty - UtX @ bx) * vinv
    out = {k: np.full(bed.m, np.nan) for k in ("beta", "se", "p", "log10p", "freq")}
    out["tested"] = np.zeros(bed.m, dtype=bool)
    for b0 in range(0, bed.m, block):
        codes = _codes(bed.rows[b0:b0 + block], bed.n)[:, keep]
        cols, idx = [], []
        for r in range(codes.shape[0]):
            raw = np.array([2.0, np.nan, 1.0, 0.0])[codes[r]]
            ok, vals, f, _ = prepare_marker(raw, min_maf)
            if not ok:
                continue
            cols.append(vals)
            idx.append(b0 + r)
            out["freq"][b0 + r] = f
        if not cols:
            continue
        utg = W.T @ np.array(cols).T
        scores = utg.T @ py
        var = (utg * (utg * vinv[:, None])).sum(axis=0)
        if not use_residuals and p:
            xvg = wutx.T @ utg
            var -= (xvg * (inv @ xvg)).sum(axis=0)
        for c, j in enumerate(idx):
            v = var[c]
            if not (v > 1e-12) or not np.isfinite(v):
                continue
            s = np.sqrt(v)
            stat = scores[c] / s
            pv = chisq_prob(stat * stat, 1)
            out["beta"][j] = scores[c] / v
            out["se"][j] = 1.0 / s
            out["p"][j] = pv
            out["log10p"][j] = -np.log10(pv) if pv > 0 else 300.0
            out["tested"][j] = True
    return out


# ---------------------------------------------------------------- MvEigenVce (numpy)

def mv_eigen_vce_prepare(G, Y, X, projection=True):
    """MvEigenVce::prepare (libCosmicCore/src/eigen_vce.cpp:496-549): the eigenbasis of
    eigen_vce_prepare with U'Y for every trait, and Vg = Ve = Cov(Y) / 2 divided by (samples
    after the projection - 1)."""
    Y = np.asarray(Y, dtype=np.float64)
    D, W, UtY, UtX = eigen_vce_prepare(G, Y, X, projection)
    n_after = len(D)
    Yc = Y - Y.mean(axis=0)
    cov = Yc.T @ Yc / (n_after - 1)
    return D, W, UtY, UtX, 0.5 * cov, 0.5 * cov.copy()


def mv_em_step(D, UtY, Vg, Ve):
    """MvEigenVce::updateEM (:551-604) with no covariates left (after the projection)."""
    n = len(D)
    V = D[:, None, None] * Vg + Ve
    P = np.linalg.inv(V)
    Wg = D[:, None, None] * (Vg @ P)
    u = np.einsum("iab,ib->ia", Wg, UtY)
    pos = D > 1e-12
    Sg = np.where(pos[:, None, None],
                  np.einsum("ia,ib->iab", u, u) / np.where(pos, D, 1.0)[:, None, None]
                  + Vg - Wg @ Vg, Vg).sum(axis=0)
    We = Ve @ P
    e = np.einsum("iab,ib->ia", We, UtY)
    Se = (np.einsum("ia,ib->iab", e, e) + Ve - We @ Ve).sum(axis=0)
    return Sg / n, Se / n


def mv_loglik(D, UtY, Vg, Ve):
    """MvEigenVce::calcLogLikelihood (:613-629)."""
    d = Vg.shape[0]
    V = D[:, None, None] * Vg + Ve + 1e-8 * np.eye(d)
    sign, ld = np.linalg.slogdet(V)
    sol = np.linalg.solve(V, UtY[:, :, None])[:, :, 0]
    return float((-0.5 * (ld + (UtY * sol).sum(axis=1))).sum())


def mv_stcg_em(K, Y, X, max_iter=10, tol=1e-8, mc_samples=32, probe_seed=20250101,
               exact_traces=False):
    """The multi-trait REML-EM of MvEigenVce::updateEM (libCosmicCore/src/eigen_vce.cpp:551-604)
    written for a general covariance V = Vg (x) K + Ve (x) I instead of the eigenbasis, with the
    covariates kept in P = V^-1 - V^-1 Xf (Xf' V^-1 Xf)^-1 Xf' V^-1, Xf = I_d (x) X:
        Vg <- Vg + Vg (Qg - Tg) Vg / (n - p),  Ve <- Ve + Ve (Qe - Te) Ve / (n - p),
        Qg = (PY)' K (PY), Qe = (PY)' (PY), Tg[a, b] = tr(P (E_ab (x) K)), Te[a, b] = tr(P (E_ab (x) I))
    (in the eigenbasis this is the reference's per-sample update).  The traces are Hutchinson
    estimates with mc_samples Rademacher probes of n x d per iteration, redrawn every iteration
    from one mt19937_64 stream (probe s, trait a = column s d + a), unless exact_traces.  Dense
    n d x n d algebra: the checker of the matrix-free GPU form at small n.  Starting values
    Vg = Ve = Cov(Y) / 2 over n - p - 1 (:536-548); stop when
    (|dVg|^2 + |dVe|^2) / max(1, 2 d^2) < tol.  Returns (Vg, Ve, iterations, converged)."""
    K = np.asarray(K, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    n, d = Y.shape
    X = np.asarray(X, dtype=np.float64).reshape(n, -1)
    p = X.shape[1]
    Yc = Y - Y.mean(axis=0)
    cov = Yc.T @ Yc / (n - p - 1)
    Vg, Ve = 0.5 * cov, 0.5 * cov.copy()
    I = np.eye(n)
    Xf = np.kron(np.eye(d), X)
    drawn = 0
    for it in range(max_iter):
        V = np.kron(Vg, K) + np.kron(Ve, I)
        Vi = np.linalg.inv(V)
        ViX = Vi @ Xf
        info = Xf.T @ ViX
        P = Vi - ViX @ np.linalg.solve(info, ViX.T)
        PY = (P @ Y.reshape(-1, order="F")).reshape(n, d, order="F")
        Qg, Qe = PY.T @ K @ PY, PY.T @ PY
        if exact_traces:
            Tg = np.array([[np.trace(P[b * n:(b + 1) * n, a * n:(a + 1) * n] @ K) for b in range(d)]
                           for a in range(d)])
            Te = np.array([[np.trace(P[b * n:(b + 1) * n, a * n:(a + 1) * n]) for b in range(d)]
                           for a in range(d)])
        else:
            Z = rademacher(probe_seed, drawn, n, mc_samples * d)
            drawn += n * mc_samples * d
            Tg = np.zeros((d, d))
            Te = np.zeros((d, d))
            for s_ in range(mc_samples):
                Zs = Z[:, s_ * d:(s_ + 1) * d]
                PZ = (P @ Zs.reshape(-1, order="F")).reshape(n, d, order="F")
                Tg += PZ.T @ (K @ Zs)
                Te += PZ.T @ Zs
            Tg /= mc_samples
            Te /= mc_samples
        Tg, Te = 0.5 * (Tg + Tg.T), 0.5 * (Te + Te.T)
        Vg_new = Vg + Vg @ (Qg - Tg) @ Vg / (n - p)
        Ve_new = Ve + Ve @ (Qe - Te) @ Ve / (n - p)
        Vg_new, Ve_new = 0.5 * (Vg_new + Vg_new.T), 0.5 * (Ve_new + Ve_new.T)
        err = (((Vg_new - Vg) ** 2).sum() + ((Ve_new - Ve) ** 2).sum()) / max(1.0, 2.0 * d * d)
        Vg, Ve = Vg_new, Ve_new
        if err < tol:
            return Vg, Ve, it + 1, True
    return Vg, Ve, max_iter, False


def _near_pd(M):
    ev, Q = np.linalg.eigh(M)
    if ev.min() <= 1e-10:
        return (Q * np.maximum(ev, 1e-10)) @ Q.T
    return M


def _mv_score_ai(D, UtY, Vg, Ve, pairs):
    d = Vg.shape[0]
    vs = len(pairs)
    V = D[:, None, None] * Vg + Ve + 1e-8 * np.eye(d)
    Vi = np.linalg.inv(V)
    v = np.einsum("iab,ib->ia", Vi, UtY)
    w = np.zeros((len(D), vs, d))
    for a, (p, q) in enumerate(pairs):
        w[:, a] = v[:, p, None] * Vi[:, :, p] if p == q else \
            v[:, q, None] * Vi[:, :, p] + v[:, p, None] * Vi[:, :, q]
    score = np.zeros(2 * vs)
    AI = np.zeros((2 * vs, 2 * vs))
    for a, (j, k) in enumerate(pairs):
        vjvk = v[:, j] * v[:, k]
        tr = Vi[:, j, j] if j == k else 2.0 * Vi[:, j, k]
        quad = vjvk if j == k else 2.0 * vjvk
        score[a] = (0.5 * D * (quad - tr)).sum()
        score[a + vs] = (0.5 * (quad - tr)).sum()
        for b in range(a, vs):
            qv = v[:, j] * w[:, b, j] if j == k else v[:, j] * w[:, b, k] + v[:, k] * w[:, b, j]
            qv = 0.5 * qv
            AI[a, b] += (D * D * qv).sum()
            AI[a, vs + b] += (D * qv).sum()
            AI[vs + a, b] += (D * qv).sum()
            AI[vs + a, vs + b] += qv.sum()
    return score, 0.5 * (AI + AI.T)


def mv_run_null(D, UtY, Vg, Ve, max_iter=1000, tol=1e-8, aireml=False, em_min_iter=10,
                ai_max_iter=50, ai_tol=1e-8):
    """MvEigenVce::runNullModel (:1031-1065): EM, or runAireml (:631-911).  Returns
    (converged, iterations, Vg, Ve, Vg_se, Ve_se, logl)."""
    d = Vg.shape[0]
    zeros = np.zeros((d, d))

    def em(Vg, Ve):
        Vg_new, Ve_new = mv_em_step(D, UtY, Vg, Ve)
        err = (((Vg_new - Vg) ** 2).sum() + ((Ve_new - Ve) ** 2).sum()) / max(1.0, 2.0 * d * d)
        return Vg_new, Ve_new, err

    if not aireml:
        for it in range(max_iter):
            Vg, Ve, err = em(Vg, Ve)
            if err < tol:
                return True, it + 1, Vg, Ve, zeros, zeros, mv_loglik(D, UtY, Vg, Ve)
        return False, max_iter, Vg, Ve, zeros, zeros, mv_loglik(D, UtY, Vg, Ve)
    pairs = [(j, k) for j in range(d) for k in range(j, d)]
    vs = len(pairs)
    em_iter = 0
    while em_iter < max_iter:
        Vg, Ve, err = em(Vg, Ve)
        if err < tol and em_iter >= em_min_iter:
            break
        em_iter += 1
    iters = min(em_iter + 1, max_iter)
    Vg, Ve = _near_pd(Vg), _near_pd(Ve)
    logl_old = mv_loglik(D, UtY, Vg, Ve)
    logl_init, Vg0, Ve0 = logl_old, Vg.copy(), Ve.copy()
    if not np.isfinite(logl_old):
        return True, iters, Vg, Ve, zeros, zeros, logl_old
    for it in range(ai_max_iter):
        score, AI = _mv_score_ai(D, UtY, Vg, Ve, pairs)
        AI[np.diag_indices_from(AI)] *= 1.0 + 1e-8
        delta = np.linalg.solve(AI, score)
        step, accepted = 1.0, False
        for h in range(12):
            Vg_t, Ve_t = Vg.copy(), Ve.copy()
            for a, (j, k) in enumerate(pairs):
                Vg_t[j, k] += step * delta[a]
                Vg_t[k, j] = Vg_t[j, k]
                Ve_t[j, k] += step * delta[a + vs]
                Ve_t[k, j] = Ve_t[j, k]
            Vg_t, Ve_t = _near_pd(Vg_t), _near_pd(Ve_t)
            ll = mv_loglik(D, UtY, Vg_t, Ve_t)
            if np.isfinite(ll) and ll >= logl_old - 1e-10:
                accepted = True
                break
            step *= 0.5
        if not accepted:
            break
        Vg, Ve = Vg_t, Ve_t
        logl_old = mv_loglik(D, UtY, Vg, Ve)
        if np.linalg.norm(delta) / np.sqrt(2 * vs) < ai_tol:
            return True, iters, Vg, Ve, zeros, zeros, logl_old
    if logl_old < logl_init + 1e-8:
        Vg, Ve, logl_old = Vg0, Ve0, logl_init
    score, AI = _mv_score_ai(D, UtY, Vg, Ve, pairs)
    AI[np.diag_indices_from(AI)] *= 1.0 + 1e-8
    inv = np.linalg.inv(AI)
    Vg_se, Ve_se = np.zeros((d, d)), np.zeros((d, d))
    for a, (j, k) in enumerate(pairs):
        Vg_se[j, k] = Vg_se[k, j] = np.sqrt(abs(inv[a, a]))
        Ve_se[j, k] = Ve_se[k, j] = np.sqrt(abs(inv[vs + a, vs + a]))
    return True, iters, Vg, Ve, Vg_se, Ve_se, logl_old
