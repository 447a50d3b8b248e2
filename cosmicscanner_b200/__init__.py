"""cosmicscanner_b200 — B200 (sm_100a) matrix-free mixed-model path of CosmicScanner.

Python mirror of the reference's C++ interfaces over the library's C ABI
(``include/cosmicscanner_b200.h``):

* :class:`Genotypes`        — ``PlinkReader`` (libCosmicCore/src/plink_reader.h)
* :class:`KinshipOperator`  — ``KinshipOperator`` / ``createKinshipOperator``
                              (src/kinship_operator.h:18-101)
* :class:`LmmEngine`        — ``LmmEngine::prepareLowRankMatrixFree`` / ``scan``
                              (src/lmm_engine.h:108-131)
* :class:`MatrixFreePCG`    — ``MatrixFreePCG`` (libCosmicCore/src/matrix_free_pcg.h:9-75)
* :class:`StcgVce`          — ``STCG_VCE`` (libCosmicCore/src/stcg_vce.h:7-54)
* :class:`Server`           — resident-genotype request loop (no reference counterpart)

Every compute call runs the CUDA kernels in ``libcosmicscanner_b200.so``; there is
no CPU fallback.  A missing library or CUDA device raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi

PRECISION = {"fp64": 0, "mixed": 1}


class CosmicError(RuntimeError):
    """Raised when a library call returns a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class InvalidArgument(CosmicError, ValueError):
    pass


def _check(rc: int):
    if rc != 0:
        msg = _abi.lib().cs_last_error().decode()
        if rc == _abi.CS_ERR_INVALID_ARGUMENT:
            raise InvalidArgument(rc, msg)
        raise CosmicError(rc, msg)


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _prec(p):
    return PRECISION[p] if isinstance(p, str) else int(p)


class Genotypes:
    """Resident packed genotype matrix (+ per-SNP mean and 1/sd over all samples)."""

    def __init__(self, handle, n_samples: int, n_snps: int):
        self._h = handle
        self.n_samples = n_samples
        self.n_snps = n_snps

    @classmethod
    def from_bed_bytes(cls, bed: np.ndarray, n_samples: int, n_snps: int) -> "Genotypes":
        bed = np.ascontiguousarray(bed, dtype=np.uint8)
        h = C.c_void_p()
        _check(_abi.lib().cs_genotypes_create(_ptr(bed), bed.nbytes, n_samples, n_snps, C.byref(h)))
        return cls(h, n_samples, n_snps)

    @classmethod
    def open_plink(cls, prefix: str) -> "Genotypes":
        h = C.c_void_p()
        _check(_abi.lib().cs_genotypes_open_plink(prefix.encode(), C.byref(h)))
        n, m, bps = C.c_int64(), C.c_int64(), C.c_int64()
        _check(_abi.lib().cs_genotypes_info(h, C.byref(n), C.byref(m), C.byref(bps)))
        return cls(h, n.value, m.value)

    def stats(self):
        m = self.n_snps
        mean, inv_std, s = np.zeros(m), np.zeros(m), np.zeros(m)
        count = np.zeros(m, dtype=np.int32)
        _check(_abi.lib().cs_genotypes_stats(self._h, _ptr(mean), _ptr(inv_std), _ptr(count), _ptr(s)))
        return {"mean": mean, "inv_std": inv_std, "count": count, "sum": s}

    def close(self):
        if self._h:
            _abi.lib().cs_genotypes_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KinshipOperator:
    """K = Z Z^T / M over a sample / variant selection; mirrors cosmic::KinshipOperator."""

    def __init__(self, genotypes: Genotypes, keep=None, variants=None):
        self._g = genotypes  # keeps the matrix alive, like the reference's non-owning reader
        self._keep = None if keep is None or len(keep) == 0 else np.ascontiguousarray(keep, dtype=np.int32)
        self._var = None if variants is None or len(variants) == 0 else np.ascontiguousarray(variants, dtype=np.int32)
        h = C.c_void_p()
        _check(_abi.lib().cs_kinship_create(
            genotypes._h, _ptr(self._keep), 0 if self._keep is None else len(self._keep),
            _ptr(self._var), 0 if self._var is None else len(self._var), C.byref(h)))
        self._h = h
        r, m = C.c_int64(), C.c_int64()
        _check(_abi.lib().cs_kinship_info(h, C.byref(r), C.byref(m)))
        self._rows, self._m = r.value, m.value

    def rows(self) -> int:
        return self._rows

    def cols(self) -> int:
        return self._rows

    def numVariants(self) -> int:
        return self._m

    def isDense(self) -> bool:
        return False

    def apply(self, X, precision="fp64") -> np.ndarray:
        """out = K X for a vector (rows,) or matrix (rows, k); host arrays."""
        X = np.asarray(X, dtype=np.float64)
        vec = X.ndim == 1
        Xf = np.asfortranarray(X.reshape(-1, 1) if vec else X)
        if Xf.shape[0] != self._rows:
            raise InvalidArgument(_abi.CS_ERR_INVALID_ARGUMENT,
                                  "PlinkKinshipOperator::apply: dimension mismatch")
        k = Xf.shape[1]
        out = np.zeros((self._rows, k), order="F")
        _check(_abi.lib().cs_kinship_apply_host(self._h, _ptr(Xf), self._rows, k, _ptr(out),
                                                self._rows, _prec(precision)))
        return out[:, 0] if vec else out

    applyTranspose = apply

    def apply_device(self, X_ptr: int, ldx: int, k: int, Y_ptr: int, ldy: int,
                     precision="fp64", stream: int = 0):
        """Device-pointer apply (column-major, leading dimensions in elements)."""
        _check(_abi.lib().cs_kinship_apply(self._h, C.c_void_p(X_ptr), ldx, k, C.c_void_p(Y_ptr),
                                           ldy, _prec(precision), C.c_void_p(stream)))

    def apply_device_f32(self, X_ptr: int, ldx: int, k: int, Y_ptr: int, ldy: int,
                         precision="fp64", stream: int = 0):
        """The FP32 device apply (float column-major X and Y, FP64 inside)."""
        _check(_abi.lib().cs_kinship_apply_f32(self._h, C.c_void_p(X_ptr), ldx, k,
                                               C.c_void_p(Y_ptr), ldy, _prec(precision),
                                               C.c_void_p(stream)))

    def multiply_Zt_v(self, X, precision="fp64") -> np.ndarray:
        """GenotypeMatrix::multiply_Zt_v (libCosmicCore/src/matrix_adapter.h:40-53): Z^T X over
        the selection, X (rows,) or (rows, k) -> (numVariants,) or (numVariants, k)."""
        X = np.asarray(X, dtype=np.float64)
        vec = X.ndim == 1
        Xf = np.asfortranarray(X.reshape(-1, 1) if vec else X)
        if Xf.shape[0] != self._rows:
            raise InvalidArgument(_abi.CS_ERR_INVALID_ARGUMENT, "Dimension mismatch in multiply_Zt_v")
        k = Xf.shape[1]
        out = np.zeros((self._m, k), order="F")
        _check(_abi.lib().cs_genotype_multiply_zt_host(self._h, _ptr(Xf), Xf.shape[0], k,
                                                       _ptr(out), self._m, _prec(precision)))
        return out[:, 0] if vec else out

    def multiply_Z_v(self, V, precision="fp64") -> np.ndarray:
        """GenotypeMatrix::multiply_Z_v: Z V over the selection, V (numVariants,) or
        (numVariants, k) -> (rows,) or (rows, k)."""
        V = np.asarray(V, dtype=np.float64)
        vec = V.ndim == 1
        Vf = np.asfortranarray(V.reshape(-1, 1) if vec else V)
        if Vf.shape[0] != self._m:
            raise InvalidArgument(_abi.CS_ERR_INVALID_ARGUMENT, "Dimension mismatch in multiply_Z_v")
        k = Vf.shape[1]
        out = np.zeros((self._rows, k), order="F")
        _check(_abi.lib().cs_genotype_multiply_z_host(self._h, _ptr(Vf), Vf.shape[0], k,
                                                      _ptr(out), self._rows, _prec(precision)))
        return out[:, 0] if vec else out

    def trace(self) -> float:
        t = C.c_double()
        _check(_abi.lib().cs_kinship_trace(self._h, C.byref(t)))
        return t.value

    def getDiagonal(self) -> np.ndarray:
        d = np.zeros(self._rows)
        _check(_abi.lib().cs_kinship_diagonal(self._h, _ptr(d)))
        return d

    def close(self):
        if self._h:
            _abi.lib().cs_kinship_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def createKinshipOperator(reader: Genotypes, keep_indices=None, variant_indices=None):
    return KinshipOperator(reader, keep_indices, variant_indices)


def profile_enable(on: bool = True):
    """Starts (and resets) or stops CUDA-event timing of the library's kernels."""
    _check(_abi.lib().cs_profile_enable(1 if on else 0))


def profile_summary() -> dict:
    """Per kernel name: launches, summed device ms, algorithmic flops and bytes."""
    import json

    need = C.c_size_t()
    _check(_abi.lib().cs_profile_summary(None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value + 1024)
    _check(_abi.lib().cs_profile_summary(buf, len(buf), None))
    return json.loads(buf.value.decode())


def normal_matrix(seed: int, n: int, cols: int) -> np.ndarray:
    """The reference's Gaussian test matrix (mt19937_64 + std::normal_distribution), drawn on
    the device: n x cols, filled column by column."""
    out = np.zeros((n, cols), order="F")
    _check(_abi.lib().cs_normal_matrix(seed, n, cols, _ptr(out)))
    return out


def launch_count() -> int:
    """Process-wide number of kernel launches the library has made."""
    n = C.c_int64()
    _check(_abi.lib().cs_launch_count(C.byref(n)))
    return n.value


class LowRankDiagnostics(C.Structure):
    _fields_ = [
        ("requested_rank", C.c_int32), ("effective_rank", C.c_int32),
        ("sketch_size", C.c_int32), ("trace_threshold_met", C.c_int32),
        ("residual_eigenvalue", C.c_double), ("relative_frobenius_error", C.c_double),
        ("trace", C.c_double), ("trace_fraction", C.c_double),
        ("sigma2_g", C.c_double), ("sigma2_e", C.c_double), ("delta", C.c_double),
        ("log_eta", C.c_double), ("reml_objective", C.c_double), ("seconds", C.c_double),
    ]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class LmmEngine:
    """Low-rank matrix-free LMM: mirrors LmmEngine (src/lmm_engine.cpp:897-1361)."""

    def __init__(self):
        h = C.c_void_p()
        _check(_abi.lib().cs_lmm_create(C.byref(h)))
        self._h = h
        self.diagnostics = None

    def prepareLowRankMatrixFree(self, y, X, kinship: KinshipOperator, rank=256, oversample=10,
                                 seed=42, trace_threshold=0.95, min_rank=1, precision="fp64"):
        y = np.ascontiguousarray(y, dtype=np.float64)
        # the reference receives covariates as Eigen::MatrixXf and casts them to double
        X = np.asfortranarray(np.asarray(X, dtype=np.float32).astype(np.float64))
        d = LowRankDiagnostics()
        _check(_abi.lib().cs_lmm_prepare_lowrank_matrix_free(
            self._h, kinship._h, _ptr(y), _ptr(X), X.shape[1], rank, oversample, seed,
            trace_threshold, min_rank, _prec(precision), C.byref(d)))
        self.diagnostics = d.as_dict()
        self._n = kinship.rows()
        return self.diagnostics

    def prepareFromVce(self, vce: "EigenVce", use_residuals: bool = False):
        """LmmEngine::prepareFromVce (src/lmm_engine.cpp:716-725): scan() then runs the exact
        scan of lmm_engine.cpp:1363-1474 on the EigenVce's basis and null model
        (use_residuals: the reference's setting for GRM algorithm 0)."""
        _check(_abi.lib().cs_lmm_prepare_from_vce(self._h, vce._h, int(bool(use_residuals))))
        self.diagnostics = dict(vce.result)
        self._n = vce.n

    def getSigma2g(self):
        return self.diagnostics["sigma2_g"]

    def getSigma2e(self):
        return self.diagnostics["sigma2_e"]

    def lowrank_basis(self):
        r = self.diagnostics["effective_rank"]
        U = np.zeros((self._n, r), order="F")
        lam = np.zeros(r)
        _check(_abi.lib().cs_lmm_lowrank_basis(self._h, _ptr(U), self._n, _ptr(lam)))
        return U, lam

    def scan(self, reader: Genotypes, keep_indices, min_maf=0.01, precision="fp64"):
        keep = np.ascontiguousarray(keep_indices, dtype=np.int32)
        m = reader.n_snps
        out = {k: np.zeros(m) for k in ("beta", "se", "p", "log10p", "freq")}
        tested = np.zeros(m, dtype=np.int32)
        _check(_abi.lib().cs_lmm_scan(self._h, reader._h, _ptr(keep), len(keep), min_maf,
                                      _prec(precision), _ptr(out["beta"]), _ptr(out["se"]),
                                      _ptr(out["p"]), _ptr(out["log10p"]), _ptr(out["freq"]),
                                      _ptr(tested)))
        out["tested"] = tested.astype(bool)
        return out

    def scan_window(self, reader: Genotypes, keep_indices, snp_begin: int, snp_end: int,
                    min_maf=0.01, precision="fp64"):
        """scan() over SNPs [snp_begin, snp_end) only (a LOCO chromosome)."""
        keep = np.ascontiguousarray(keep_indices, dtype=np.int32)
        w = int(snp_end) - int(snp_begin)
        out = {k: np.zeros(max(w, 0)) for k in ("beta", "se", "p", "log10p", "freq")}
        tested = np.zeros(max(w, 0), dtype=np.int32)
        _check(_abi.lib().cs_lmm_scan_window(self._h, reader._h, _ptr(keep), len(keep),
                                             int(snp_begin), int(snp_end), min_maf,
                                             _prec(precision), _ptr(out["beta"]), _ptr(out["se"]),
                                             _ptr(out["p"]), _ptr(out["log10p"]),
                                             _ptr(out["freq"]), _ptr(tested)))
        out["tested"] = tested.astype(bool)
        return out

    def close(self):
        if self._h:
            _abi.lib().cs_lmm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- dense exact tier

class GrmOptions(C.Structure):
    _fields_ = [("min_maf", C.c_double), ("algorithm", C.c_int32)]


class EigenVceResult(C.Structure):
    _fields_ = [
        ("sigma2_g", C.c_double), ("sigma2_e", C.c_double), ("delta", C.c_double),
        ("sigma2_g_se", C.c_double), ("sigma2_e_se", C.c_double),
        ("log_likelihood", C.c_double), ("max_score", C.c_double), ("n_eig", C.c_int64),
        ("converged", C.c_int32), ("seconds", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class GrmBuilder:
    """GrmBuilder (libCosmicCore/src/grm_builder.h): the dense GRM over every sample of the
    genotypes, resident on the device (algorithm 1 VanRaden by default; 0/3 Yang, 2 Zeng,
    4 Vitezica, 5 TrueVar)."""

    def __init__(self, min_maf: float = 0.01, algorithm: int = 1):
        self.options = GrmOptions(float(min_maf), int(algorithm))
        self._h = None

    def compute(self, reader: Genotypes, variants=None):
        self.close()
        h = C.c_void_p()
        v = None if variants is None else np.ascontiguousarray(variants, dtype=np.int32)
        _check(_abi.lib().cs_grm_create(reader._h, _ptr(v), 0 if v is None else len(v),
                                        C.byref(self.options), C.byref(h)))
        self._h = h
        return self

    @classmethod
    def from_matrix(cls, G) -> "GrmBuilder":
        """A caller's own GRM (EigenVce::prepare accepts any symmetric G)."""
        G = np.asfortranarray(G, dtype=np.float64)
        b = cls()
        h = C.c_void_p()
        _check(_abi.lib().cs_grm_from_host(G.shape[0], _ptr(G), G.shape[0], C.byref(h)))
        b._h = h
        return b

    @classmethod
    def loco(cls, global_grm: "GrmBuilder", chrom_grm: "GrmBuilder") -> "GrmBuilder":
        """The LOCO GRM of src/gwas_scanner.cpp:476-491 from the global GRM and the GRM of
        one chromosome's SNPs (GrmBuilder::computeSplit's per-chromosome part)."""
        b = cls(algorithm=global_grm.options.algorithm)
        h = C.c_void_p()
        _check(_abi.lib().cs_grm_loco(global_grm._h, chrom_grm._h, C.byref(h)))
        b._h = h
        return b

    def _info(self):
        n, nv, s = C.c_int64(), C.c_int64(), C.c_double()
        _check(_abi.lib().cs_grm_info(self._h, C.byref(n), C.byref(nv), C.byref(s)))
        return n.value, nv.value, s.value

    def getNumSamples(self) -> int:
        return self._info()[0]

    def getTotalSnps(self) -> int:
        return self._info()[1]

    def getSum2pq(self) -> float:
        return self._info()[2]

    def getGrm(self, keep=None) -> np.ndarray:
        """G, or G[keep, keep] (DataFilter::subsetSquare), as a host array."""
        if keep is None:
            n = self.getNumSamples()
            out = np.zeros((n, n), order="F")
            _check(_abi.lib().cs_grm_copy(self._h, None, 0, _ptr(out), n))
            return out
        k = np.ascontiguousarray(keep, dtype=np.int32)
        out = np.zeros((len(k), len(k)), order="F")
        _check(_abi.lib().cs_grm_copy(self._h, _ptr(k), len(k), _ptr(out), len(k)))
        return out

    def close(self):
        if self._h:
            _abi.lib().cs_grm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EigenVce:
    """EigenVce (libCosmicCore/src/eigen_vce.h): prepare() = eigen_vce.cpp:19-63 on
    G[keep, keep] (covariate projection by default), runNullModel() = the Brent branch
    (eigen_vce.cpp:83-153, vce.cpp:3073-3175)."""

    def __init__(self, use_covariate_projection: bool = True):
        self.use_covariate_projection = bool(use_covariate_projection)
        self._h = None
        self.result = None

    def prepare(self, y, X, grm: GrmBuilder, keep=None):
        self.close()
        y = np.ascontiguousarray(y, dtype=np.float64)
        X = np.asfortranarray(np.asarray(X, dtype=np.float32).astype(np.float64))
        k = None if keep is None else np.ascontiguousarray(keep, dtype=np.int32)
        h = C.c_void_p()
        _check(_abi.lib().cs_eigen_vce_prepare(grm._h, _ptr(k), 0 if k is None else len(k),
                                               _ptr(y), _ptr(X), X.shape[1],
                                               int(self.use_covariate_projection), C.byref(h)))
        self._h = h
        n, ne, p = C.c_int64(), C.c_int64(), C.c_int64()
        _check(_abi.lib().cs_eigen_vce_dims(h, C.byref(n), C.byref(ne), C.byref(p)))
        self.n, self.n_eig, self.p = n.value, ne.value, p.value
        return self

    def runNullModel(self) -> dict:
        r = EigenVceResult()
        _check(_abi.lib().cs_eigen_vce_run_null(self._h, C.byref(r)))
        self.result = r.as_dict()
        return self.result

    def getSigma2g(self):
        return self.result["sigma2_g"]

    def getSigma2e(self):
        return self.result["sigma2_e"]

    def getDelta(self):
        return self.result["delta"]

    def _get(self, which):
        D, Uty = np.zeros(self.n_eig), np.zeros(self.n_eig)
        UtX = np.zeros((self.n_eig, self.p), order="F")
        W = np.zeros((self.n, self.n_eig), order="F") if which == "W" else None
        _check(_abi.lib().cs_eigen_vce_get(self._h, _ptr(D), _ptr(Uty), _ptr(UtX), _ptr(W),
                                           self.n))
        return {"D": D, "Uty": Uty, "UtX": UtX, "W": W}[which]

    def getEigenvalues(self) -> np.ndarray:
        return self._get("D")

    def getUty(self) -> np.ndarray:
        return self._get("Uty")

    def getUtX(self) -> np.ndarray:
        return self._get("UtX")

    def getProjectedW(self) -> np.ndarray:
        return self._get("W")

    def close(self):
        if self._h:
            _abi.lib().cs_eigen_vce_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- PCG and AI-REML

def pcg_solve_device(op: KinshipOperator, B_ptr: int, ldb: int, k: int, X_ptr: int, ldx: int,
                     sigma2_g: float, sigma2_e: float, tol: float = 1e-10, max_iter: int = 2000,
                     relative: bool = False, precision="fp64", kinship_divisor: float = 0.0,
                     stream: int = 0) -> np.ndarray:
    """MatrixFreePCG::solve (libCosmicCore/src/matrix_free_pcg.h:20-68) for k right-hand sides
    of (sigma2_g K + sigma2_e I) X = B on device column-major buffers; returns iterations."""
    it = np.zeros(max(k, 1), dtype=np.int32)
    _check(_abi.lib().cs_pcg_solve(op._h, float(kinship_divisor), float(sigma2_g), float(sigma2_e),
                                   C.c_void_p(B_ptr), ldb, k, C.c_void_p(X_ptr), ldx, float(tol),
                                   int(relative), int(max_iter), _prec(precision), _ptr(it),
                                   C.c_void_p(stream)))
    return it[:k]


def pcg_solve_records_device(op: KinshipOperator, rec_to_row, n_records: int, B_ptr: int,
                            ldb: int, k: int, X_ptr: int, ldx: int, sigma2_g: float,
                            sigma2_e: float, sigma2_pe: float = 0.0, with_pe: bool = False,
                            tol: float = 1e-10, max_iter: int = 2000, relative: bool = False,
                            precision="fp64", kinship_divisor: float = 0.0,
                            stream: int = 0) -> np.ndarray:
    """MatrixFreePCG::solve with STCG_VCE's record-level covariance (stcg_vce.cpp:80-126):
    V = sigma2_g Zr K Zr^T + sigma2_pe Zr Zr^T + sigma2_e I; returns iterations per column."""
    rmap = None if rec_to_row is None else np.ascontiguousarray(rec_to_row, dtype=np.int32)
    it = np.zeros(max(k, 1), dtype=np.int32)
    _check(_abi.lib().cs_pcg_solve_records(
        op._h, float(kinship_divisor), _ptr(rmap), int(n_records), int(bool(with_pe)),
        float(sigma2_g), float(sigma2_pe), float(sigma2_e), C.c_void_p(B_ptr), ldb, k,
        C.c_void_p(X_ptr), ldx, float(tol), int(relative), int(max_iter), _prec(precision),
        _ptr(it), C.c_void_p(stream)))
    return it[:k]


class MatrixFreePCG:
    """Host-array convenience over :func:`pcg_solve_device` (device memory through torch).
    With ``rec_to_row`` (and optionally ``with_pe`` / ``sigma2_pe``) the system is STCG_VCE's
    record-level covariance."""

    def __init__(self, op: KinshipOperator, sigma2_g: float, sigma2_e: float, precision="fp64",
                 kinship_divisor: float = 0.0, rec_to_row=None, with_pe: bool = False,
                 sigma2_pe: float = 0.0):
        self.op, self.sg2, self.se2 = op, sigma2_g, sigma2_e
        self.precision, self.divisor = precision, kinship_divisor
        self.rec_to_row, self.with_pe, self.spe2 = rec_to_row, with_pe, sigma2_pe
        self.iterations = None

    def solve(self, b, tol: float = 1e-8, max_iter: int = 1000, relative: bool = False):
        import torch

        b = np.asarray(b, dtype=np.float64)
        vec = b.ndim == 1
        B = b.reshape(len(b), -1) if vec else b
        n, k = B.shape
        dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()  # column-major n x k
        dX = torch.zeros_like(dB)
        stream = torch.cuda.current_stream().cuda_stream
        if self.rec_to_row is None and not self.with_pe:
            self.iterations = pcg_solve_device(self.op, dB.data_ptr(), n, k, dX.data_ptr(), n,
                                               self.sg2, self.se2, tol, max_iter, relative,
                                               self.precision, self.divisor, stream)
        else:
            self.iterations = pcg_solve_records_device(
                self.op, self.rec_to_row, n, dB.data_ptr(), n, k, dX.data_ptr(), n, self.sg2,
                self.se2, self.spe2, self.with_pe, tol, max_iter, relative, self.precision,
                self.divisor, stream)
        torch.cuda.current_stream().synchronize()
        x = dX.cpu().numpy().T
        return x[:, 0].copy() if vec else np.asfortranarray(x)


class MvStcgOptions(C.Structure):
    _fields_ = [
        ("max_iter", C.c_int32), ("tol", C.c_double), ("mc_samples", C.c_int32),
        ("pcg_tol", C.c_double), ("pcg_relative", C.c_int32), ("pcg_max_iter", C.c_int32),
        ("probe_seed", C.c_uint64), ("precision", C.c_int32),
    ]


class MvStcgResult(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("converged", C.c_int32), ("pcg_iterations", C.c_int64),
        ("operator_applies", C.c_int64), ("operator_columns", C.c_int64), ("seconds", C.c_double),
    ]


def mv_stcg_solve(op: "KinshipOperator", Y, X, kinship_divisor: float = 0.0, **options):
    """The multi-trait matrix-free REML (cs_mv_stcg_solve): MvEigenVce's EM for
    Vg (x) K + Ve (x) I from kinship applies, CG and Hutchinson probes.  Y (n, d), X (n, p).
    Returns (Vg, Ve, result dict)."""
    Y = np.asfortranarray(np.asarray(Y, dtype=np.float64).reshape(op.rows(), -1))
    X = np.asfortranarray(np.asarray(X, dtype=np.float64).reshape(op.rows(), -1))
    d = Y.shape[1]
    o = MvStcgOptions()
    _abi.lib().cs_mv_stcg_default_options(C.byref(o))
    for k, v in options.items():
        setattr(o, k, _prec(v) if k == "precision" else v)
    Vg = np.zeros((d, d), order="F")
    Ve = np.zeros((d, d), order="F")
    r = MvStcgResult()
    _check(_abi.lib().cs_mv_stcg_solve(op._h, float(kinship_divisor), _ptr(Y), d, _ptr(X),
                                       X.shape[1], C.byref(o), _ptr(Vg), _ptr(Ve), C.byref(r)))
    return Vg, Ve, {f[0]: getattr(r, f[0]) for f in r._fields_}


class VceOptions(C.Structure):
    _fields_ = [
        ("max_iter", C.c_int32), ("tol", C.c_double), ("mc_samples", C.c_int32),
        ("pcg_tol", C.c_double), ("pcg_relative", C.c_int32), ("pcg_max_iter", C.c_int32),
        ("slq_probes", C.c_int32), ("slq_steps", C.c_int32), ("probe_seed", C.c_uint64),
        ("precision", C.c_int32), ("precond_rank", C.c_int32),
    ]


class VceResult(C.Structure):
    _fields_ = [
        ("sigma2_g", C.c_double), ("sigma2_pe", C.c_double), ("sigma2_e", C.c_double),
        ("logl", C.c_double), ("iterations", C.c_int32), ("converged", C.c_int32),
        ("pcg_iterations", C.c_int64), ("operator_applies", C.c_int64),
        ("operator_columns", C.c_int64), ("seconds", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class StcgVce:
    """STCG_VCE (libCosmicCore/src/stcg_vce.h:7-54): matrix-free AI-REML with PCG solves and
    Hutchinson trace probes.  ``rec_to_row=None`` is the single-record LMM (records are the
    operator's rows); ``with_pe`` adds the permanent-environment component."""

    def __init__(self):
        h = C.c_void_p()
        _check(_abi.lib().cs_vce_create(C.byref(h)))
        self._h = h
        self.result = None
        self._rows = 0
        self._p = 0

    @staticmethod
    def default_options(**overrides) -> VceOptions:
        o = VceOptions()
        _abi.lib().cs_vce_default_options(C.byref(o))
        for k, v in overrides.items():
            if k == "precision":
                v = _prec(v)
            setattr(o, k, v)
        return o

    def solve(self, op: KinshipOperator, y, X, rec_to_row=None, with_pe=False,
              kinship_divisor: float = 0.0, **options) -> dict:
        y = np.ascontiguousarray(y, dtype=np.float64)
        X = np.asfortranarray(np.asarray(X, dtype=np.float64).reshape(len(y), -1))
        rmap = None if rec_to_row is None else np.ascontiguousarray(rec_to_row, dtype=np.int32)
        opt = self.default_options(**options)
        res = VceResult()
        _check(_abi.lib().cs_vce_solve_stcg(self._h, op._h, float(kinship_divisor), _ptr(rmap),
                                            len(y), int(bool(with_pe)), _ptr(y), _ptr(X),
                                            X.shape[1], C.byref(opt), C.byref(res)))
        self.result = res.as_dict()
        self._rows = op.rows()
        self._p = X.shape[1]
        return self.result

    def getVarE(self):
        return self.result["sigma2_e"]

    def getVarsU(self):
        return [self.result["sigma2_g"], self.result["sigma2_pe"]]

    def solution(self):
        beta = np.zeros(self._p)
        a = np.zeros(self._rows)
        pe = np.zeros(self._rows)
        _check(_abi.lib().cs_vce_solution(self._h, _ptr(beta), _ptr(a), _ptr(pe)))
        return beta, a, pe

    def history(self) -> np.ndarray:
        it = C.c_int64()
        _check(_abi.lib().cs_vce_history(self._h, None, C.byref(it)))
        out = np.zeros(5 * max(it.value, 1))
        _check(_abi.lib().cs_vce_history(self._h, _ptr(out), C.byref(it)))
        return out[:5 * it.value].reshape(-1, 5)

    def close(self):
        if self._h:
            _abi.lib().cs_vce_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


ASSOC_LAYOUTS = {"unified": 0, "stcg": 1, "ssf": 2}


def _result_arrays(results):
    arr = {k: np.ascontiguousarray(results[k], dtype=np.float64)
           for k in ("freq", "beta", "se", "p", "log10p")}
    tested = results.get("tested")
    tested = None if tested is None else np.ascontiguousarray(tested, dtype=np.int32)
    return arr, tested


def write_assoc_txt(path: str, bim_path: str, results: dict, n_obs: int, stcg_columns=False,
                    layout: str = None, gzip: bool = False, order=None):
    """Writes `.assoc.txt` (src/gwas_output.cpp:123-183) from a scan result dict.  layout
    "stcg" (or stcg_columns) gives `.stcg.assoc.txt`, "ssf" the `--out-ssf` GWAS-SSF rows;
    gzip the `--out-gz` form; order the SNP indices in row order (default .bim order)."""
    m = len(results["p"])
    arr, tested = _result_arrays(results)
    if layout is None:
        layout = "stcg" if stcg_columns else "unified"
    if layout not in ASSOC_LAYOUTS:
        raise InvalidArgument(_abi.CS_ERR_INVALID_ARGUMENT, f"unknown layout {layout!r}")
    if order is not None:
        order = np.ascontiguousarray(order, dtype=np.int64)
    _check(_abi.lib().cs_write_assoc(path.encode(), bim_path.encode(), m, int(n_obs),
                                     _ptr(arr["freq"]), _ptr(arr["beta"]), _ptr(arr["se"]),
                                     _ptr(arr["p"]), _ptr(arr["log10p"]), _ptr(tested),
                                     _ptr(order), 0 if order is None else len(order),
                                     ASSOC_LAYOUTS[layout], int(bool(gzip))))


def append_cosmic_sumstats(path: str, bim_path: str, results: dict, n_obs: int,
                           model: str = "LMM", append: bool = False, gzip: bool = False,
                           created: str = None):
    """`OUT.cosmic.sumstats` (GwasScanner::appendCosmicSumstats, src/gwas_output.cpp:186-234):
    append=False replaces the file and writes the header (created: the "# Created:" text,
    default the current UTC time), append=True adds the rows of another chromosome."""
    m = len(results["p"])
    arr, tested = _result_arrays(results)
    _check(_abi.lib().cs_append_cosmic_sumstats(
        path.encode(), bim_path.encode(), m, int(n_obs), _ptr(arr["freq"]), _ptr(arr["beta"]),
        _ptr(arr["se"]), _ptr(arr["p"]), _ptr(arr["log10p"]), _ptr(tested), model.encode(),
        int(bool(append)), int(bool(gzip)), None if created is None else created.encode()))


# ---------------------------------------------------------------- serving loop

class ServerOptions(C.Structure):
    _fields_ = [
        ("rank", C.c_int32), ("oversample", C.c_int32), ("trace_threshold", C.c_double),
        ("min_rank", C.c_int32), ("min_maf", C.c_double), ("precision", C.c_int32),
        ("max_batch_columns", C.c_int64), ("memory_budget_gb", C.c_double),
        ("max_active", C.c_int32), ("batch_window_ms", C.c_double),
        ("subset_fraction", C.c_double),
    ]


class ServeRequest(C.Structure):
    _fields_ = [
        ("samples", C.c_void_p), ("n_samples", C.c_int64), ("Y", C.c_void_p),
        ("n_traits", C.c_int32), ("X", C.c_void_p), ("p", C.c_int32),
        ("snp_begin", C.c_int64), ("snp_end", C.c_int64), ("seed", C.c_uint64),
    ]


class ServeStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("latency_s", C.c_double), ("queue_s", C.c_double),
                ("effective_rank", C.c_int32)]


class ServerStatistics(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
        ("p50_s", C.c_double), ("p99_s", C.c_double), ("mean_s", C.c_double),
        ("throughput_rps", C.c_double), ("wall_s", C.c_double), ("applies", C.c_int64),
        ("apply_columns", C.c_int64), ("max_requests_per_apply", C.c_int64),
        ("max_concurrent", C.c_int64), ("own_view_requests", C.c_int64),
        ("memory_budget_gb", C.c_double),
    ]


class Server:
    """Resident-genotype association server with continuous batching of kinship applies
    across requests (no reference counterpart; each request is the matrix-free LMM job of
    src/gwas_scanner.cpp on a cohort subset and a SNP window)."""

    def __init__(self, genotypes: Genotypes, variants=None, **options):
        o = ServerOptions()
        _abi.lib().cs_server_default_options(C.byref(o))
        for k, v in options.items():
            setattr(o, k, _prec(v) if k == "precision" else v)
        self._g = genotypes
        var = None if variants is None else np.ascontiguousarray(variants, dtype=np.int32)
        h = C.c_void_p()
        _check(_abi.lib().cs_server_create(genotypes._h, _ptr(var),
                                           0 if var is None else len(var), C.byref(o),
                                           C.byref(h)))
        self._h = h
        self._windows = {}

    def submit(self, samples, Y, X, snp_begin=0, snp_end=None, seed=42) -> int:
        samples = np.ascontiguousarray(samples, dtype=np.int32)
        Y = np.asfortranarray(np.asarray(Y, dtype=np.float64).reshape(len(samples), -1))
        X = np.asfortranarray(np.asarray(X, dtype=np.float64).reshape(len(samples), -1))
        end = self._g.n_snps if snp_end is None else int(snp_end)
        q = ServeRequest(samples.ctypes.data, len(samples), Y.ctypes.data, Y.shape[1],
                         X.ctypes.data if X.shape[1] else None, X.shape[1], int(snp_begin), end,
                         int(seed))
        rid = C.c_int64()
        _check(_abi.lib().cs_server_submit(self._h, C.byref(q), C.byref(rid)))
        self._windows[rid.value] = (end - int(snp_begin), Y.shape[1])
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0) -> dict:
        st = ServeStatus()
        _check(_abi.lib().cs_server_wait(self._h, rid, float(timeout), C.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def result(self, rid: int, trait: int = 0) -> dict:
        w, _ = self._windows[rid]
        out = {k: np.zeros(w) for k in ("beta", "se", "p", "log10p", "freq")}
        tested = np.zeros(w, dtype=np.int32)
        s2 = np.zeros(2)
        _check(_abi.lib().cs_server_result(self._h, rid, trait, _ptr(s2), _ptr(out["beta"]),
                                           _ptr(out["se"]), _ptr(out["p"]), _ptr(out["log10p"]),
                                           _ptr(out["freq"]), _ptr(tested)))
        out["tested"] = tested.astype(bool)
        out["sigma2_g"], out["sigma2_e"] = float(s2[0]), float(s2[1])
        return out

    def release(self, rid: int):
        _check(_abi.lib().cs_server_release(self._h, rid))
        self._windows.pop(rid, None)

    def stats(self) -> dict:
        st = ServerStatistics()
        _check(_abi.lib().cs_server_stats(self._h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def close(self):
        if self._h:
            _abi.lib().cs_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def stcg_scan(genotypes: Genotypes, G, subject_rows, obs_to_subject, y, X, vg, vpe, ve,
              min_maf=0.01, snp_begin=0, snp_end=None) -> dict:
    """RepeatabilityModel::scanSTCG's scan with a given subject GRM
    (src/models/repeatability_scan_stcg.cpp:42-140) on the GPU; per-SNP dict for
    [snp_begin, snp_end): beta, se, p, log10p, maf (folded, the FREQ column), tested."""
    G = np.asfortranarray(G, dtype=np.float64)
    q = G.shape[0]
    subj = np.ascontiguousarray(subject_rows, dtype=np.int32)
    o2s = np.ascontiguousarray(obs_to_subject, dtype=np.int32)
    y = np.ascontiguousarray(y, dtype=np.float64)
    X = np.asfortranarray(np.asarray(X, dtype=np.float64).reshape(len(y), -1))
    end = genotypes.n_snps if snp_end is None else int(snp_end)
    w = end - int(snp_begin)
    out = {k: np.zeros(max(w, 0)) for k in ("beta", "se", "p", "log10p", "maf")}
    tested = np.zeros(max(w, 0), dtype=np.int32)
    _check(_abi.lib().cs_stcg_scan(genotypes._h, _ptr(G), q, _ptr(subj), _ptr(o2s), len(y),
                                   _ptr(y), _ptr(X), X.shape[1], float(vg), float(vpe), float(ve),
                                   float(min_maf), int(snp_begin), end, _ptr(out["beta"]),
                                   _ptr(out["se"]), _ptr(out["p"]), _ptr(out["log10p"]),
                                   _ptr(out["maf"]), _ptr(tested)))
    out["tested"] = tested.astype(bool)
    return out


def mvlmm_scan(genotypes: Genotypes, keep, W, D, Uty, UtX, Vg, Ve, snp_begin=0, snp_end=None,
               precision="fp64") -> dict:
    """MvLmmEngine::scan(PlinkReader) (src/mvlmm_engine.cpp:756-931) on the GPU with a given
    null (W: n x r eigenbasis, D: r, U'y: r x d, U'X: r x p, Vg, Ve: d x d).  Per SNP: beta
    (d), cov (d x d), wald, p, freq, status (0 OK, 1 roundoff, 2 boundary, 3 singular)."""
    keep = np.ascontiguousarray(keep, dtype=np.int32)
    W = np.asfortranarray(W, dtype=np.float64)
    n, r = W.shape
    D = np.ascontiguousarray(D, dtype=np.float64)
    Uty = np.asfortranarray(np.asarray(Uty, dtype=np.float64).reshape(r, -1))
    d = Uty.shape[1]
    UtX = np.asfortranarray(np.asarray(UtX, dtype=np.float64).reshape(r, -1))
    Vg = np.asfortranarray(Vg, dtype=np.float64)
    Ve = np.asfortranarray(Ve, dtype=np.float64)
    end = genotypes.n_snps if snp_end is None else int(snp_end)
    m = end - int(snp_begin)
    beta = np.zeros((m, d))
    cov = np.zeros((m, d, d))
    wald, pv, fr = np.zeros(m), np.zeros(m), np.zeros(m)
    st = np.zeros(m, dtype=np.int32)
    _check(_abi.lib().cs_mvlmm_scan(genotypes._h, _ptr(keep), n, _ptr(W), r, _ptr(D), _ptr(Uty), d,
                                    _ptr(UtX), UtX.shape[1], _ptr(Vg), _ptr(Ve), int(snp_begin), end,
                                    _prec(precision), _ptr(beta), _ptr(cov), _ptr(wald), _ptr(pv),
                                    _ptr(fr), _ptr(st)))
    return {"beta": beta, "cov": cov, "wald": wald, "p": pv, "freq": fr, "status": st}


class MvVceOptions(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("tol", C.c_double), ("aireml", C.c_int32),
                ("em_min_iter", C.c_int32), ("ai_max_iter", C.c_int32), ("ai_tol", C.c_double)]


class MvEigenVce:
    """MvEigenVce (libCosmicCore/src/eigen_vce.h): prepare() = eigen_vce.cpp:496-549 on
    G[keep, keep] (covariate projection by default), runNullModel() = EM or AI-REML
    (:551-911, 1031-1065) with the multivariate model's defaults (--reml-maxit 1000,
    --reml-tol 1e-8)."""

    def __init__(self, use_projection: bool = True, aireml: bool = False, **options):
        self.use_projection = bool(use_projection)
        self.options = MvVceOptions()
        _abi.lib().cs_mv_vce_default_options(C.byref(self.options))
        self.options.aireml = int(bool(aireml))
        for k, v in options.items():
            setattr(self.options, k, v)
        self._h = None

    def prepare(self, Y, X, grm: GrmBuilder, keep=None):
        self.close()
        Y = np.asfortranarray(np.asarray(Y, dtype=np.float64).reshape(len(Y), -1))
        X = np.asfortranarray(np.asarray(X, dtype=np.float64).reshape(len(Y), -1))
        k = None if keep is None else np.ascontiguousarray(keep, dtype=np.int32)
        h = C.c_void_p()
        _check(_abi.lib().cs_mv_eigen_vce_prepare(grm._h, _ptr(k), 0 if k is None else len(k),
                                                  _ptr(Y), Y.shape[1], _ptr(X), X.shape[1],
                                                  int(self.use_projection), C.byref(h)))
        self._h = h
        n, ne, d = C.c_int64(), C.c_int64(), C.c_int64()
        _check(_abi.lib().cs_mv_eigen_vce_dims(h, C.byref(n), C.byref(ne), C.byref(d)))
        self.n, self.n_eig, self.d = n.value, ne.value, d.value
        return self

    def runNullModel(self) -> bool:
        conv, it, logl = C.c_int32(), C.c_int32(), C.c_double()
        _check(_abi.lib().cs_mv_eigen_vce_run_null(self._h, C.byref(self.options), C.byref(conv),
                                                   C.byref(it), C.byref(logl)))
        self.converged, self.iterations, self.logl = bool(conv.value), it.value, logl.value
        return self.converged

    def _get(self):
        d = self.d
        out = {k: np.zeros((d, d), order="F") for k in ("Vg", "Ve", "Vg_se", "Ve_se")}
        out["D"] = np.zeros(self.n_eig)
        out["Uty"] = np.zeros((self.n_eig, d), order="F")
        _check(_abi.lib().cs_mv_eigen_vce_get(self._h, _ptr(out["Vg"]), _ptr(out["Ve"]),
                                              _ptr(out["Vg_se"]), _ptr(out["Ve_se"]),
                                              _ptr(out["D"]), _ptr(out["Uty"])))
        return out

    def getVg(self):
        return self._get()["Vg"]

    def getVe(self):
        return self._get()["Ve"]

    def getVgSE(self):
        return self._get()["Vg_se"]

    def getVeSE(self):
        return self._get()["Ve_se"]

    def getEigenvalues(self):
        return self._get()["D"]

    def getUty(self):
        return self._get()["Uty"]

    def scan(self, genotypes: Genotypes, keep, snp_begin=0, snp_end=None, precision="fp64"):
        """MvLmmEngine::prepareFromVce + scan (src/mvlmm_engine.cpp:195-207, 756-931) with the
        device eigenbasis; the outputs of mvlmm_scan()."""
        keep = np.ascontiguousarray(keep, dtype=np.int32)
        end = genotypes.n_snps if snp_end is None else int(snp_end)
        m, d = end - int(snp_begin), self.d
        beta, cov = np.zeros((m, d)), np.zeros((m, d, d))
        wald, pv, fr = np.zeros(m), np.zeros(m), np.zeros(m)
        st = np.zeros(m, dtype=np.int32)
        _check(_abi.lib().cs_mvlmm_scan_vce(genotypes._h, _ptr(keep), len(keep), self._h,
                                            int(snp_begin), end, _prec(precision), _ptr(beta),
                                            _ptr(cov), _ptr(wald), _ptr(pv), _ptr(fr), _ptr(st)))
        return {"beta": beta, "cov": cov, "wald": wald, "p": pv, "freq": fr, "status": st}

    def close(self):
        if self._h:
            _abi.lib().cs_mv_eigen_vce_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_assoc_mv_txt(path: str, bim_path: str, results: dict):
    """Writes `.assoc.mv.txt` (src/models/multivariate_output.cpp:40-70) from mvlmm_scan()."""
    m, d = results["beta"].shape
    arr = {k: np.ascontiguousarray(results[k], dtype=np.float64) for k in ("freq", "wald", "p", "beta", "cov")}
    _check(_abi.lib().cs_write_assoc_mv_txt(path.encode(), bim_path.encode(), m, d,
                                            _ptr(arr["freq"]), _ptr(arr["wald"]), _ptr(arr["p"]),
                                            _ptr(arr["beta"]), _ptr(arr["cov"])))


class Samples:
    """The .fam sample list (PlinkReader::readFam, libCosmicCore/src/plink_reader.cpp:34-48):
    FID / IID keys in file order and the .fam phenotype column."""

    def __init__(self, fam_path: str):
        self._h = C.c_void_p()
        _check(_abi.lib().cs_fam_read(fam_path.encode(), C.byref(self._h)))
        n = C.c_int64()
        _check(_abi.lib().cs_samples_count(self._h, C.byref(n)))
        self.n = n.value

    def __len__(self):
        return self.n

    def ids(self):
        fid, iid = C.create_string_buffer(4096), C.create_string_buffer(4096)
        out = []
        for i in range(self.n):
            _check(_abi.lib().cs_samples_id(self._h, i, fid, 4096, iid, 4096))
            out.append((fid.value.decode(), iid.value.decode()))
        return out

    def fam_phenotype(self) -> np.ndarray:
        y = np.empty(self.n)
        _check(_abi.lib().cs_samples_fam_phenotype(self._h, _ptr(y)))
        return y

    def close(self):
        if getattr(self, "_h", None):
            _abi.lib().cs_samples_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PhenoReader:
    """PhenoReader (libCosmicCore/src/pheno_reader.cpp): load(path, col_idx) / align(samples)
    for one trait, loadMatrix(path, cols) / alignMatrix(samples) for several."""

    def __init__(self):
        self._h = None

    def _reset(self):
        if self._h:
            _abi.lib().cs_pheno_destroy(self._h)
        self._h = C.c_void_p()

    def load(self, path: str, col_idx: int = 1, missing_val: float = -9.0):
        self._reset()
        _check(_abi.lib().cs_pheno_load(path.encode(), int(col_idx), float(missing_val),
                                        C.byref(self._h)))

    def loadMatrix(self, path: str, cols=(), missing_val: float = -9.0):
        self._reset()
        c = np.ascontiguousarray(cols, dtype=np.int32)
        _check(_abi.lib().cs_pheno_load_matrix(path.encode(), _ptr(c) if len(c) else None,
                                               len(c), float(missing_val), C.byref(self._h)))

    def num_traits(self) -> int:
        t = C.c_int32()
        _check(_abi.lib().cs_pheno_traits(self._h, C.byref(t)))
        return t.value

    def align(self, samples: Samples):
        """y in .fam order (NaN where unmatched or missing) and the matched count."""
        y = np.empty(samples.n)
        m = C.c_int64()
        _check(_abi.lib().cs_pheno_align(self._h, samples._h, _ptr(y), C.byref(m)))
        return y, m.value

    def alignMatrix(self, samples: Samples):
        t = self.num_traits()
        Y = np.empty((t, samples.n))  # column-major n x t
        m = C.c_int64()
        _check(_abi.lib().cs_pheno_align_matrix(self._h, samples._h, _ptr(Y), samples.n, C.byref(m)))
        return Y.T.copy(), m.value

    def __del__(self):
        try:
            if self._h:
                _abi.lib().cs_pheno_destroy(self._h)
        except Exception:
            pass


class CovarReader:
    """CovarReader (libCosmicCore/src/covar_reader.cpp): load (quantitative, float) or
    loadCategorical (k levels -> k - 1 dummies), then align(samples) -> float32 n x p."""

    def __init__(self):
        self._h = None

    def _reset(self):
        if self._h:
            _abi.lib().cs_covar_destroy(self._h)
        self._h = C.c_void_p()

    def load(self, path: str, missing_val: float = -9.0):
        self._reset()
        _check(_abi.lib().cs_covar_load(path.encode(), float(missing_val), C.byref(self._h)))

    def loadCategorical(self, path: str, missing_val: str = "-9"):
        self._reset()
        _check(_abi.lib().cs_covar_load_categorical(path.encode(), missing_val.encode(),
                                                    C.byref(self._h)))

    def num_covars(self) -> int:
        p = C.c_int32()
        _check(_abi.lib().cs_covar_columns(self._h, C.byref(p)))
        return p.value

    def align(self, samples: Samples):
        p = self.num_covars()
        X = np.empty((p, samples.n), dtype=np.float32)  # column-major n x p
        m = C.c_int64()
        _check(_abi.lib().cs_covar_align(self._h, samples._h, _ptr(X) if p else None, samples.n,
                                         C.byref(m)))
        return X.T.copy(), m.value

    def __del__(self):
        try:
            if self._h:
                _abi.lib().cs_covar_destroy(self._h)
        except Exception:
            pass


class DataFilter:
    """DataFilter::filterSamples (libCosmicCore/src/data_filter.h:21-41)."""

    @staticmethod
    def filterSamples(y, X) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        X = np.asarray(X, dtype=np.float32)
        if X.ndim != 2 or X.shape[0] != y.shape[0]:
            raise InvalidArgument(-1, "DataFilter: X and y dimension mismatch")
        Xc = np.asfortranarray(X)
        keep = np.empty(len(y), dtype=np.int32)
        nk = C.c_int64()
        _check(_abi.lib().cs_filter_samples(_ptr(y), len(y), _ptr(Xc) if X.shape[1] else None,
                                            len(y), X.shape[1], _ptr(keep), C.byref(nk)))
        return keep[:nk.value].copy()


def load_association_inputs(bfile: str, pheno: str = None, mpheno: int = 1, qcovar: str = None,
                            covar: str = None, missing_val: float = -9.0) -> dict:
    """What the reference's standard LMM prepares before the engines run
    (UnivariateModel::prepare, src/models/univariate_model.cpp:389-426, with
    DataLoader::loadPhenotype / loadCovariates, src/data_loader.h:219-285): y from the
    phenotype file (or the .fam column), X = [1 | quantitative | categorical dummies] as
    float, the keep list of complete samples, and y / X restricted to it (X as float64
    holding the float32 values).  Fewer than 10 kept samples is an error, as there."""
    samples = Samples(bfile + ".fam")
    if pheno:
        pr = PhenoReader()
        pr.load(pheno, mpheno, missing_val)
        y, _ = pr.align(samples)
    else:
        y = samples.fam_phenotype()
    cols = [np.ones((samples.n, 1), dtype=np.float32)]
    if qcovar:
        cr = CovarReader()
        cr.load(qcovar, missing_val)
        cols.append(cr.align(samples)[0])
    if covar:
        cr = CovarReader()
        cr.loadCategorical(covar)
        cols.append(cr.align(samples)[0])
    X = np.concatenate(cols, axis=1)
    keep = DataFilter.filterSamples(y, X)
    if len(keep) < 10:
        raise CosmicError(-1, "Too few valid samples.")
    return {"samples": samples, "keep": keep, "y": y[keep].copy(),
            "X": X[keep].astype(np.float64), "y_all": y, "X_all": X}


def grm_variant_selection(stats: dict, min_maf: float = 0.01) -> np.ndarray:
    """Variants of the matrix-free GRM (src/gwas_scanner.cpp:258-277): 1/sd != 0 and
    MAF (from the all-sample mean) >= min_maf; extract/exclude lists are not modelled."""
    freq = stats["mean"] / 2.0
    maf = np.minimum(freq, 1.0 - freq)
    ok = (stats["inv_std"] != 0.0) & ~(maf < min_maf) & ~(np.abs(maf) < 1e-8)
    return np.nonzero(ok)[0].astype(np.int32)


def read_bim(path: str) -> dict:
    """A .bim file as PlinkReader::readBim parses it (libCosmicCore/src/plink_reader.cpp:52-65):
    chrom, id, cm, bp, A1 (column 5), A2 (column 6) per non-empty line."""
    cols = {k: [] for k in ("chrom", "id", "cm", "bp", "a1", "a2")}
    with open(path) as f:
        for line in f:
            if not line.strip():
                continue
            t = line.split()
            cols["chrom"].append(t[0])
            cols["id"].append(t[1])
            cols["cm"].append(float(t[2]))
            cols["bp"].append(int(t[3]))
            cols["a1"].append(t[4])
            cols["a2"].append(t[5])
    cols["chrom"] = np.asarray(cols["chrom"], dtype=object)
    cols["bp"] = np.asarray(cols["bp"], dtype=np.int64)
    return cols


def _stoi(text: str):
    """std::stoi: optional sign and leading digits after whitespace; None when it throws."""
    t = text.lstrip()
    i = 1 if t[:1] in "+-" else 0
    j = i
    while j < len(t) and t[j].isdigit():
        j += 1
    return int(t[:j]) if j > i else None


def sort_chrom_labels(labels) -> list:
    """The LOCO chromosome order of src/gwas_scanner.cpp:62-72: numeric labels compare as
    integers (std::stoi), anything else as strings, over the distinct labels."""
    import functools

    def before(a, b):
        ia, ib = _stoi(a), _stoi(b)
        if ia is not None and ib is not None:
            return -1 if ia < ib else (1 if ib < ia else 0)
        return -1 if a < b else (1 if b < a else 0)

    return sorted(set(str(x) for x in labels), key=functools.cmp_to_key(before))


class LmmRunOptions(C.Structure):
    _fields_ = [
        ("rank", C.c_int32), ("oversample", C.c_int32), ("seed", C.c_int64),
        ("trace_threshold", C.c_double), ("min_rank", C.c_int32), ("min_maf", C.c_double),
        ("precision", C.c_int32), ("loco", C.c_int32), ("no_fallback", C.c_int32),
        ("error_tol", C.c_double),
    ]


class LmmRunScope(C.Structure):
    _fields_ = [("label", C.c_char * 32), ("diag", LowRankDiagnostics), ("fallback", C.c_int32)]


_FALLBACKS = {0: "none", 1: "trace_threshold", 2: "error_tolerance"}


def _run_options(rank, oversample, seed, trace_threshold, min_rank, min_maf, precision, loco,
                 no_fallback, error_tol) -> LmmRunOptions:
    o = LmmRunOptions()
    _abi.lib().cs_lmm_run_default_options(C.byref(o))
    o.rank, o.oversample, o.seed = int(rank), int(oversample), int(seed)
    o.trace_threshold, o.min_rank, o.min_maf = float(trace_threshold), int(min_rank), float(min_maf)
    o.precision, o.loco, o.no_fallback = _prec(precision), int(bool(loco)), int(bool(no_fallback))
    o.error_tol = float(error_tol)
    return o


def run_lmm_matrix_free(bed, n_samples: int, n_snps: int, y, X, keep=None, rank=256,
                        oversample=10, seed=42, trace_threshold=0.95, min_rank=1,
                        min_maf=0.01, precision="fp64", genotypes: Genotypes | None = None,
                        chrom=None, loco=True, no_fallback=True, error_tol=1.0):
    """The `gwas --model lmm --fastlmm --fastlmm-matrix-free --fastlmm-no-fallback --no-loco`
    path (src/gwas_scanner.cpp:121-129, 254-346, 447) from host buffers: upload + stats, then
    the library's C++ job (cs_run_lmm_matrix_free): GRM variant selection, operator, low-rank
    REML null model, scan of every SNP.  With per-SNP chromosome labels spanning more than one
    chromosome (and loco=True) it runs the reference's default leave-one-chromosome-out loop
    (src/gwas_scanner.cpp:299-314, 464-472): per chromosome, an operator without that
    chromosome's GRM variants, its own null model, and the scan of that chromosome's SNPs.
    no_fallback=False lets a null whose sketch misses the trace threshold (or exceeds
    error_tol) fall back as the reference does.  Returns (results dict, diagnostics dict; per
    chromosome under LOCO), each diagnostics dict with its "fallback" label."""
    g = genotypes if genotypes is not None else Genotypes.from_bed_bytes(bed, n_samples, n_snps)
    try:
        m = g.n_snps
        y = np.ascontiguousarray(y, dtype=np.float64)
        X = np.asfortranarray(np.asarray(X, dtype=np.float32).astype(np.float64).reshape(len(y), -1))
        keep_arr = None if keep is None else np.ascontiguousarray(keep, dtype=np.int32)
        labels = None
        if chrom is not None:
            enc = [str(c).encode() for c in chrom]
            labels = (C.c_char_p * len(enc))(*enc)
        out = {k: np.zeros(m) for k in ("beta", "se", "p", "log10p", "freq")}
        tested = np.zeros(m, dtype=np.int32)
        scopes = (LmmRunScope * 128)()
        n_sc = C.c_int32()
        o = _run_options(rank, oversample, seed, trace_threshold, min_rank, min_maf, precision,
                         loco, no_fallback, error_tol)
        _check(_abi.lib().cs_run_lmm_matrix_free(
            g._h, _ptr(keep_arr), 0 if keep_arr is None else len(keep_arr), _ptr(y), _ptr(X),
            X.shape[1], labels, C.byref(o), _ptr(out["beta"]), _ptr(out["se"]), _ptr(out["p"]),
            _ptr(out["log10p"]), _ptr(out["freq"]), _ptr(tested), scopes, len(scopes),
            C.byref(n_sc)))
        out["tested"] = tested.astype(bool)
        diags = {}
        for i in range(min(n_sc.value, len(scopes))):
            sc = scopes[i]
            diags[sc.label.decode()] = dict(sc.diag.as_dict(), fallback=_FALLBACKS[sc.fallback])
        if list(diags) == ["GLOBAL"]:
            return out, diags["GLOBAL"]
        return out, diags
    finally:
        if genotypes is None:
            g.close()


class GwasLmmOptions(C.Structure):
    _fields_ = [
        ("bfile", C.c_char_p), ("out", C.c_char_p), ("pheno", C.c_char_p), ("mpheno", C.c_int32),
        ("qcovar", C.c_char_p), ("covar", C.c_char_p), ("missing_code", C.c_double),
        ("run", LmmRunOptions), ("out_gz", C.c_int32), ("out_ssf", C.c_int32),
        ("created", C.c_char_p),
    ]


def gwas_lmm_files(bfile: str, out: str, pheno: str = None, mpheno: int = 1, qcovar: str = None,
                   covar: str = None, rank=256, oversample=10, seed=42, trace_threshold=0.95,
                   min_rank=1, min_maf=0.01, precision="mixed", loco=True, out_gz=False,
                   out_ssf=False, created=None, no_fallback=True, error_tol=1.0):
    """The whole `gwas --model lmm --fastlmm --fastlmm-matrix-free` run from files to files in
    the library's C++ (cs_run_gwas_lmm): inputs, null model(s), scan and every result file.
    Returns (kept samples, null models)."""
    o = GwasLmmOptions()
    _abi.lib().cs_gwas_lmm_default_options(C.byref(o))
    enc = lambda v: None if v is None else str(v).encode()
    o.bfile, o.out, o.pheno, o.mpheno = enc(bfile), enc(out), enc(pheno), int(mpheno)
    o.qcovar, o.covar, o.created = enc(qcovar), enc(covar), enc(created)
    o.run = _run_options(rank, oversample, seed, trace_threshold, min_rank, min_maf, precision,
                         loco, no_fallback, error_tol)
    o.out_gz, o.out_ssf = int(bool(out_gz)), int(bool(out_ssf))
    nk, ns = C.c_int64(), C.c_int32()
    _check(_abi.lib().cs_run_gwas_lmm(C.byref(o), C.byref(nk), C.byref(ns)))
    return nk.value, ns.value


def _chromosome_runs(chrom, c):
    """The SNPs of chromosome c as contiguous [begin, end) runs of the .bim order."""
    idx = np.flatnonzero(chrom == c)
    breaks = np.flatnonzero(np.diff(idx) != 1)
    return zip(np.r_[idx[0], idx[breaks + 1]], np.r_[idx[breaks] + 1, idx[-1] + 1])


def run_lmm_exact(genotypes: Genotypes, y, X, keep=None, chrom=None, loco=True, min_maf=0.01,
                  grm_algorithm=1, use_covariate_projection=True, precision="mixed"):
    """The default `gwas --model lmm` route (src/gwas_scanner.cpp:131-215, 384-399, 458-499):
    the dense GRM over every sample (GrmBuilder, VanRaden by default), G[keep, keep], EigenVce
    (covariate projection, Brent null model), LmmEngine::prepareFromVce and the exact scan.
    With chromosome labels spanning more than one chromosome and loco=True, per chromosome
    the LOCO GRM G (S / S_loco) - raw_chr / S_loco, its own null model and the scan of that
    chromosome's SNPs, in the reference's chromosome order.  use_residuals follows the
    reference (GRM algorithm 0).  Returns (results dict, null-model dict; per chromosome
    under LOCO)."""
    g = genotypes
    keep_arr = np.arange(g.n_samples, dtype=np.int32) if keep is None else np.asarray(keep, np.int32)
    residuals = grm_algorithm == 0
    glob = GrmBuilder(min_maf, grm_algorithm).compute(g)

    def null_and_scan(grm, windows):
        v = EigenVce(use_covariate_projection).prepare(y, X, grm, keep_arr)
        r = v.runNullModel()
        eng = LmmEngine()
        eng.prepareFromVce(v, use_residuals=residuals)
        parts = [(b, e, eng.scan_window(g, keep_arr, int(b), int(e), min_maf=min_maf,
                                        precision=precision)) for b, e in windows]
        eng.close()
        v.close()
        return r, parts

    try:
        m = g.n_snps
        if chrom is not None and loco and len(set(str(c) for c in chrom)) > 1:
            chrom = np.asarray(chrom).astype(str)
            out = {k: np.full(m, np.nan) for k in ("beta", "se", "p", "log10p", "freq")}
            out["tested"] = np.zeros(m, dtype=bool)
            diags = {}
            for c in sort_chrom_labels(chrom):
                chr_grm = GrmBuilder(min_maf, grm_algorithm).compute(
                    g, np.flatnonzero(chrom == c).astype(np.int32))
                loco_grm = GrmBuilder.loco(glob, chr_grm)
                chr_grm.close()
                diags[c], parts = null_and_scan(loco_grm, _chromosome_runs(chrom, c))
                loco_grm.close()
                for b, e, r in parts:
                    for k in ("beta", "se", "p", "log10p", "freq", "tested"):
                        out[k][b:e] = r[k]
            return out, diags
        diag, parts = null_and_scan(glob, [(0, m)])
        return parts[0][2], diag
    finally:
        glob.close()


def write_scan_meta(out_prefix: str, requested_rank: int = 256, trace_threshold: float = 0.95,
                    full_eigen: bool = False):
    """OUT.scan.meta.txt (src/gwas_scanner.cpp:93-108) of the matrix-free low-rank LMM, or of
    the dense route with full_eigen."""
    if full_eigen:
        _check(_abi.lib().cs_write_scan_meta_full_eigen(out_prefix.encode()))
        return
    _check(_abi.lib().cs_write_scan_meta(out_prefix.encode(), int(requested_rank),
                                         float(trace_threshold)))


def append_scan_common_meta(out_prefix: str, n: int, loco: bool, covariate_projection=True,
                            vce_converged=True, model: str = "additive"):
    """The lines appended to OUT.scan.meta.txt after the scan (src/gwas_output_schema.h:57-73,
    src/gwas_scanner.cpp:507-509)."""
    _check(_abi.lib().cs_append_scan_common_meta(out_prefix.encode(), model.encode(), int(n),
                                                 int(bool(loco)), int(bool(covariate_projection)),
                                                 int(bool(vce_converged))))


def write_low_rank_meta(out_prefix: str, rows, n: int, error_tol: float = 1.0,
                        fallback: str = "none"):
    """OUT.low_rank.meta.tsv (src/gwas_scanner.cpp:109-115, 409-428): rows = [(scope,
    diagnostics dict from prepareLowRankMatrixFree)], scope "GLOBAL" or the chromosome; the
    FALLBACK column is the dict's "fallback" entry when present, else `fallback`."""
    rows = list(rows)
    diags = (LowRankDiagnostics * max(1, len(rows)))()
    scopes = (C.c_char_p * max(1, len(rows)))()
    labels = (C.c_char_p * max(1, len(rows)))()
    for i, (scope, dd) in enumerate(rows):
        for name, _ in LowRankDiagnostics._fields_:
            setattr(diags[i], name, dd[name])
        scopes[i] = str(scope).encode()
        labels[i] = str(dd.get("fallback", fallback)).encode()
    _check(_abi.lib().cs_write_low_rank_meta(out_prefix.encode(), len(rows), scopes, diags,
                                             int(n), float(error_tol), labels))


def run_gwas_lmm(bfile: str, out: str, pheno: str = None, mpheno: int = 1, qcovar: str = None,
                 covar: str = None, rank=256, oversample=10, seed=42, trace_threshold=0.95,
                 min_rank=1, min_maf=0.01, precision="mixed", loco=True, out_gz=False,
                 out_ssf=False, created=None, exact=False, no_fallback=True, error_tol=1.0):
    """`cosmicscanner gwas --model lmm --fastlmm --fastlmm-matrix-free --fastlmm-no-fallback
    --bfile BFILE --pheno PHENO --mpheno N [--qcovar Q] [--covar C] --out OUT` end to end:
    the samples, phenotype, covariates and keep list as the reference prepares them
    (load_association_inputs), the .bed resident on the device, the low-rank matrix-free
    null model and scan (leave-one-chromosome-out when the .bim has more than one chromosome
    and loco is set, as the reference's default), OUT.assoc.txt (N = kept samples; rows
    chromosome by chromosome under LOCO; GWAS-SSF rows with out_ssf, gzip with out_gz),
    OUT.cosmic.sumstats (one append per chromosome under LOCO; created fixes its "# Created:"
    line) and the run metadata OUT.scan.meta.txt / OUT.low_rank.meta.tsv.  exact=True takes
    the default dense route instead (`--model lmm` without --fastlmm: run_lmm_exact; no
    .low_rank.meta.tsv).  Returns (results, diagnostics, inputs)."""
    inputs = load_association_inputs(bfile, pheno=pheno, mpheno=mpheno, qcovar=qcovar, covar=covar)
    g = Genotypes.open_plink(bfile)
    try:
        if g.n_samples != len(inputs["samples"]):
            raise InvalidArgument(_abi.CS_ERR_INVALID_ARGUMENT,
                                  ".fam and .bed sample counts differ")
        bim = read_bim(bfile + ".bim")
        if exact:
            res, diag = run_lmm_exact(g, inputs["y"], inputs["X"], keep=inputs["keep"],
                                      chrom=bim["chrom"] if loco else None, loco=loco,
                                      min_maf=min_maf, precision=precision)
        else:
            res, diag = run_lmm_matrix_free(None, g.n_samples, g.n_snps, inputs["y"], inputs["X"],
                                            keep=inputs["keep"], rank=rank, oversample=oversample,
                                            seed=seed, trace_threshold=trace_threshold,
                                            min_rank=min_rank, min_maf=min_maf,
                                            precision=precision, genotypes=g,
                                            chrom=bim["chrom"] if loco else None, loco=loco,
                                            no_fallback=no_fallback, error_tol=error_tol)
        n_keep = len(inputs["keep"])
        write_scan_meta(out, rank, trace_threshold, full_eigen=exact)
        if not exact:
            scoped = list(diag.items()) if "sigma2_g" not in diag else [("GLOBAL", diag)]
            write_low_rank_meta(out, scoped, n=n_keep, error_tol=error_tol)
        chrom = np.asarray(bim["chrom"]).astype(str)
        used_loco = "sigma2_g" not in diag
        groups = ([np.flatnonzero(chrom == c) for c in sort_chrom_labels(chrom)] if used_loco
                  else [np.arange(g.n_snps)])
        for i, idx in enumerate(groups):
            part = dict(res)
            mask = np.zeros(g.n_snps, dtype=np.int32)
            mask[idx] = np.asarray(res["tested"])[idx]
            part["tested"] = mask
            append_cosmic_sumstats(out + ".cosmic.sumstats", bfile + ".bim", part, n_keep,
                                   append=i > 0, gzip=out_gz, created=created)
        write_assoc_txt(out + ".assoc.txt", bfile + ".bim", res, n_obs=n_keep,
                        layout="ssf" if out_ssf else "unified", gzip=out_gz,
                        order=np.concatenate(groups))
        append_scan_common_meta(out, n_keep, loco=used_loco)
    finally:
        g.close()
    return res, diag, inputs


