"""ctypes declarations of the C ABI in include/cosmicscanner_b200.h."""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcosmicscanner_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "cosmicscanner_b200.h")

CS_OK = 0
CS_ERR_INVALID_ARGUMENT = -1
CS_ERR_CUDA = -2
CS_ERR_IO = -3
CS_ERR_FORMAT = -4
CS_ERR_NUMERIC = -5
CS_ERR_NOT_CONVERGED = -6
CS_ERR_UNSUPPORTED = -7

_P = C.c_void_p
_I64 = C.c_int64
_D = C.c_double
_I = C.c_int

_SIGNATURES = {
    "cs_last_error": ([], C.c_char_p),
    "cs_version": ([], C.c_char_p),
    "cs_genotypes_create": ([_P, C.c_size_t, _I64, _I64, _P], _I),
    "cs_genotypes_open_plink": ([C.c_char_p, _P], _I),
    "cs_genotypes_info": ([_P, _P, _P, _P], _I),
    "cs_genotypes_stats": ([_P, _P, _P, _P, _P], _I),
    "cs_genotypes_destroy": ([_P], None),
    "cs_kinship_create": ([_P, _P, _I64, _P, _I64, _P], _I),
    "cs_kinship_info": ([_P, _P, _P], _I),
    "cs_kinship_apply": ([_P, _P, _I64, _I64, _P, _I64, _I, _P], _I),
    "cs_kinship_apply_host": ([_P, _P, _I64, _I64, _P, _I64, _I], _I),
    "cs_kinship_apply_noalloc": ([_P, _P, _I64, _I64, _P, _I64, _P], _I),
    "cs_genotype_multiply_zt": ([_P, _P, _I64, _I64, _P, _I64, _I, _P], _I),
    "cs_genotype_multiply_z": ([_P, _P, _I64, _I64, _P, _I64, _I, _P], _I),
    "cs_genotype_multiply_zt_host": ([_P, _P, _I64, _I64, _P, _I64, _I], _I),
    "cs_genotype_multiply_z_host": ([_P, _P, _I64, _I64, _P, _I64, _I], _I),
    "cs_kinship_trace": ([_P, _P], _I),
    "cs_kinship_diagonal": ([_P, _P], _I),
    "cs_kinship_destroy": ([_P], None),
    "cs_lmm_create": ([_P], _I),
    "cs_grm_default_options": ([_P], None),
    "cs_kinship_apply_f32": ([_P, _P, _I64, _I64, _P, _I64, _I, _P], _I),
    "cs_mv_vce_default_options": ([_P], None),
    "cs_mv_eigen_vce_prepare": ([_P, _P, _I64, _P, _I64, _P, _I64, _I, _P], _I),
    "cs_mv_eigen_vce_run_null": ([_P, _P, _P, _P, _P], _I),
    "cs_mv_eigen_vce_dims": ([_P, _P, _P, _P], _I),
    "cs_mv_eigen_vce_get": ([_P, _P, _P, _P, _P, _P, _P], _I),
    "cs_mv_eigen_vce_destroy": ([_P], None),
    "cs_mvlmm_scan_vce": ([_P, _P, _I64, _P, _I64, _I64, _I, _P, _P, _P, _P, _P, _P], _I),
    "cs_grm_create": ([_P, _P, _I64, _P, _P], _I),
    "cs_grm_from_host": ([_I64, _P, _I64, _P], _I),
    "cs_grm_loco": ([_P, _P, _P], _I),
    "cs_grm_info": ([_P, _P, _P, _P], _I),
    "cs_grm_copy": ([_P, _P, _I64, _P, _I64], _I),
    "cs_grm_destroy": ([_P], None),
    "cs_eigen_vce_prepare": ([_P, _P, _I64, _P, _P, _I64, _I, _P], _I),
    "cs_eigen_vce_run_null": ([_P, _P], _I),
    "cs_eigen_vce_dims": ([_P, _P, _P, _P], _I),
    "cs_eigen_vce_get": ([_P, _P, _P, _P, _P, _I64], _I),
    "cs_eigen_vce_destroy": ([_P], None),
    "cs_lmm_prepare_from_vce": ([_P, _P, _I], _I),
    "cs_lmm_prepare_lowrank_matrix_free": (
        [_P, _P, _P, _P, _I64, _I, _I, _I64, _D, _I, _I, _P], _I),
    "cs_lmm_lowrank_basis": ([_P, _P, _I64, _P], _I),
    "cs_lmm_scan": ([_P, _P, _P, _I64, _D, _I, _P, _P, _P, _P, _P, _P], _I),
    "cs_lmm_scan_window": ([_P, _P, _P, _I64, _I64, _I64, _D, _I, _P, _P, _P, _P, _P, _P], _I),
    "cs_lmm_destroy": ([_P], None),
    "cs_normal_matrix": ([C.c_uint64, _I64, _I64, _P], _I),
    "cs_mv_stcg_default_options": ([_P], None),
    "cs_mv_stcg_solve": ([_P, _D, _P, C.c_int32, _P, _I64, _P, _P, _P, _P], _I),
    "cs_lmm_run_default_options": ([_P], None),
    "cs_run_lmm_matrix_free": ([_P, _P, _I64, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                _I, _P], _I),
    "cs_gwas_lmm_default_options": ([_P], None),
    "cs_run_gwas_lmm": ([_P, _P, _P], _I),
    "cs_pcg_solve": ([_P, _D, _D, _D, _P, _I64, _I64, _P, _I64, _D, _I, _I, _I, _P, _P], _I),
    "cs_pcg_solve_records": ([_P, _D, _P, _I64, _I, _D, _D, _D, _P, _I64, _I64, _P, _I64, _D, _I,
                              _I, _I, _P, _P], _I),
    "cs_vce_default_options": ([_P], None),
    "cs_vce_create": ([_P], _I),
    "cs_vce_solve_stcg": ([_P, _P, _D, _P, _I64, _I, _P, _P, _I64, _P, _P], _I),
    "cs_vce_solution": ([_P, _P, _P, _P], _I),
    "cs_vce_history": ([_P, _P, _P], _I),
    "cs_vce_destroy": ([_P], None),
    "cs_stcg_scan": ([_P, _P, _I64, _P, _P, _I64, _P, _P, _I64, _D, _D, _D, _D, _I64, _I64,
                      _P, _P, _P, _P, _P, _P], _I),
    "cs_mvlmm_scan": ([_P, _P, _I64, _P, _I64, _P, _P, _I64, _P, _I64, _P, _P, _I64, _I64, _I,
                       _P, _P, _P, _P, _P, _P], _I),
    "cs_server_default_options": ([_P], None),
    "cs_server_create": ([_P, _P, _I64, _P, _P], _I),
    "cs_server_submit": ([_P, _P, _P], _I),
    "cs_server_wait": ([_P, _I64, _D, _P], _I),
    "cs_server_result": ([_P, _I64, C.c_int32, _P, _P, _P, _P, _P, _P, _P], _I),
    "cs_server_release": ([_P, _I64], _I),
    "cs_server_stats": ([_P, _P], _I),
    "cs_server_destroy": ([_P], None),
    "cs_write_assoc_txt": ([C.c_char_p, C.c_char_p, _I64, C.c_int32, _P, _P, _P, _P, _P, _P, _I], _I),
    "cs_write_assoc_mv_txt": ([C.c_char_p, C.c_char_p, _I64, C.c_int32, _P, _P, _P, _P, _P], _I),
    "cs_write_scan_meta": ([C.c_char_p, C.c_int32, _D], _I),
    "cs_write_scan_meta_full_eigen": ([C.c_char_p], _I),
    "cs_write_assoc": ([C.c_char_p, C.c_char_p, _I64, C.c_int32, _P, _P, _P, _P, _P, _P, _P, _I64,
                        _I, _I], _I),
    "cs_append_cosmic_sumstats": ([C.c_char_p, C.c_char_p, _I64, C.c_int32, _P, _P, _P, _P, _P,
                                   _P, C.c_char_p, _I, _I, C.c_char_p], _I),
    "cs_append_scan_common_meta": ([C.c_char_p, C.c_char_p, _I64, _I, _I, _I], _I),
    "cs_write_low_rank_meta": ([C.c_char_p, C.c_int32, _P, _P, _I64, _D, _P], _I),
    "cs_fam_read": ([C.c_char_p, _P], _I),
    "cs_samples_count": ([_P, _P], _I),
    "cs_samples_id": ([_P, _I64, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t], _I),
    "cs_samples_fam_phenotype": ([_P, _P], _I),
    "cs_samples_destroy": ([_P], None),
    "cs_pheno_load": ([C.c_char_p, C.c_int32, _D, _P], _I),
    "cs_pheno_load_matrix": ([C.c_char_p, _P, C.c_int32, _D, _P], _I),
    "cs_pheno_traits": ([_P, _P], _I),
    "cs_pheno_align": ([_P, _P, _P, _P], _I),
    "cs_pheno_align_matrix": ([_P, _P, _P, _I64, _P], _I),
    "cs_pheno_destroy": ([_P], None),
    "cs_covar_load": ([C.c_char_p, _D, _P], _I),
    "cs_covar_load_categorical": ([C.c_char_p, C.c_char_p, _P], _I),
    "cs_covar_columns": ([_P, _P], _I),
    "cs_covar_align": ([_P, _P, _P, _I64, _P], _I),
    "cs_covar_destroy": ([_P], None),
    "cs_filter_samples": ([_P, _I64, _P, _I64, C.c_int32, _P, _P], _I),
    "cs_profile_enable": ([_I], _I),
    "cs_profile_summary": ([C.c_char_p, C.c_size_t, _P], _I),
    "cs_launch_count": ([_P], _I),
}

_lib = None


def declared_functions() -> list[str]:
    """Function names declared in the public header."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cs_[a-z0-9_]+)\s*\(", text)))


def load(path: str = LIB_PATH):
    """Loads the shared library; raises if it has not been built."""
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m cosmicscanner_b200.build` "
            "(the package has no CPU fallback)")
    L = C.CDLL(path)
    for name, (args, res) in _SIGNATURES.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L


def lib():
    global _lib
    if _lib is None:
        _lib = load()
    return _lib
