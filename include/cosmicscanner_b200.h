/*
 * cosmicscanner_b200 — C ABI of the B200 (sm_100a) matrix-free mixed-model path.
 *
 * Every entry point returns an int status (CS_OK = 0, negative on error) and never
 * throws; cs_last_error() returns the message of the calling thread's last failure.
 * Handles are opaque.  Dense matrices are column-major with an explicit leading
 * dimension, as Eigen stores them in the reference; "_host" entry points take host
 * pointers and synchronise, the others take device pointers and a cudaStream_t
 * (passed as void*, NULL = the legacy default stream).
 *
 * Each declaration names the reference interface it replaces (file:line in the
 * CosmicScanner sources).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CS_OK = 0,
    CS_ERR_INVALID_ARGUMENT = -1, /* dimension / index errors: std::runtime_error in the reference */
    CS_ERR_CUDA = -2,             /* CUDA runtime or library failure */
    CS_ERR_IO = -3,               /* file cannot be opened / read */
    CS_ERR_FORMAT = -4,           /* bad .bed magic or unsupported mode */
    CS_ERR_NUMERIC = -5,          /* singular system, failed factorisation, non-finite values */
    CS_ERR_NOT_CONVERGED = -6,    /* iteration limit reached where convergence is required */
    CS_ERR_UNSUPPORTED = -7,      /* configuration the library does not implement */
};

/* Arithmetic of an operator apply. */
enum {
    CS_PRECISION_FP64 = 0,  /* FP64 decode-GEMM (the plain form) */
    CS_PRECISION_MIXED = 1, /* tensor-core form: exact genotypes x split right-hand sides */
};

typedef struct cs_genotypes cs_genotypes;
typedef struct cs_kinship cs_kinship;
typedef struct cs_lmm cs_lmm;

const char* cs_last_error(void);
const char* cs_version(void);

/* ---------------------------------------------------------------- genotypes
 * Replaces PlinkReader::load / openBed (libCosmicCore/src/plink_reader.cpp:28-92)
 * and PlinkReader::computeStats (plink_reader.cpp:187-239).  The packed SNP-major
 * matrix is copied to HBM once and stays resident; statistics (mean, 1/sd over all
 * .fam samples) are computed on the device, bit-exact with the reference. */
int cs_genotypes_create(const uint8_t* bed_bytes, size_t n_bytes, int64_t n_samples,
                        int64_t n_snps, cs_genotypes** out);
/* Reads prefix.fam / prefix.bim (line counts) and prefix.bed. */
int cs_genotypes_open_plink(const char* prefix, cs_genotypes** out);
int cs_genotypes_info(const cs_genotypes* g, int64_t* n_samples, int64_t* n_snps,
                      int64_t* bytes_per_snp);
/* Host copies of the per-SNP statistics (any output may be NULL). */
int cs_genotypes_stats(const cs_genotypes* g, double* mean, double* inv_std, int32_t* count,
                       double* sum);
void cs_genotypes_destroy(cs_genotypes* g);

/* ---------------------------------------------------------------- kinship operator
 * Replaces cosmic::KinshipOperator / PlinkKinshipOperator (src/kinship_operator.h:18-95)
 * and createKinshipOperator (src/kinship_operator.cpp:370-374):
 * K = Z Z^T / M over the selected samples (keep, NULL = all) and variants (NULL = all);
 * Z = (G - mean) * inv_std with missing calls contributing zero.  Out-of-range
 * indices and an empty variant set fail with CS_ERR_INVALID_ARGUMENT, as the reference
 * constructor throws. */
int cs_kinship_create(const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                      const int32_t* variants, int64_t n_variants, cs_kinship** out);
/* rows() / cols() / numVariants() (kinship_operator.h:22-27). */
int cs_kinship_info(const cs_kinship* op, int64_t* rows, int64_t* num_variants);
/* apply(const MatrixXd& X, MatrixXd& out) / apply_block (kinship_operator.cpp:220-302):
 * Y = K X for X rows() x k.  Y may alias X.  k == 0 is a no-op.  Device pointers. */
int cs_kinship_apply(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                     int64_t ldy, int precision, void* stream);
/* The FP32 variant of cs_kinship_apply for callers that keep V in single precision: X and Y
 * are float (device, column-major); the apply runs in the requested form on FP64-widened
 * inputs and the result is rounded to float once.  Y may alias X. */
int cs_kinship_apply_f32(cs_kinship* op, const float* X, int64_t ldx, int64_t k, float* Y,
                         int64_t ldy, int precision, void* stream);
/* Same with host pointers (synchronous). */
int cs_kinship_apply_host(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                          int64_t ldy, int precision);
/* No counterpart in the reference.  The FP64 Y = K X of cs_kinship_apply for callers that
 * cannot let the library allocate device memory (a process that has reserved HBM for its
 * own pool, or a request loop that cannot absorb cudaMalloc's synchronisation).  Scratch
 * comes from a fixed 16 MiB array in the library's device memory, so it needs
 * (2 * rows() + selected variants) * k <= 2^21 doubles, else CS_ERR_INVALID_ARGUMENT.
 * Allocates nothing.  The first call on a device looks up the array's device address and
 * should come before any stream capture.  Calls share the array: calls whose work
 * overlaps on the GPU race and must be serialised by the caller.  The operator's device
 * must be current (else CS_ERR_INVALID_ARGUMENT), and the library must not be used across a
 * cudaDeviceReset of that device (the array's address is looked up once).  Device pointers. */
int cs_kinship_apply_noalloc(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                             int64_t ldy, void* stream);
/* GenotypeMatrix::multiply_Zt_v / multiply_Z_v (libCosmicCore/src/matrix_adapter.h:40-53, as
 * PlinkReader implements them, plink_reader.cpp:241-438 with the keep-subset forms) over the
 * operator's selection: Z is rows() x numVariants(), z = (dosage - mean) / sd with the
 * all-sample statistics, missing calls 0, variants with 1/sd == 0 all zero, no 1/M scaling.
 * multiply_zt: U (numVariants x k) = Z^T X for X (rows x k); multiply_z: Y (rows x k) = Z V for
 * V (numVariants x k).  Column-major device pointers; precision as cs_kinship_apply.  The
 * _host forms take host arrays and return when the result is there. */
int cs_genotype_multiply_zt(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* U,
                            int64_t ldu, int precision, void* stream);
int cs_genotype_multiply_z(cs_kinship* op, const double* V, int64_t ldv, int64_t k, double* Y,
                           int64_t ldy, int precision, void* stream);
int cs_genotype_multiply_zt_host(cs_kinship* op, const double* X, int64_t ldx, int64_t k,
                                 double* U, int64_t ldu, int precision);
int cs_genotype_multiply_z_host(cs_kinship* op, const double* V, int64_t ldv, int64_t k,
                                double* Y, int64_t ldy, int precision);
/* trace() and getDiagonal() (kinship_operator.cpp:306-368); diag is a host array. */
int cs_kinship_trace(const cs_kinship* op, double* trace);
int cs_kinship_diagonal(cs_kinship* op, double* diag);
void cs_kinship_destroy(cs_kinship* op);

/* ---------------------------------------------------------------- low-rank LMM engine
 * Replaces LmmEngine::prepareLowRankMatrixFree (src/lmm_engine.cpp:897-1095):
 * randomized subspace iteration on K (Omega ~ N(0,1) from mt19937_64(seed), two power
 * iterations, QR, eigendecomposition of Q^T K Q), trace-fraction rank selection, tail-mean
 * residual eigenvalue, then REML over log(eta) by an 81-point grid and golden-section
 * search.  y has rows() entries, X is rows() x p column-major (the reference receives X
 * as MatrixXf: callers mirroring it pass FP32-rounded values).  Host pointers. */
typedef struct {
    int32_t requested_rank;
    int32_t effective_rank;
    int32_t sketch_size;
    int32_t trace_threshold_met;
    double residual_eigenvalue;
    double relative_frobenius_error;
    double trace;
    double trace_fraction;
    double sigma2_g;
    double sigma2_e;
    double delta;
    double log_eta;
    double reml_objective;
    double seconds;
} cs_lowrank_diagnostics;

int cs_lmm_create(cs_lmm** out);
int cs_lmm_prepare_lowrank_matrix_free(cs_lmm* lmm, cs_kinship* op, const double* y,
                                       const double* X, int64_t p, int rank, int oversample,
                                       int64_t seed, double trace_threshold, int min_rank,
                                       int precision, cs_lowrank_diagnostics* diag);
/* Low-rank basis after preparation: U (rows() x rank, column-major, host) and eigenvalues. */
int cs_lmm_lowrank_basis(const cs_lmm* lmm, double* U, int64_t ldu, double* lambda);
/* Replaces LmmEngine::scan(PlinkReader, ...) -> scanLowRank (src/lmm_engine.cpp:1269-1361)
 * for every SNP of g (no chromosome filter): keep lists the analysed samples in the order
 * of y.  Per-SNP host outputs of length n_snps; tested[j] = 0 where the reference writes no
 * row (MAF filter, variance <= 1e-12).  Any output may be NULL. */
int cs_lmm_scan(cs_lmm* lmm, const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                double min_maf, int precision, double* beta, double* se, double* pvalue,
                double* log10p, double* freq, int32_t* tested);
/* The same scan restricted to SNPs [snp_begin, snp_end) of g (a chromosome of a LOCO run,
 * src/gwas_scanner.cpp:447 with chrom_filter; or a --scan-from/to-bp window); the outputs
 * have snp_end - snp_begin entries. */
int cs_lmm_scan_window(cs_lmm* lmm, const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                       int64_t snp_begin, int64_t snp_end, double min_maf, int precision,
                       double* beta, double* se, double* pvalue, double* log10p, double* freq,
                       int32_t* tested);
void cs_lmm_destroy(cs_lmm* lmm);

/* ---------------------------------------------------------------- multi-trait matrix-free REML
 * The multivariate null model of `--model multivariate` (MvEigenVce::runNullModel's EM,
 * libCosmicCore/src/eigen_vce.cpp:551-604, 1031-1065) without the dense N x N eigenbasis:
 * vec(Y) ~ N((I_d (x) X) b, Vg (x) K + Ve (x) I), K = Z Z^T / kinship_divisor over the operator's
 * samples.  Each EM iteration solves (Q V Q) x = Q [Y | Z_1 .. Z_S] by conjugate gradients
 * (Q = I - X (X'X)^-1 X' per trait; P = Q (Q V Q)^+ Q), S Rademacher probes of n x d redrawn per
 * iteration from mt19937_64(probe_seed), so every kinship apply carries (1 + S) d columns; one
 * more apply K [PY | Z] gives (PY)' K (PY) and the Hutchinson estimates of tr(P (E_ab (x) K)).
 * Update Vg += Vg (Qg - Tg) Vg / (n - p), Ve likewise; starting values Cov(Y) / 2; stop when
 * (|dVg|^2 + |dVe|^2) / max(1, 2 d^2) < tol.  Y n x d and X n x p column-major host arrays; Vg, Ve
 * d x d column-major outputs. */
typedef struct cs_mv_stcg_options {
    int32_t max_iter;      /* EM iterations (100) */
    double tol;            /* the reference's EM stopping threshold (1e-8) */
    int32_t mc_samples;    /* probes per iteration (32) */
    double pcg_tol;        /* CG threshold (1e-8) */
    int32_t pcg_relative;  /* 1: ||r|| < pcg_tol ||b|| per probe / trait group (default); 0: absolute */
    int32_t pcg_max_iter;  /* (2000) */
    uint64_t probe_seed;   /* (20250101) */
    int32_t precision;     /* CS_PRECISION_FP64 or CS_PRECISION_MIXED for the kinship applies */
} cs_mv_stcg_options;
typedef struct cs_mv_stcg_result {
    int32_t iterations, converged;
    int64_t pcg_iterations;    /* CG iterations summed over probe / trait groups */
    int64_t operator_applies;  /* kinship applies */
    int64_t operator_columns;  /* right-hand sides they carried */
    double seconds;
} cs_mv_stcg_result;
void cs_mv_stcg_default_options(cs_mv_stcg_options* opt);
int cs_mv_stcg_solve(cs_kinship* op, double kinship_divisor, const double* Y, int32_t d,
                     const double* X, int64_t p, const cs_mv_stcg_options* opt, double* Vg,
                     double* Ve, cs_mv_stcg_result* res);

/* ---------------------------------------------------------------- the whole job
 * GwasScanner::runLocoScan's PLINK matrix-free branch (src/gwas_scanner.cpp:74-509) in the
 * library's C++: GRM variant selection from the all-sample statistics (:258-277), one null
 * model (or, when chrom spans more than one chromosome and loco is set, the
 * leave-one-chromosome-out loop of :299-314, 464-472 in sort_chrom_labels order, :62-72), each
 * with the low-rank fall-back rule of :347-383, then the scan of every SNP. */
typedef struct cs_lmm_run_options {
    int32_t rank;            /* --fastlmm-max-rank (256) */
    int32_t oversample;      /* --lmm-low-rank-oversample (10) */
    int64_t seed;            /* --lmm-low-rank-seed (42) */
    double trace_threshold;  /* --fastlmm-trace-threshold (0.95) */
    int32_t min_rank;        /* (1) */
    double min_maf;          /* --maf (0.01): GRM selection and scan filter */
    int32_t precision;       /* CS_PRECISION_MIXED (default) or CS_PRECISION_FP64 */
    int32_t loco;            /* 1: leave one chromosome out when there are several (--no-loco: 0) */
    int32_t no_fallback;     /* --fastlmm-no-fallback (1) */
    double error_tol;        /* --lmm-low-rank-error-tol (1.0) */
} cs_lmm_run_options;
enum { CS_FALLBACK_NONE = 0, CS_FALLBACK_TRACE_THRESHOLD = 1, CS_FALLBACK_ERROR_TOLERANCE = 2 };
typedef struct cs_lmm_run_scope {
    char label[32];                 /* "GLOBAL" or the left-out chromosome */
    cs_lowrank_diagnostics diag;    /* the first sketch's diagnostics, refit VCs on fall-back */
    int32_t fallback;               /* CS_FALLBACK_* */
} cs_lmm_run_scope;
void cs_lmm_run_default_options(cs_lmm_run_options* opt);
/* g resident; keep (NULL: every sample) lists the analysed samples in the order of y; X is
 * n_keep x p column-major (FP32-rounded values where the caller mirrors the reference's
 * MatrixXf covariates); chrom (NULL: one chromosome) holds each SNP's .bim label.  Per-SNP host
 * outputs of g's SNP count (NaN / tested 0 where the reference writes no row); scopes receives
 * up to max_scopes null models and n_scopes their number.  Host pointers. */
int cs_run_lmm_matrix_free(const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                           const double* y, const double* X, int64_t p, const char* const* chrom,
                           const cs_lmm_run_options* opt, double* beta, double* se,
                           double* pvalue, double* log10p, double* freq, int32_t* tested,
                           cs_lmm_run_scope* scopes, int32_t max_scopes, int32_t* n_scopes);
/* `cosmicscanner gwas --model lmm --fastlmm --fastlmm-matrix-free --bfile B --out O
 * [--pheno P --mpheno k] [--qcovar Q] [--covar C]` from files to files: the .fam samples,
 * phenotype (.fam column without --pheno), [1 | quantitative | categorical dummies] as
 * float and the complete-sample keep list (src/models/univariate_model.cpp:389-426), the job
 * above, then O.assoc.txt (rows chromosome by chromosome under LOCO; GWAS-SSF with out_ssf,
 * gzip with out_gz), O.cosmic.sumstats, O.scan.meta.txt and O.low_rank.meta.tsv. */
typedef struct cs_gwas_lmm_options {
    const char* bfile;       /* PLINK prefix */
    const char* out;         /* output prefix */
    const char* pheno;       /* NULL: the .fam phenotype */
    int32_t mpheno;          /* 1-based phenotype column (1) */
    const char* qcovar;      /* quantitative covariates (NULL: none) */
    const char* covar;       /* categorical covariates (NULL: none) */
    double missing_code;     /* -9 */
    cs_lmm_run_options run;
    int32_t out_gz, out_ssf;
    const char* created;     /* "# Created:" of .cosmic.sumstats (NULL: now, UTC) */
} cs_gwas_lmm_options;
void cs_gwas_lmm_default_options(cs_gwas_lmm_options* opt);
int cs_run_gwas_lmm(const cs_gwas_lmm_options* opt, int64_t* n_kept, int32_t* n_scopes);

/* ---------------------------------------------------------------- dense exact tier
 * The default `gwas --model lmm` route (src/gwas_scanner.cpp:131-215, 384-399; no LOCO):
 * the dense GRM, EigenVce's eigenbasis and Brent null model, and LmmEngine::scan's exact
 * branch.  All matrices stay on the device; host pointers in and out.
 *
 * cs_grm_create replaces GrmBuilder::compute (libCosmicCore/src/grm_builder.cpp:87-394) for
 * one population, unit SNP weights and no HWE filter, over every sample of g: per SNP
 * (variants in .bed order, NULL = all) the code counts decide validity (observed, MAF >=
 * (float)min_maf and > 1e-8), the value map of the algorithm (0/3 Yang: (x - 2p) / sqrt(2pq);
 * 1 VanRaden: x - 2p; 2 Zeng; 4 Vitezica; 5 TrueVar) with 2p rounded to float as the
 * reference stores it, then G = sum Z Z^T divided by the valid-SNP count (0, 3), the mean
 * diagonal (2) or the float-rounded sum of 2pq (1, 4, 5). */
typedef struct cs_grm cs_grm;
typedef struct cs_eigen_vce cs_eigen_vce;
typedef struct {
    double min_maf;     /* GrmBuilder::Options::min_maf (compared as float); default 0.01 */
    int32_t algorithm;  /* GrmBuilder::Options::algorithm; default 1 (VanRaden) */
} cs_grm_options;
void cs_grm_default_options(cs_grm_options* opt);
int cs_grm_create(const cs_genotypes* g, const int32_t* variants, int64_t n_variants,
                  const cs_grm_options* opt, cs_grm** out);
/* The LOCO GRM of src/gwas_scanner.cpp:476-491 from the global GRM and the GRM of one
 * chromosome's SNPs (both cs_grm_create over the same genotypes and options; the reference's
 * GrmBuilder::computeSplit keeps the chromosome's raw sum, here raw = G_chr x its divisor):
 * G_loco = G (S / S_loco) - raw_chr / S_loco with S the valid-SNP count (algorithms 0, 3) or
 * the 2pq sum, S_loco = S - S_chr; the global GRM unchanged when S_chr = 0 or S_loco <= 1e-6. */
int cs_grm_loco(const cs_grm* global, const cs_grm* chrom, cs_grm** out);
/* A caller's own n x n GRM (host, column-major, ld >= n), as EigenVce::prepare accepts any G. */
int cs_grm_from_host(int64_t n, const double* G, int64_t ldg, cs_grm** out);
/* getNumSamples / getTotalSnps / getSum2pq of the builder (valid = 0, sum = 0 for a host GRM). */
int cs_grm_info(const cs_grm* grm, int64_t* n, int64_t* n_valid, double* sum_2pq);
/* G[keep, keep] (DataFilter::subsetSquare, libCosmicCore/src/data_filter.h) to host
 * (column-major, ld >= n_keep); keep = NULL copies all of G. */
int cs_grm_copy(const cs_grm* grm, const int32_t* keep, int64_t n_keep, double* out, int64_t ld);
void cs_grm_destroy(cs_grm* grm);

/* EigenVce::prepare (libCosmicCore/src/eigen_vce.cpp:19-63) on G[keep, keep]: with
 * use_covariate_projection and p > 0 the eigenbasis of the covariate-projected G — n - p
 * eigenvalues D (ascending, negatives set to 0), W_proj (n x (n - p)) spanning the complement
 * of X, Uty = W_proj^T y, no UtX; otherwise the eigenbasis of G with UtX = U^T X.  The
 * complement is formed as P G P + alpha X(X^T X)^{-1} X^T with alpha above the spectrum, so
 * the covariate directions separate from the rest without forming Q's complement; X must
 * have full column rank.  y: n_keep, X: n_keep x p column-major (FP32-rounded values, as the
 * reference's MatrixXf).  keep = NULL uses every sample of the GRM. */
int cs_eigen_vce_prepare(const cs_grm* grm, const int32_t* keep, int64_t n_keep, const double* y,
                         const double* X, int64_t p, int use_covariate_projection,
                         cs_eigen_vce** out);
typedef struct {
    double sigma2_g, sigma2_e, delta;  /* delta = sigma2_e / sigma2_g */
    double sigma2_g_se, sigma2_e_se;   /* from the AI matrix; the simplified SEs when singular */
    double log_likelihood;             /* REML log-likelihood at the estimate */
    double max_score;                  /* max |score| at the estimate */
    int64_t n_eig;
    int32_t converged;
    double seconds;
} cs_eigen_vce_result;
/* EigenVce::runNullModel with the Brent solver (eigen_vce.cpp:83-112): VCESolver::
 * solveDiagonal's golden-section search over log10 delta in [-5, 5], tol 1e-5
 * (libCosmicCore/src/vce.cpp:3073-3175), then updateRemlDiagnostics (eigen_vce.cpp:114-153). */
int cs_eigen_vce_run_null(cs_eigen_vce* vce, cs_eigen_vce_result* out);
int cs_eigen_vce_dims(const cs_eigen_vce* vce, int64_t* n, int64_t* n_eig, int64_t* p);
/* getEigenvalues / getUty / getUtX / getProjectedW to host; any output may be NULL (W:
 * n x n_eig column-major, ld >= n). */
int cs_eigen_vce_get(const cs_eigen_vce* vce, double* D, double* Uty, double* UtX, double* W,
                     int64_t ldw);
void cs_eigen_vce_destroy(cs_eigen_vce* vce);
/* LmmEngine::prepareFromVce (src/lmm_engine.cpp:716-725): cs_lmm_scan / cs_lmm_scan_window
 * then run the exact scan (:1363-1474): per SNP UtG = W_proj^T g (tensor-core projection in
 * mixed precision, FP64 decode-GEMM otherwise), score = UtG . P y, var = UtG^T V^-1 UtG minus
 * the covariate term (skipped with use_residuals, the reference's setting for GRM algorithm
 * 0), P = chisq(score^2 / var, 1).  The run must have gone through cs_eigen_vce_run_null. */
int cs_lmm_prepare_from_vce(cs_lmm* lmm, const cs_eigen_vce* vce, int use_residuals);

/* The multi-trait dense null (`--model multivariate`, src/models/multivariate_model.cpp:
 * 955-1015): MvEigenVce (libCosmicCore/src/eigen_vce.cpp:496-911, 1031-1065) on the same
 * device eigenbasis as cs_eigen_vce_prepare, then the mvLMM scan from it. */
typedef struct cs_mv_eigen_vce cs_mv_eigen_vce;
typedef struct {
    int32_t max_iter;    /* MvEigenVce::Options::max_iter; the multivariate model passes
                          * --reml-maxit (1000) */
    double tol;          /* tol on the mean squared EM change (--reml-tol, 1e-8) */
    int32_t aireml;      /* VceSolver::AIREML (--mv-aireml) instead of EM */
    int32_t em_min_iter; /* EM warm-up of the AI-REML route (10) */
    int32_t ai_max_iter; /* AI-REML iterations (50) */
    double ai_tol;       /* AI-REML stop on |delta| / sqrt(parameters) (1e-8) */
} cs_mv_vce_options;
void cs_mv_vce_default_options(cs_mv_vce_options* opt);
/* MvEigenVce::prepare (:496-549) on G[keep, keep] with Y (n_keep x d, column-major, 1 <= d <= 8)
 * and X (n_keep x p): the eigenbasis (covariate projection when use_projection; covariates
 * without it are not supported), U'Y, and the starting Vg = Ve = Cov(Y) / 2 with the
 * reference's divisor (samples after the projection - 1). */
int cs_mv_eigen_vce_prepare(const cs_grm* grm, const int32_t* keep, int64_t n_keep,
                            const double* Y, int64_t d, const double* X, int64_t p,
                            int use_projection, cs_mv_eigen_vce** out);
/* runNullModel (:1031-1065): EM (updateEM :551-604) until the mean squared change of (Vg, Ve)
 * is below tol — converged = 0 after max_iter updates, where the reference's driver stops with
 * "Multivariate null model did not converge" — or runAireml (:631-911) with aireml.  logl is
 * the REML log-likelihood of calcLogLikelihood (:613-629) at the result. */
int cs_mv_eigen_vce_run_null(cs_mv_eigen_vce* vce, const cs_mv_vce_options* opt,
                             int32_t* converged, int32_t* iterations, double* logl);
int cs_mv_eigen_vce_dims(const cs_mv_eigen_vce* vce, int64_t* n, int64_t* n_eig, int64_t* d);
/* getVg / getVe / their SEs (AI-REML only, else 0) as d x d, eigenvalues (n_eig), U'Y
 * (n_eig x d); any output may be NULL. */
int cs_mv_eigen_vce_get(const cs_mv_eigen_vce* vce, double* Vg, double* Ve, double* Vg_se,
                        double* Ve_se, double* D, double* Uty);
void cs_mv_eigen_vce_destroy(cs_mv_eigen_vce* vce);
/* MvLmmEngine::prepareFromVce + scan (src/mvlmm_engine.cpp:195-207, 756-931) with the device
 * eigenbasis of vce; outputs as cs_mvlmm_scan. */
int cs_mvlmm_scan_vce(const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                      const cs_mv_eigen_vce* vce, int64_t snp_begin, int64_t snp_end,
                      int precision, double* beta, double* cov, double* wald, double* pvalue,
                      double* freq, int32_t* status);

/* The test matrix of src/lmm_engine.cpp:917-922 (also libCosmicCore/src/rng.h:27-33):
 * n x cols standard normals drawn column by column from std::normal_distribution<double>
 * over std::mt19937_64(seed), generated on the device (engine, polar acceptance, transform)
 * and copied to `out` (host, column-major, ld = n). */
int cs_normal_matrix(uint64_t seed, int64_t n, int64_t cols, double* out);

/* ---------------------------------------------------------------- PCG and AI-REML
 * Replaces cosmic::MatrixFreePCG (libCosmicCore/src/matrix_free_pcg.h:9-75) for the mixed-
 * model covariance V = sigma2_g K + sigma2_e I with the scalar preconditioner
 * 1/(sigma2_g + sigma2_e) (libCosmicCore/src/stcg_vce.cpp:117-126).  B and X are device,
 * column-major (rows() x k, leading dimensions ldb / ldx); all k right-hand sides advance
 * together, each with its own CG recurrence, and stop when ||r|| < tol (relative = 0, the
 * reference's absolute rule, matrix_free_pcg.h:51) or ||r|| < tol ||b|| (relative = 1), or at
 * max_iter without an error (the reference returns silently too).  K is the operator's
 * Z Z^T scaled by 1 / kinship_divisor (<= 0: the operator's own selected-variant count).
 * iterations (host, k entries, may be NULL) receives each column's iteration count. */
int cs_pcg_solve(cs_kinship* op, double kinship_divisor, double sigma2_g, double sigma2_e,
                 const double* B, int64_t ldb, int64_t k, double* X, int64_t ldx, double tol,
                 int relative, int max_iter, int precision, int32_t* iterations, void* stream);

/* MatrixFreePCG::solve (matrix_free_pcg.h:20-68) with the covariance STCG_VCE hands it
 * (libCosmicCore/src/stcg_vce.cpp:80-126): V = sigma2_g Zr K Zr^T + sigma2_pe Zr Zr^T +
 * sigma2_e I over n_records records, Zr mapping record i to operator row rec_to_row[i] (-1: no
 * genotype row; NULL: record i is row i, n_records == rows()), K = Z Z^T / kinship_divisor, the
 * permanent-environment term only with with_pe, the scalar preconditioner
 * 1/(sigma2_g + [sigma2_pe] + sigma2_e).  B and X are device, column-major
 * (n_records x k); stopping as cs_pcg_solve. */
int cs_pcg_solve_records(cs_kinship* op, double kinship_divisor, const int32_t* rec_to_row,
                         int64_t n_records, int with_pe, double sigma2_g, double sigma2_pe,
                         double sigma2_e, const double* B, int64_t ldb, int64_t k, double* X,
                         int64_t ldx, double tol, int relative, int max_iter, int precision,
                         int32_t* iterations, void* stream);

/* Options of the matrix-free AI-REML (VCEConfig, libCosmicCore/src/vce.h:139-160, as
 * src/models/repeatability_model.cpp:604-612 fills it). */
typedef struct cs_vce_options {
    int32_t max_iter;     /* AI-REML iterations (--reml-maxit, 50) */
    double tol;           /* stop when the largest relative change of theta < tol (1e-6) */
    int32_t mc_samples;   /* Rademacher probes per iteration (VCEConfig::mc_samples, 20) */
    double pcg_tol;       /* CG threshold on ||r|| (VCEConfig::pcg_tol, 1e-10) */
    int32_t pcg_relative; /* 0: absolute ||r|| < pcg_tol (reference); 1: ||r|| < pcg_tol ||b|| */
    int32_t pcg_max_iter; /* VCEConfig::pcg_max_iter, 2000 */
    int32_t slq_probes;   /* SLQ probes for the log-likelihood (30); 0 skips it */
    int32_t slq_steps;    /* Lanczos steps per SLQ probe (15) */
    uint64_t probe_seed;  /* mt19937_64 seed of the trace probes (20250101) */
    int32_t precision;    /* CS_PRECISION_FP64 or CS_PRECISION_MIXED for the kinship applies */
    int32_t precond_rank; /* 0: the reference's scalar preconditioner 1/(sum of components);
                             r > 0: low-rank deflation M^-1 = base I + U diag(c) U^T with the
                             top r eigenpairs of K from a randomized sketch (records that map
                             one-to-one onto operator rows only; otherwise the scalar one) */
} cs_vce_options;

typedef struct cs_vce_result {
    double sigma2_g, sigma2_pe, sigma2_e;
    double logl;               /* REML log-likelihood of the last iteration (NaN without SLQ) */
    int32_t iterations, converged;
    int64_t pcg_iterations;    /* CG iterations summed over right-hand sides */
    int64_t operator_applies;  /* kinship applies (each carries a block of right-hand sides) */
    int64_t operator_columns;  /* right-hand sides carried by those applies */
    double seconds;
} cs_vce_result;

typedef struct cs_vce cs_vce;

void cs_vce_default_options(cs_vce_options* opt);
int cs_vce_create(cs_vce** out);
/* Replaces STCG_VCE::solve() (libCosmicCore/src/stcg_vce.cpp:157-407): matrix-free AI-REML
 * for theta = (sigma2_g, sigma2_pe, sigma2_e) with V = sg2 Zr K Zr^T + spe2 Zr Zr^T + se2 I
 * over n_records records.  rec_to_row[i] is the operator row of record i (-1: none; NULL:
 * record i is row i, the single-record LMM).  with_pe = 0 drops the permanent-environment
 * component.  K = Z Z^T / kinship_divisor: STCG divides by the reader's total SNP count,
 * monomorphic SNPs included (stcg_vce.cpp:86).  y (n_records) and X (n_records x p,
 * column-major) are host arrays.  Starting values, trace probes (one mt19937_64 stream),
 * EM warm-up, damped AI steps with clamps and the stopping rule follow the reference. */
int cs_vce_solve_stcg(cs_vce* vce, cs_kinship* op, double kinship_divisor,
                      const int32_t* rec_to_row, int64_t n_records, int with_pe, const double* y,
                      const double* X, int64_t p, const cs_vce_options* opt, cs_vce_result* res);
/* The final solution (stcg_vce.cpp:364-406): beta (p), genetic values a = sg2 K Zr^T P y and
 * permanent-environment effects spe2 Zr^T P y over all operator rows (host; NULL skips). */
int cs_vce_solution(const cs_vce* vce, double* beta, double* a_rows, double* pe_rows);
/* Per iteration: theta after the update (3), the log-likelihood and 1 for an AI step / 0 for
 * an EM step; 5 doubles per iteration (the reference's verbose history lines). */
int cs_vce_history(const cs_vce* vce, double* out, int64_t* n_iterations);
void cs_vce_destroy(cs_vce* vce);

/* Replaces the repeatability scan after the STCG null model (RepeatabilityModel::scanSTCG,
 * scan_stcg_with_grm, src/models/repeatability_scan_stcg.cpp:42-140) for SNPs
 * [snp_begin, snp_end) of g.  G: the q x q subject GRM (host, column-major; the reference's
 * G_subject_ or a LOCO G_loco), subject s is operator row subject_rows[s]; record i belongs to
 * subject obs_to_subject[i]; y (n_obs) and X (n_obs x p, column-major, host) are the records'
 * phenotype and fixed effects; vg / vpe / ve the null variance components.  Per SNP: the
 * record dosages centred on their mean (missing calls at -mean), skip when fewer than 10
 * records carry a call or the folded MAF < min_maf, score = g' P y, var = g' P g (skip below
 * 1e-15), P = erfc(|z| / sqrt 2), LOG10P as the reference.  maf receives the folded MAF (the
 * file's FREQ column).  Outputs have snp_end - snp_begin entries (NaN where tested = 0). */
int cs_stcg_scan(const cs_genotypes* g, const double* G, int64_t q, const int32_t* subject_rows,
                 const int32_t* obs_to_subject, int64_t n_obs, const double* y, const double* X,
                 int64_t p, double vg, double vpe, double ve, double min_maf, int64_t snp_begin,
                 int64_t snp_end, double* beta, double* se, double* pvalue, double* log10p,
                 double* maf, int32_t* tested);

/* Replaces MvLmmEngine::scan(PlinkReader, ...) (src/mvlmm_engine.cpp:756-931, processBlock
 * :210-396) for SNPs [snp_begin, snp_end) of g, with the null model of prepareFromVce
 * (:195-207): W (n x r eigenbasis, column-major), D (r), U'y (r x d), U'X (r x p), Vg and Ve
 * (d x d), all host arrays; keep lists the n analysed samples (rows of W).  Default options of
 * the reference (centred genotypes, LLT-based Sigma inverses, Wald = b' Schur b, df = d).
 * Per SNP o: beta[o*d ..] (d), cov[o*d*d ..] (the d x d Var(beta), may be NULL), wald,
 * pvalue, freq (mean dosage / 2 over observed kept samples), status = 0 OK,
 * 1 NUMERICAL_ROUNDOFF (covariance clipped), 2 BOUNDARY_SOLUTION, 3 TRUE_SINGULARITY (no
 * row written by the reference; outputs NaN).  precision selects the genotype rotation:
 * FP64 decode-GEMM or the int8 tensor-core projection. */
int cs_mvlmm_scan(const cs_genotypes* g, const int32_t* keep, int64_t n, const double* W,
                  int64_t r, const double* D, const double* Uty, int64_t d, const double* UtX,
                  int64_t p, const double* Vg, const double* Ve, int64_t snp_begin,
                  int64_t snp_end, int precision, double* beta, double* cov, double* wald,
                  double* pvalue, double* freq, int32_t* status);

/* ---------------------------------------------------------------- serving loop
 * No reference counterpart (the reference runs one job per process).  A server keeps the
 * packed genotypes resident and answers requests, each the matrix-free LMM job of
 * cs_lmm_prepare_lowrank_matrix_free + cs_lmm_scan on a cohort subset: low-rank sketch of the
 * subset's kinship, REML per trait, scan of a SNP window.  Kinship applies of all running
 * requests are stacked into one multi-right-hand-side apply whenever the GPU is free
 * (continuous batching; requests of different subset sizes share an apply through the full
 * sample space); requests are admitted FIFO as worker slots and the memory budget allow. */
typedef struct cs_server_options {
    int32_t rank;              /* low-rank basis size (--fastlmm-max-rank, 256) */
    int32_t oversample;        /* sketch oversampling (10) */
    double trace_threshold;    /* trace fraction for rank selection (0.95) */
    int32_t min_rank;          /* (1) */
    double min_maf;            /* scan MAF filter (0.01) */
    int32_t precision;         /* kinship applies and scan projection (CS_PRECISION_MIXED) */
    int64_t max_batch_columns; /* right-hand sides per stacked apply (4096) */
    double memory_budget_gb;   /* admission budget for request working sets in GB (0: the
                                  device's free memory at server creation less 4 GB) */
    int32_t max_active;        /* requests running at once (8) */
    double batch_window_ms;    /* after the first pending apply, wait up to this long (or until
                                  every running request waits on an apply) before stacking (0) */
    double subset_fraction;    /* cohorts smaller than this fraction of the resident samples get
                                  their own repacked subset operator instead of sharing the
                                  stacked full-space applies (0.5; 0: always stack) */
} cs_server_options;

typedef struct cs_serve_request {
    const int32_t* samples;  /* operator rows of the cohort subset (distinct), in y's order */
    int64_t n_samples;
    const double* Y;         /* n_samples x n_traits, column-major (host, copied) */
    int32_t n_traits;
    const double* X;         /* n_samples x p covariates, column-major (host, copied) */
    int32_t p;
    int64_t snp_begin, snp_end; /* scan window [begin, end) */
    uint64_t seed;           /* sketch seed (42) */
} cs_serve_request;

typedef struct cs_serve_status {
    int32_t state;           /* 0 queued, 1 running, 2 done, -1 failed */
    double latency_s;        /* submit -> done (-1 while not done) */
    double queue_s;          /* submit -> admitted (-1 while queued) */
    int32_t effective_rank;
} cs_serve_status;

typedef struct cs_server_statistics {
    int64_t submitted, completed, failed;
    double p50_s, p99_s, mean_s;   /* latency of completed requests */
    double throughput_rps, wall_s; /* completed / (last completion - first submit) */
    int64_t applies, apply_columns;
    int64_t max_requests_per_apply, max_concurrent;
    int64_t own_view_requests;     /* requests that ran on their own subset operator */
    double memory_budget_gb;       /* the admission budget in force */
} cs_server_statistics;

typedef struct cs_server cs_server;

void cs_server_default_options(cs_server_options* opt);
/* variants: the GRM variant selection (as for cs_kinship_create over all samples). */
int cs_server_create(const cs_genotypes* g, const int32_t* variants, int64_t n_variants,
                     const cs_server_options* opt, cs_server** out);
/* Copies the request's inputs and returns at once with its id. */
int cs_server_submit(cs_server* server, const cs_serve_request* request, int64_t* id);
/* Waits for a request (timeout_s < 0: without limit); a failed request returns CS_ERR_CUDA
 * with its message. */
int cs_server_wait(cs_server* server, int64_t id, double timeout_s, cs_serve_status* status);
/* One trait's results: sigma2 = (sigma2_g, sigma2_e); per-SNP arrays of the window length
 * (NaN where tested = 0, as cs_lmm_scan).  Any output may be NULL. */
int cs_server_result(cs_server* server, int64_t id, int32_t trait, double* sigma2, double* beta,
                     double* se, double* pvalue, double* log10p, double* freq, int32_t* tested);
/* Drops a finished request's results. */
int cs_server_release(cs_server* server, int64_t id);
int cs_server_stats(cs_server* server, cs_server_statistics* stats);
/* Finishes running requests, drops queued ones, frees the server. */
void cs_server_destroy(cs_server* server);

/* ---------------------------------------------------------------- result files
 * Writes association results the way GwasScanner::flushAssocResults writes `.assoc.txt`
 * (src/gwas_output.cpp:123-183, columns of src/gwas_output_schema.h:14-37): the unified
 * header, one additive row per SNP with a non-NaN P (and tested[j] != 0 when tested is not
 * NULL), NA in the six dominance / joint fields, numbers at the stream's default 6
 * significant digits.  CHR / SNP / BP / A1 / A2 come from bim_path (one line per SNP, in
 * the order of the result arrays); n_obs fills N.  stcg_columns = 1 writes the
 * `.stcg.assoc.txt` layout instead (CHR SNP BP A1 A2 FREQ N BETA SE P LOG10P,
 * src/models/repeatability_scan_stcg.cpp:190-193). */
int cs_write_assoc_txt(const char* out_path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                       const double* freq, const double* beta, const double* se,
                       const double* pvalue, const double* log10p, const int32_t* tested,
                       int stcg_columns);

/* Row layouts of cs_write_assoc: the unified `.assoc.txt`, `.stcg.assoc.txt`, and the
 * GWAS-SSF form of `--out-ssf` (src/gwas_output.cpp:81-82 header, :149-153 rows: chromosome,
 * base_pair_location, effect_allele = A1, other_allele = A2, effect_allele_frequency,
 * sample_size, beta, standard_error, p_value, variant_id). */
enum { CS_ASSOC_UNIFIED = 0, CS_ASSOC_STCG = 1, CS_ASSOC_SSF = 2 };
/* cs_write_assoc_txt with a layout, a row order and `--out-gz` (gzip != 0): the same text
 * through zlib's gz writer as src/gzip_writer.cpp:12-55 opens it ("wb" +
 * Z_DEFAULT_COMPRESSION, which zlib reads as level 1); the file name is the caller's (the
 * reference keeps `.assoc.txt`).  order (NULL: .bim order) lists the SNP indices in the order
 * their rows are written, each at most once — the reference writes the LOCO scan's rows
 * chromosome by chromosome (src/gwas_scanner.cpp:449, 499). */
int cs_write_assoc(const char* out_path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                   const double* freq, const double* beta, const double* se, const double* pvalue,
                   const double* log10p, const int32_t* tested, const int64_t* order,
                   int64_t n_order, int layout, int gzip);
/* `OUT.cosmic.sumstats` as GwasScanner::appendCosmicSumstats writes it
 * (src/gwas_output.cpp:186-234): append = 0 replaces the file and writes the comment header
 * (version 1.0, "# Created: <created>" — NULL gives the current UTC time as
 * "%Y-%m-%d %H:%M:%S UTC" — and "# Model: <model>" when model is not empty) and the column
 * header; append = 1 adds rows only (the reference's later chromosomes; with gzip a new
 * member).  One row per SNP with a non-NaN P and tested[j] != 0: BETA / SE / P at 10
 * significant digits, AF / LOG10P / Z = BETA/SE / WEIGHT = 1/SE^2 at 6, INFO 1, WARNING ".". */
int cs_append_cosmic_sumstats(const char* path, const char* bim_path, int64_t n_snps,
                              int32_t n_obs, const double* freq, const double* beta,
                              const double* se, const double* pvalue, const double* log10p,
                              const int32_t* tested, const char* model, int append, int gzip,
                              const char* created);

/* `.assoc.mv.txt` of the multivariate model (src/models/multivariate_model.cpp:943-951,
 * src/models/multivariate_output.cpp:40-70) from cs_mvlmm_scan outputs: per SNP freq, wald,
 * p, beta (d), cov (d x d); rows with NaN P are skipped; SE_t = sqrt(cov[t][t]). */
int cs_write_assoc_mv_txt(const char* out_path, const char* bim_path, int64_t n_snps, int32_t d,
                          const double* freq, const double* wald, const double* pvalue,
                          const double* beta, const double* cov);

/* Run metadata of the matrix-free low-rank LMM, as src/gwas_scanner.cpp writes them:
 *   cs_write_scan_meta        OUT.scan.meta.txt (:93-108) for `--fastlmm
 *                             --fastlmm-matrix-free` with default scan tier, additive model and
 *                             no HWE filter; requested_rank = --fastlmm-max-rank
 *   cs_write_low_rank_meta    OUT.low_rank.meta.tsv header (:109-115) and one row per null
 *                             model (:409-428): scope "GLOBAL" or the LOCO chromosome, the
 *                             diagnostics of cs_lmm_prepare_lowrank_matrix_free, the analysed
 *                             sample count n, --lmm-low-rank-error-tol and per row the fallback
 *                             label (NULL: "none", as with --fastlmm-no-fallback;
 *                             "trace_threshold" / "error_tolerance" when the run fell
 *                             back, src/gwas_scanner.cpp:347-362).  Like the reference's
 *                             matrix-free engine (src/lmm_engine.cpp:1077-1094), REQUESTED_RANK
 *                             reports the selected rank. */
int cs_write_scan_meta(const char* out_prefix, int32_t requested_rank, double trace_threshold);
/* The same file for the dense route (`--model lmm` without --fastlmm / --lmm-low-rank):
 * matrix_approximation full_eigen, requested_rank 0, trace_threshold 0, RANK_SELECTION FULL;
 * the reference writes no .low_rank.meta.tsv there. */
int cs_write_scan_meta_full_eigen(const char* out_prefix);
/* The lines appended to OUT.scan.meta.txt after the scan (gwas_output::appendCommonMetadata,
 * src/gwas_output_schema.h:57-73, called from src/gwas_scanner.cpp:507-509): MODEL ("additive"),
 * N (analysed samples), the N / FREQ semantics, LOCO, COVARIATE_PROJECTION and VCE_CONVERGED
 * (every null model converged; the low-rank route's REML either converges or fails). */
int cs_append_scan_common_meta(const char* out_prefix, const char* model, int64_t n, int loco,
                               int covariate_projection, int vce_converged);
int cs_write_low_rank_meta(const char* out_prefix, int32_t n_rows, const char* const* scopes,
                           const cs_lowrank_diagnostics* diags, int64_t n, double error_tol,
                           const char* const* fallbacks);

/* ---------------------------------------------------------------- input side
 * The samples, phenotypes, covariates and keep list that the reference's association path
 * builds before the engines run, with its parsing rules:
 *   cs_fam_read           PlinkReader::readFam (libCosmicCore/src/plink_reader.cpp:34-48)
 *   cs_pheno_load         PhenoReader::load (libCosmicCore/src/pheno_reader.cpp:13-61):
 *                         column col_idx (1-based, after FID IID), missing code within 1e-6
 *                         and NA / na / NaN / nan / NAN -> NaN
 *   cs_pheno_align        PhenoReader::align (:138-187): y in .fam order (NaN unmatched);
 *                         a constant trait (>= 2 finite values) -> CS_ERR_INVALID_ARGUMENT
 *                         with the reference's message
 *   cs_pheno_load_matrix  PhenoReader::loadMatrix (:63-125), cols 1-based (NULL = all)
 *   cs_pheno_align_matrix PhenoReader::alignMatrix (:189-215): Y n x traits, column-major
 *   cs_covar_load         CovarReader::load (libCosmicCore/src/covar_reader.cpp:19-62):
 *                         quantitative covariates as float, missing code within 1e-8 -> NaN
 *   cs_covar_load_categorical  CovarReader::loadCategorical (:64-176): k levels -> k - 1
 *                         dummy columns, the alphabetically first level the reference
 *   cs_covar_align        CovarReader::align (:468-500): X n x p float, column-major
 *   cs_filter_samples     DataFilter::filterSamples (libCosmicCore/src/data_filter.h:21-41):
 *                         the rows whose y and covariates are all non-NaN, ascending
 * Counts and matched numbers come back through out-parameters; tables are freed by their
 * destroy call. */
typedef struct cs_samples cs_samples;
typedef struct cs_pheno cs_pheno;
typedef struct cs_covar cs_covar;
int cs_fam_read(const char* fam_path, cs_samples** out);
int cs_samples_count(const cs_samples* s, int64_t* n);
/* FID and IID of sample i, NUL-terminated, truncated to the buffer sizes */
int cs_samples_id(const cs_samples* s, int64_t i, char* fid, size_t fid_len, char* iid, size_t iid_len);
/* the .fam phenotype column (the reference uses it when no phenotype file is given) */
int cs_samples_fam_phenotype(const cs_samples* s, double* y);
void cs_samples_destroy(cs_samples* s);
int cs_pheno_load(const char* path, int32_t col_idx, double missing_code, cs_pheno** out);
int cs_pheno_load_matrix(const char* path, const int32_t* cols, int32_t n_cols, double missing_code,
                         cs_pheno** out);
int cs_pheno_traits(const cs_pheno* p, int32_t* n_traits);
int cs_pheno_align(const cs_pheno* p, const cs_samples* s, double* y, int64_t* matched);
int cs_pheno_align_matrix(const cs_pheno* p, const cs_samples* s, double* Y, int64_t ldy,
                          int64_t* matched);
void cs_pheno_destroy(cs_pheno* p);
int cs_covar_load(const char* path, double missing_code, cs_covar** out);
int cs_covar_load_categorical(const char* path, const char* missing_token, cs_covar** out);
int cs_covar_columns(const cs_covar* c, int32_t* p);
int cs_covar_align(const cs_covar* c, const cs_samples* s, float* X, int64_t ldx, int64_t* matched);
void cs_covar_destroy(cs_covar* c);
int cs_filter_samples(const double* y, int64_t n, const float* X, int64_t ldx, int32_t p,
                      int32_t* keep, int64_t* n_keep);

/* ---------------------------------------------------------------- instrumentation
 * No reference counterpart beyond the stage timers of src/gwas_scanner.cpp:42-49 and
 * PlinkKinshipOperator::BlockProfile (src/kinship_operator.h:55-63): a process-wide count
 * of the library's kernel launches, and optional CUDA-event timing per kernel name with
 * the algorithmic FLOPs / bytes of each launch.  Enabling resets the records; the summary
 * (JSON) synchronises the device. */
int cs_profile_enable(int on);
int cs_profile_summary(char* buf, size_t len, size_t* needed);
int cs_launch_count(int64_t* count);

#ifdef __cplusplus
}
#endif
