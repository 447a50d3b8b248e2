/*
 * CPU oracle for the matrix-free mixed-model path — TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain loops over FP64, the reference CosmicScanner
 * algorithms that the CUDA library replaces.  It exists so the tests (and the
 * CPU-baseline leg of bench.py) can check the GPU results on the same inputs.
 * Nothing in the product links or calls it.
 *
 * Parity status: the kinship-operator restatement is pinned against the
 * reference's own known-answer recipe (tests/test_kinship_batch.cpp: dense
 * Z Z^T / M within 1e-10, trace, empty RHS, bad dimensions), regenerated here
 * byte-for-byte from the same mt19937_64 seed.  The sketch / REML / scan
 * restatements have no golden outputs in the reference (Eigen is not available
 * in this container, so the reference cannot be built): parity unpinned for
 * those, beyond agreement with an independent dense FP64 computation.
 *
 * Matrices are column-major with explicit leading dimensions, like Eigen's
 * default storage in the reference.  `bed` always points at the first SNP row
 * (the 3 magic bytes already skipped); row j starts at bed + j*stride.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* libCosmicCore/src/plink_reader.cpp:187-239 (PlinkReader::computeStats). */
void orc_compute_stats(const uint8_t* bed, int64_t n_samples, int64_t n_snps, int64_t stride,
                       double* mean, double* inv_std, int32_t* count, double* sum);

/* src/kinship_operator.cpp:74-218: multiplyZt + multiplyZ + scaling (vector apply).
 * keep == NULL means all samples; variants == NULL means all SNPs.
 * n_threads reproduces the per-worker buffers reduced in worker order. */
int orc_kinship_apply_vector(const uint8_t* bed, int64_t n_fam, int64_t stride,
                             const double* mean, const double* inv_std,
                             const int32_t* keep, int64_t n_keep,
                             const int32_t* variants, int64_t n_var,
                             const double* v, double* out, int n_threads);

/* src/kinship_operator.cpp:225-302 (apply_block): 512-SNP decode to FP64 z, z^T X, z*proj. */
int orc_kinship_apply_block(const uint8_t* bed, int64_t n_fam, int64_t stride,
                            const double* mean, const double* inv_std,
                            const int32_t* keep, int64_t n_keep,
                            const int32_t* variants, int64_t n_var,
                            const double* X, int64_t ldx, int64_t k,
                            double* out, int64_t ldo, int n_threads);

/* src/kinship_operator.cpp:306-368 */
double orc_kinship_trace(const uint8_t* bed, int64_t n_fam, int64_t stride,
                         const double* mean, const double* inv_std,
                         const int32_t* keep, int64_t n_keep,
                         const int32_t* variants, int64_t n_var);
void orc_kinship_diagonal(const uint8_t* bed, int64_t n_fam, int64_t stride,
                          const double* mean, const double* inv_std,
                          const int32_t* keep, int64_t n_keep,
                          const int32_t* variants, int64_t n_var, double* diag);

/* Dense Z (rows x numVariants, column-major) exactly as tests/test_kinship_batch.cpp:61-72
 * builds it from float dosages: z = (dosage - mean) * inv_std, NaN -> 0. */
void orc_dense_z(const uint8_t* bed, int64_t n_fam, int64_t stride,
                 const double* mean, const double* inv_std,
                 const int32_t* keep, int64_t n_keep,
                 const int32_t* variants, int64_t n_var, double* z, int64_t ldz);

/* The fixture of tests/test_kinship_batch.cpp:26-43: writes 3 + m*ceil(n/4) BED bytes
 * (magic included) into bed_out, drawn from mt19937_64(seed); then continues the SAME
 * engine to draw the omega matrices of the test's loop (:47-80): for each of the
 * n_sel selections with rows[s] rows, for each width in widths[0..n_widths), a fresh
 * std::normal_distribution draws width*rows values column by column.  Writes them
 * consecutively to omega_out (may be NULL to skip). */
void orc_kinship_batch_fixture(int n, int m, uint64_t seed, uint8_t* bed_out,
                               int n_sel, const int32_t* rows, int n_widths,
                               const int32_t* widths, double* omega_out);

/* n*cols standard normals from mt19937_64(seed) and one std::normal_distribution<double>,
 * filled column by column (src/lmm_engine.cpp:917-922). */
void orc_normal_matrix(uint64_t seed, int64_t n, int64_t cols, double* out);

/* src/genetics/genotype_encoding.h:33-81, additive model, HWE disabled.
 * raw: n values, NaN = missing.  Writes centred values; returns passes_maf. */
int orc_prepare_marker(const double* raw, int64_t n, double min_maf, double* values,
                       double* freq, int32_t* observed);

/* src/lmm_engine.cpp:22-64 */
double orc_chisq_prob(double stat, int df);

/* Low-rank matrix-free null model, src/lmm_engine.cpp:897-1095.
 * Inputs: the operator's selection, y (n), X (n x p, column-major, already FP32-rounded
 * by the caller when mirroring the reference's MatrixXf covariates).
 * Outputs: U (n x rank_out, ld n; caller provides n*rank), lambda (rank), scalars. */
typedef struct {
    int32_t rank;            /* selected rank */
    int32_t sketch_size;
    double residual_eigenvalue;
    double relative_frobenius_error;
    double trace;
    double trace_fraction;
    int32_t trace_threshold_met;
    double sigma2_g, sigma2_e, delta, best_log_eta, best_objective;
} orc_lowrank_result;

int orc_lowrank_prepare(const uint8_t* bed, int64_t n_fam, int64_t stride,
                        const double* mean, const double* inv_std,
                        const int32_t* keep, int64_t n_keep,
                        const int32_t* variants, int64_t n_var,
                        const double* y, const double* X, int64_t p,
                        int rank, int oversample, uint64_t seed,
                        double trace_threshold, int min_rank, int n_threads,
                        double* U_out, double* lambda_out, orc_lowrank_result* res);

/* Low-rank REML search only (grid + golden), given a basis: src/lmm_engine.cpp:1010-1073. */
int orc_lowrank_reml(const double* U, const double* lambda, int64_t n, int64_t rank, double r0,
                     const double* y, const double* X, int64_t p, orc_lowrank_result* res);

/* src/lmm_engine.cpp:1269-1361 (scanLowRank) for all SNPs of the reader, no chromosome
 * filter.  keep lists the analysed samples (n entries).  Per-SNP outputs (n_snps each);
 * tested[j] = 1 when the SNP produced a row. */
int orc_scan_lowrank(const uint8_t* bed, int64_t n_fam, int64_t stride, int64_t n_snps,
                     const int32_t* keep, int64_t n,
                     const double* U, const double* lambda, int64_t rank, double r0,
                     double sigma2_g, double sigma2_e,
                     const double* y, const double* X, int64_t p, double min_maf,
                     double* beta, double* se, double* pval, double* log10p,
                     double* freq, int32_t* tested);

/* libCosmicCore/src/matrix_free_pcg.h:20-68 on the operator A = sg2*K + se2*I with the
 * scalar preconditioner 1/(sg2+se2); absolute stopping ||r|| < tol.  Returns iterations. */
int orc_pcg_solve(const uint8_t* bed, int64_t n_fam, int64_t stride,
                  const double* mean, const double* inv_std,
                  const int32_t* keep, int64_t n_keep,
                  const int32_t* variants, int64_t n_var,
                  double sg2, double se2, const double* b, double tol, int max_iter,
                  double* x);

/* libCosmicCore/src/stcg_vce.cpp:157-407 (STCG_VCE::solve): matrix-free AI-REML with
 * theta = (sigma2_g, sigma2_pe, sigma2_e), V = sg2 Zr (Z Z^T / n_snps) Zr^T + spe2 Zr Zr^T
 * + se2 I over records.  The genotype operator is PlinkReader::multiply_Zt_v/multiply_Z_v
 * over every SNP of the reader (plink_reader.cpp:241-402), scaled by the SNP count.
 * rec_to_ind[i] is the genotype row of record i (NULL: record i is row i).  with_pe = 0
 * drops the permanent-environment component (the single-record LMM).  Probes: one
 * mt19937_64(probe_seed) stream with uniform_int_distribution<int>(0, 1).  SLQ is the
 * estimator's one-thread schedule (seed 42 + iteration).  Outputs: beta (p), the genetic
 * BLUP a = sg2 K gather(Py) and pe = spe2 gather(Py) over all n_fam rows. */
typedef struct {
    int32_t max_iter;
    double tol;
    int32_t mc_samples;
    double pcg_tol;
    int32_t pcg_max_iter;
    int32_t slq_probes;
    int32_t slq_steps;
    uint64_t probe_seed;
} orc_stcg_options;

typedef struct {
    double sigma2_g, sigma2_pe, sigma2_e, logl;
    int32_t iterations, converged;
    int64_t pcg_iterations;
} orc_stcg_result;

int orc_stcg_vce(const uint8_t* bed, int64_t n_fam, int64_t stride, int64_t n_snps,
                 const double* mean, const double* inv_std, const int32_t* rec_to_ind,
                 int64_t n_rec, int with_pe, const double* y, const double* X, int64_t p,
                 const orc_stcg_options* opt, orc_stcg_result* res, double* beta_out,
                 double* a_ind_out, double* pe_ind_out);

/* orc_stcg_vce with the kinship operator given as a dense K = Z Z^T / M (n_fam x n_fam,
 * column-major), each application one matrix-vector product. */
int orc_stcg_vce_dense(const double* K, int64_t n_fam, const int32_t* rec_to_ind, int64_t n_rec,
                       int with_pe, const double* y, const double* X, int64_t p,
                       const orc_stcg_options* opt, orc_stcg_result* res, double* beta_out,
                       double* a_ind_out, double* pe_ind_out);

/* src/models/repeatability_scan_stcg.cpp:42-140 (scan_stcg_with_grm) with a given q x q
 * subject GRM G (column-major) for SNPs [snp_begin, snp_end); maf_out = folded MAF. */
int orc_stcg_scan(const uint8_t* bed, int64_t n_fam, int64_t stride, const double* G, int64_t q,
                  const int32_t* subject_rows, const int32_t* obs_to_subject, int64_t n_obs,
                  const double* y, const double* X, int64_t p, double vg, double vpe, double ve,
                  double min_maf, int64_t snp_begin, int64_t snp_end, double* beta, double* se,
                  double* pval, double* log10p, double* maf_out, int32_t* tested);

/* src/mvlmm_engine.cpp:756-931 (MvLmmEngine::scan(PlinkReader)) with processBlock :210-396
 * and the checks of src/mvlmm_numerics.h, default options, for SNPs [snp_begin, snp_end). */
int orc_mvlmm_scan(const uint8_t* bed, int64_t n_fam, int64_t stride, const int32_t* keep,
                   int64_t n, const double* W, int64_t r, const double* Dv, const double* Uty,
                   int64_t d, const double* UtX, int64_t p, const double* Vg, const double* Ve,
                   int64_t snp_begin, int64_t snp_end, double* beta, double* cov, double* wald,
                   double* pvalue, double* freq, int32_t* status);

/* Helpers of the timed CPU restatement of the whole low-rank job (bench.py's CPU legs), every
 * sample in .fam order, OpenMP over SNPs:
 *  - orc_decode_z_cols: columns snps[0..count) of Z (n x count, ld ldz) with the decode
 *    values of src/kinship_operator.cpp:276-283 ({(2-mu)s, 0, (1-mu)s, -mu s});
 *  - orc_scan_encode_cols: genetics::prepareAssociationMarker (src/genetics/genotype_encoding.h:
 *    33-81) for SNPs first..first+count-1: mean-imputed, centred dosages, A1 frequency, pass
 *    flag and the column's sum of squares;
 *  - orc_chisq_prob_vec: chisq_prob (src/lmm_engine.cpp:22-64) over an array. */
void orc_decode_z_cols(const uint8_t* bed, int64_t stride, const double* mean,
                       const double* inv_std, const int32_t* snps, int64_t count, int64_t n,
                       double* z, int64_t ldz, int n_threads);
void orc_scan_encode_cols(const uint8_t* bed, int64_t stride, int64_t first, int64_t count,
                          int64_t n, double min_maf, double* g, int64_t ldg, double* freq,
                          int32_t* pass, double* gsq, int n_threads);
void orc_chisq_prob_vec(const double* stat, int64_t count, int df, double* out, int n_threads);

/* Rademacher probes from std::mt19937_64(seed) + uniform_int_distribution<int>(0, 1) after
 * `skip` draws: n x cols column-major, column by column. */
void orc_rademacher(uint64_t seed, int64_t skip, int64_t n, int64_t cols, double* out);

#ifdef __cplusplus
}
#endif
