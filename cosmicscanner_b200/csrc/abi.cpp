// C ABI: status codes + thread-local error text around the C++ implementation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "cs_internal.h"
#include "dense_internal.h"
#include "input_internal.h"

namespace cs {
cs_genotypes* genotypes_from_bed(const uint8_t* bed, size_t n_bytes, int64_t n_samples,
                                 int64_t n_snps);
cs_genotypes* genotypes_open_plink(const std::string& prefix);
cs_kinship* kinship_create(const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                           const int32_t* variants, int64_t n_var);
void kinship_apply_colmajor(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                            int64_t ldy, int precision, cudaStream_t s);
void kinship_diagonal(cs_kinship* op, double* diag_host);
void kinship_apply_noalloc(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                           int64_t ldy, cudaStream_t s);
cs_lmm* lmm_create();
void lmm_destroy(cs_lmm* l);
void kinship_apply_f32(cs_kinship* op, const float* X, int64_t ldx, int64_t k, float* Y,
                       int64_t ldy, int precision, cudaStream_t s);
cs_grm* grm_create(const cs_genotypes* g, const int32_t* variants, int64_t n_variants,
                   const cs_grm_options* opt);
cs_grm* grm_from_host(int64_t n, const double* G, int64_t ldg);
cs_grm* grm_loco(const cs_grm* global, const cs_grm* chrom);
void grm_copy(const cs_grm* grm, const int32_t* keep, int64_t n_keep, double* out, int64_t ld);
cs_eigen_vce* eigen_prepare(const cs_grm* grm, const int32_t* keep, int64_t n_keep,
                            const double* y, const double* X, int64_t p, bool projection);
void eigen_run_null(cs_eigen_vce* v, cs_eigen_vce_result* out);
void eigen_get(const cs_eigen_vce* v, double* D, double* Uty, double* UtX, double* W, int64_t ldw);
void lmm_prepare_from_vce(cs_lmm* l, const cs_eigen_vce* v, bool use_residuals);
cs_mv_eigen_vce* mv_prepare(const cs_grm* grm, const int32_t* keep, int64_t n_keep,
                            const double* Y, int64_t d, const double* X, int64_t p,
                            bool projection);
bool mv_run_null(cs_mv_eigen_vce* v, const cs_mv_vce_options* opt);
void mv_get(const cs_mv_eigen_vce* v, double* Vg, double* Ve, double* Vg_se, double* Ve_se,
            double* D, double* Uty);
void mv_scan(const cs_genotypes* g, const int32_t* keep, int64_t n_keep, const cs_mv_eigen_vce* v,
             int64_t snp_begin, int64_t snp_end, int precision, double* beta, double* cov,
             double* wald, double* pvalue, double* freq, int32_t* status);
void lmm_prepare_lowrank(cs_lmm* lmm, cs_kinship* op, const double* y, const double* X, int64_t p,
                         int rank, int oversample, int64_t seed, double trace_threshold,
                         int min_rank, int precision, cs_lowrank_diagnostics* diag);
void lmm_lowrank_basis(const cs_lmm* lmm, double* U, int64_t ldu, double* lambda);
void lmm_scan(cs_lmm* lmm, const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
              double min_maf, int precision, double* beta, double* se, double* pvalue,
              double* log10p, double* freq, int32_t* tested);
void vce_default_options(cs_vce_options* o);
cs_vce* vce_create();
void vce_destroy(cs_vce* v);
void vce_solve_stcg(cs_vce* v, cs_kinship* op, double divisor, const int32_t* rec_to_row,
                    int64_t n_rec, int with_pe, const double* y, const double* X, int64_t p,
                    const cs_vce_options* opt, cs_vce_result* res);
void vce_solution(const cs_vce* v, double* beta, double* a_rows, double* pe_rows);
void vce_history(const cs_vce* v, double* out, int64_t* n_iter);
void pcg_solve_public(cs_kinship* op, double divisor, double sg2, double se2, const double* B,
                      int64_t ldb, int64_t k, double* X, int64_t ldx, double tol, int relative,
                      int max_iter, int precision, int32_t* iterations, cudaStream_t s);
void pcg_solve_records_public(cs_kinship* op, double divisor, const int32_t* rec_to_row,
                              int64_t n_rec, bool with_pe, double sg2, double spe2, double se2,
                              const double* B, int64_t ldb, int64_t k, double* X, int64_t ldx,
                              double tol, int relative, int max_iter, int precision,
                              int32_t* iterations, cudaStream_t s);
void mv_stcg_default_options(cs_mv_stcg_options* o);
void mv_stcg_solve(cs_kinship* op, double divisor, const double* Y, int32_t d, const double* X,
                   int64_t p, const cs_mv_stcg_options* opt, double* Vg, double* Ve,
                   cs_mv_stcg_result* res);
void genotype_multiply_zt(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* U,
                          int64_t ldu, int precision, cudaStream_t s);
void genotype_multiply_z(cs_kinship* op, const double* V, int64_t ldv, int64_t k, double* Y,
                         int64_t ldy, int precision, cudaStream_t s);
void stcg_scan(const cs_genotypes* g, const double* G, int64_t q, const int32_t* subject_rows,
               const int32_t* obs_to_subject, int64_t n_obs, const double* y, const double* X,
               int64_t p, double vg, double vpe, double ve, double min_maf, int64_t snp_begin,
               int64_t snp_end, double* beta, double* se, double* pvalue, double* log10p,
               double* maf, int32_t* tested);
void mvlmm_scan(const cs_genotypes* g, const int32_t* keep, int64_t n, const double* Wp, int64_t r,
                const double* Dv, const double* Uty, int64_t d, const double* UtX, int64_t p,
                const double* Vg, const double* Ve, int64_t snp_begin, int64_t snp_end,
                int precision, double* beta, double* cov, double* wald, double* pvalue,
                double* freq, int32_t* status);
void server_default_options(cs_server_options* o);
cs_server* server_create(const cs_genotypes* g, const int32_t* variants, int64_t n_var,
                         const cs_server_options* opt);
int64_t server_submit(cs_server* sv, const cs_serve_request* q);
void server_wait(cs_server* sv, int64_t id, double timeout_s, cs_serve_status* out);
void server_result(cs_server* sv, int64_t id, int32_t trait, double* sigma2, double* beta,
                   double* se, double* pval, double* log10p, double* freq, int32_t* tested);
void server_release(cs_server* sv, int64_t id);
void server_stats(cs_server* sv, cs_server_statistics* out);
void server_destroy(cs_server* sv);
void write_assoc_mv_txt(const char* out_path, const char* bim_path, int64_t n_snps, int32_t d,
                        const double* freq, const double* wald, const double* p, const double* beta,
                        const double* cov);
void write_scan_meta(const char* out_prefix, int32_t requested_rank, double trace_threshold,
                     bool full_eigen);
void write_low_rank_meta(const char* out_prefix, int32_t n_rows, const char* const* scopes,
                         const cs_lowrank_diagnostics* diags, int64_t n, double error_tol,
                         const char* const* fallbacks);
void write_assoc_txt(const char* out_path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                     const double* freq, const double* beta, const double* se, const double* p,
                     const double* log10p, const int32_t* tested, int stcg_columns);
void write_assoc(const char* out_path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                 const double* freq, const double* beta, const double* se, const double* p,
                 const double* log10p, const int32_t* tested, const int64_t* order,
                 int64_t n_order, int layout, bool gzip);
void append_cosmic_sumstats(const char* path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                            const double* freq, const double* beta, const double* se,
                            const double* p, const double* log10p, const int32_t* tested,
                            const char* model, bool append, bool gzip, const char* created);
void append_scan_common_meta(const char* out_prefix, const char* model, int64_t n, bool loco,
                             bool covariate_projection, bool vce_converged);
}  // namespace cs

namespace {
thread_local std::string g_last_error;

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return CS_OK;
    } catch (const cs::Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return CS_ERR_INVALID_ARGUMENT;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return CS_ERR_INVALID_ARGUMENT;
    }
}

void require(bool ok, const char* msg) {
    if (!ok) cs::fail(CS_ERR_INVALID_ARGUMENT, msg);
}
}  // namespace

namespace cs {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace cs

extern "C" {

const char* cs_last_error(void) { return g_last_error.c_str(); }
const char* cs_version(void) { return "cosmicscanner_b200 0.1.0 (sm_100a)"; }

int cs_genotypes_create(const uint8_t* bed_bytes, size_t n_bytes, int64_t n_samples,
                        int64_t n_snps, cs_genotypes** out) {
    return guarded([&] {
        require(out != nullptr, "null output handle");
        *out = cs::genotypes_from_bed(bed_bytes, n_bytes, n_samples, n_snps);
    });
}

int cs_genotypes_open_plink(const char* prefix, cs_genotypes** out) {
    return guarded([&] {
        require(out != nullptr && prefix != nullptr, "null argument");
        *out = cs::genotypes_open_plink(prefix);
    });
}

int cs_genotypes_info(const cs_genotypes* g, int64_t* n_samples, int64_t* n_snps,
                      int64_t* bytes_per_snp) {
    return guarded([&] {
        require(g != nullptr, "null genotypes handle");
        if (n_samples) *n_samples = g->n_samples;
        if (n_snps) *n_snps = g->n_snps;
        if (bytes_per_snp) *bytes_per_snp = g->bytes_per_snp;
    });
}

int cs_genotypes_stats(const cs_genotypes* g, double* mean, double* inv_std, int32_t* count,
                       double* sum) {
    return guarded([&] {
        require(g != nullptr, "null genotypes handle");
        const size_t M = (size_t)g->n_snps;
        if (mean) std::memcpy(mean, g->mean.data(), M * 8);
        if (inv_std) std::memcpy(inv_std, g->inv_std.data(), M * 8);
        if (count) std::memcpy(count, g->count.data(), M * 4);
        if (sum) std::memcpy(sum, g->sum.data(), M * 8);
    });
}

void cs_genotypes_destroy(cs_genotypes* g) { delete g; }

int cs_kinship_create(const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                      const int32_t* variants, int64_t n_variants, cs_kinship** out) {
    return guarded([&] {
        require(out != nullptr, "null output handle");
        *out = cs::kinship_create(g, keep, n_keep, variants, n_variants);
    });
}

int cs_kinship_info(const cs_kinship* op, int64_t* rows, int64_t* num_variants) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        if (rows) *rows = op->rows;
        if (num_variants) *num_variants = op->num_variants;
    });
}

int cs_kinship_apply(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                     int64_t ldy, int precision, void* stream) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        cs::kinship_apply_colmajor(op, X, ldx, k, Y, ldy, precision, (cudaStream_t)stream);
    });
}

int cs_kinship_apply_f32(cs_kinship* op, const float* X, int64_t ldx, int64_t k, float* Y,
                         int64_t ldy, int precision, void* stream) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        cs::kinship_apply_f32(op, X, ldx, k, Y, ldy, precision, (cudaStream_t)stream);
    });
}

int cs_kinship_apply_host(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                          int64_t ldy, int precision) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        if (k < 0) cs::fail(CS_ERR_INVALID_ARGUMENT, "negative column count");
        if (ldx < op->rows || ldy < op->rows)
            cs::fail(CS_ERR_INVALID_ARGUMENT, "PlinkKinshipOperator::apply: dimension mismatch");
        if (k == 0) return;
        const int64_t n = op->rows;
        cs::DeviceBuffer<double> dx;
        dx.resize(n * k);
        CS_CUDA(cudaMemcpy2D(dx.get(), n * 8, X, ldx * 8, n * 8, k, cudaMemcpyHostToDevice));
        cs::kinship_apply_colmajor(op, dx.get(), n, k, dx.get(), n, precision, 0);
        CS_CUDA(cudaMemcpy2D(Y, ldy * 8, dx.get(), n * 8, n * 8, k, cudaMemcpyDeviceToHost));
    });
}

int cs_kinship_apply_noalloc(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                             int64_t ldy, void* stream) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        cs::kinship_apply_noalloc(op, X, ldx, k, Y, ldy, (cudaStream_t)stream);
    });
}

int cs_genotype_multiply_zt(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* U,
                            int64_t ldu, int precision, void* stream) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        cs::genotype_multiply_zt(op, X, ldx, k, U, ldu, precision, (cudaStream_t)stream);
    });
}

int cs_genotype_multiply_z(cs_kinship* op, const double* V, int64_t ldv, int64_t k, double* Y,
                           int64_t ldy, int precision, void* stream) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        cs::genotype_multiply_z(op, V, ldv, k, Y, ldy, precision, (cudaStream_t)stream);
    });
}

int cs_genotype_multiply_zt_host(cs_kinship* op, const double* X, int64_t ldx, int64_t k,
                                 double* U, int64_t ldu, int precision) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        if (k < 0) cs::fail(CS_ERR_INVALID_ARGUMENT, "negative column count");
        if (ldx < op->rows || ldu < op->num_variants)
            cs::fail(CS_ERR_INVALID_ARGUMENT, "Dimension mismatch in multiply_Zt_v");
        if (k == 0) return;
        const int64_t n = op->rows, nv = op->num_variants;
        cs::DeviceBuffer<double> dx, du;
        dx.resize(n * k);
        du.resize(nv * k);
        CS_CUDA(cudaMemcpy2D(dx.get(), n * 8, X, ldx * 8, n * 8, k, cudaMemcpyHostToDevice));
        cs::genotype_multiply_zt(op, dx.get(), n, k, du.get(), nv, precision, 0);
        CS_CUDA(cudaMemcpy2D(U, ldu * 8, du.get(), nv * 8, nv * 8, k, cudaMemcpyDeviceToHost));
    });
}

int cs_genotype_multiply_z_host(cs_kinship* op, const double* V, int64_t ldv, int64_t k,
                                double* Y, int64_t ldy, int precision) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        if (k < 0) cs::fail(CS_ERR_INVALID_ARGUMENT, "negative column count");
        if (ldv < op->num_variants || ldy < op->rows)
            cs::fail(CS_ERR_INVALID_ARGUMENT, "Dimension mismatch in multiply_Z_v");
        if (k == 0) return;
        const int64_t n = op->rows, nv = op->num_variants;
        cs::DeviceBuffer<double> dv, dy;
        dv.resize(nv * k);
        dy.resize(n * k);
        CS_CUDA(cudaMemcpy2D(dv.get(), nv * 8, V, ldv * 8, nv * 8, k, cudaMemcpyHostToDevice));
        cs::genotype_multiply_z(op, dv.get(), nv, k, dy.get(), n, precision, 0);
        CS_CUDA(cudaMemcpy2D(Y, ldy * 8, dy.get(), n * 8, n * 8, k, cudaMemcpyDeviceToHost));
    });
}

int cs_kinship_trace(const cs_kinship* op, double* trace) {
    return guarded([&] {
        require(op != nullptr && trace != nullptr, "null argument");
        *trace = op->trace;
    });
}

int cs_kinship_diagonal(cs_kinship* op, double* diag) {
    return guarded([&] {
        require(op != nullptr && diag != nullptr, "null argument");
        cs::kinship_diagonal(op, diag);
    });
}

void cs_kinship_destroy(cs_kinship* op) { delete op; }

int cs_lmm_create(cs_lmm** out) {
    return guarded([&] {
        require(out != nullptr, "null output handle");
        *out = cs::lmm_create();
    });
}

int cs_lmm_prepare_lowrank_matrix_free(cs_lmm* lmm, cs_kinship* op, const double* y,
                                       const double* X, int64_t p, int rank, int oversample,
                                       int64_t seed, double trace_threshold, int min_rank,
                                       int precision, cs_lowrank_diagnostics* diag) {
    return guarded([&] {
        require(lmm != nullptr && op != nullptr && y != nullptr, "null argument");
        cs::lmm_prepare_lowrank(lmm, op, y, X, p, rank, oversample, seed, trace_threshold,
                                min_rank, precision, diag);
    });
}

int cs_lmm_lowrank_basis(const cs_lmm* lmm, double* U, int64_t ldu, double* lambda) {
    return guarded([&] {
        require(lmm != nullptr, "null lmm handle");
        cs::lmm_lowrank_basis(lmm, U, ldu, lambda);
    });
}

int cs_lmm_scan(cs_lmm* lmm, const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                double min_maf, int precision, double* beta, double* se, double* pvalue,
                double* log10p, double* freq, int32_t* tested) {
    return guarded([&] {
        require(lmm != nullptr && g != nullptr, "null argument");
        cs::lmm_scan(lmm, g, keep, n_keep, min_maf, precision, beta, se, pvalue, log10p, freq,
                     tested);
    });
}

int cs_lmm_scan_window(cs_lmm* lmm, const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                       int64_t snp_begin, int64_t snp_end, double min_maf, int precision,
                       double* beta, double* se, double* pvalue, double* log10p, double* freq,
                       int32_t* tested) {
    return guarded([&] {
        require(lmm != nullptr && g != nullptr, "null argument");
        cs::lmm_scan_window(lmm, g, keep, n_keep, snp_begin, snp_end, min_maf, precision, beta,
                            se, pvalue, log10p, freq, tested, 0);
    });
}

void cs_lmm_destroy(cs_lmm* lmm) { cs::lmm_destroy(lmm); }

void cs_grm_default_options(cs_grm_options* opt) {
    if (!opt) return;
    opt->min_maf = 0.01;
    opt->algorithm = 1;
}

int cs_grm_create(const cs_genotypes* g, const int32_t* variants, int64_t n_variants,
                  const cs_grm_options* opt, cs_grm** out) {
    return guarded([&] {
        require(g != nullptr && out != nullptr, "null argument");
        *out = cs::grm_create(g, variants, n_variants, opt);
    });
}

int cs_grm_loco(const cs_grm* global, const cs_grm* chrom, cs_grm** out) {
    return guarded([&] {
        require(out != nullptr, "null argument");
        *out = cs::grm_loco(global, chrom);
    });
}

int cs_grm_from_host(int64_t n, const double* G, int64_t ldg, cs_grm** out) {
    return guarded([&] {
        require(out != nullptr, "null argument");
        *out = cs::grm_from_host(n, G, ldg);
    });
}

int cs_grm_info(const cs_grm* grm, int64_t* n, int64_t* n_valid, double* sum_2pq) {
    return guarded([&] {
        require(grm != nullptr, "null argument");
        if (n) *n = grm->n;
        if (n_valid) *n_valid = grm->n_valid;
        if (sum_2pq) *sum_2pq = grm->sum_2pq;
    });
}

int cs_grm_copy(const cs_grm* grm, const int32_t* keep, int64_t n_keep, double* out, int64_t ld) {
    return guarded([&] { cs::grm_copy(grm, keep, n_keep, out, ld); });
}

void cs_grm_destroy(cs_grm* grm) { delete grm; }

int cs_eigen_vce_prepare(const cs_grm* grm, const int32_t* keep, int64_t n_keep, const double* y,
                         const double* X, int64_t p, int use_covariate_projection,
                         cs_eigen_vce** out) {
    return guarded([&] {
        require(out != nullptr, "null argument");
        *out = cs::eigen_prepare(grm, keep, n_keep, y, X, p, use_covariate_projection != 0);
    });
}

int cs_eigen_vce_run_null(cs_eigen_vce* vce, cs_eigen_vce_result* out) {
    return guarded([&] { cs::eigen_run_null(vce, out); });
}

int cs_eigen_vce_dims(const cs_eigen_vce* vce, int64_t* n, int64_t* n_eig, int64_t* p) {
    return guarded([&] {
        require(vce != nullptr && vce->d != nullptr, "null argument");
        if (n) *n = vce->d->n;
        if (n_eig) *n_eig = vce->d->n_eig;
        if (p) *p = vce->d->p;
    });
}

int cs_eigen_vce_get(const cs_eigen_vce* vce, double* D, double* Uty, double* UtX, double* W,
                     int64_t ldw) {
    return guarded([&] { cs::eigen_get(vce, D, Uty, UtX, W, ldw); });
}

void cs_eigen_vce_destroy(cs_eigen_vce* vce) { delete vce; }

void cs_mv_vce_default_options(cs_mv_vce_options* opt) {
    if (!opt) return;
    opt->max_iter = 1000;
    opt->tol = 1e-8;
    opt->aireml = 0;
    opt->em_min_iter = 10;
    opt->ai_max_iter = 50;
    opt->ai_tol = 1e-8;
}

int cs_mv_eigen_vce_prepare(const cs_grm* grm, const int32_t* keep, int64_t n_keep,
                            const double* Y, int64_t d, const double* X, int64_t p,
                            int use_projection, cs_mv_eigen_vce** out) {
    return guarded([&] {
        require(out != nullptr, "null argument");
        *out = cs::mv_prepare(grm, keep, n_keep, Y, d, X, p, use_projection != 0);
    });
}

int cs_mv_eigen_vce_run_null(cs_mv_eigen_vce* vce, const cs_mv_vce_options* opt,
                             int32_t* converged, int32_t* iterations, double* logl) {
    return guarded([&] {
        const bool ok = cs::mv_run_null(vce, opt);
        if (converged) *converged = ok ? 1 : 0;
        if (iterations) *iterations = vce->iterations;
        if (logl) *logl = vce->logl;
    });
}

int cs_mv_eigen_vce_dims(const cs_mv_eigen_vce* vce, int64_t* n, int64_t* n_eig, int64_t* d) {
    return guarded([&] {
        require(vce != nullptr && vce->d != nullptr, "null argument");
        if (n) *n = vce->d->n;
        if (n_eig) *n_eig = vce->d->n_eig;
        if (d) *d = vce->traits;
    });
}

int cs_mv_eigen_vce_get(const cs_mv_eigen_vce* vce, double* Vg, double* Ve, double* Vg_se,
                        double* Ve_se, double* D, double* Uty) {
    return guarded([&] { cs::mv_get(vce, Vg, Ve, Vg_se, Ve_se, D, Uty); });
}

void cs_mv_eigen_vce_destroy(cs_mv_eigen_vce* vce) { delete vce; }

int cs_mvlmm_scan_vce(const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                      const cs_mv_eigen_vce* vce, int64_t snp_begin, int64_t snp_end,
                      int precision, double* beta, double* cov, double* wald, double* pvalue,
                      double* freq, int32_t* status) {
    return guarded([&] {
        require(g != nullptr && keep != nullptr, "null argument");
        cs::mv_scan(g, keep, n_keep, vce, snp_begin, snp_end, precision, beta, cov, wald, pvalue,
                    freq, status);
    });
}

int cs_lmm_prepare_from_vce(cs_lmm* lmm, const cs_eigen_vce* vce, int use_residuals) {
    return guarded([&] {
        require(lmm != nullptr, "null argument");
        cs::lmm_prepare_from_vce(lmm, vce, use_residuals != 0);
    });
}

int cs_normal_matrix(uint64_t seed, int64_t n, int64_t cols, double* out) {
    return guarded([&] {
        require(n >= 0 && cols >= 0 && (out != nullptr || n * cols == 0), "bad arguments");
        if (n * cols == 0) return;
        cs::OmegaWorkspace ws;
        cs::DeviceBuffer<double> d, t;
        d.resize(n * cols);
        t.resize(n * cols);
        cs::generate_omega_device(seed, n, cols, d.get(), cols, ws, 0);
        cs::rowmajor_to_colmajor(d.get(), cols, n, cols, t.get(), n, 0);
        CS_CUDA(cudaMemcpy(out, t.get(), 8 * n * cols, cudaMemcpyDeviceToHost));
    });
}

int cs_pcg_solve(cs_kinship* op, double kinship_divisor, double sigma2_g, double sigma2_e,
                 const double* B, int64_t ldb, int64_t k, double* X, int64_t ldx, double tol,
                 int relative, int max_iter, int precision, int32_t* iterations, void* stream) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        require(k == 0 || (B != nullptr && X != nullptr), "null argument");
        cs::pcg_solve_public(op, kinship_divisor, sigma2_g, sigma2_e, B, ldb, k, X, ldx, tol,
                             relative, max_iter, precision, iterations, (cudaStream_t)stream);
    });
}

int cs_pcg_solve_records(cs_kinship* op, double kinship_divisor, const int32_t* rec_to_row,
                         int64_t n_records, int with_pe, double sigma2_g, double sigma2_pe,
                         double sigma2_e, const double* B, int64_t ldb, int64_t k, double* X,
                         int64_t ldx, double tol, int relative, int max_iter, int precision,
                         int32_t* iterations, void* stream) {
    return guarded([&] {
        require(op != nullptr, "null kinship handle");
        require(k == 0 || (B != nullptr && X != nullptr), "null argument");
        cs::pcg_solve_records_public(op, kinship_divisor, rec_to_row, n_records, with_pe != 0,
                                     sigma2_g, sigma2_pe, sigma2_e, B, ldb, k, X, ldx, tol,
                                     relative, max_iter, precision, iterations,
                                     (cudaStream_t)stream);
    });
}

void cs_mv_stcg_default_options(cs_mv_stcg_options* opt) {
    if (opt) cs::mv_stcg_default_options(opt);
}

int cs_mv_stcg_solve(cs_kinship* op, double kinship_divisor, const double* Y, int32_t d,
                     const double* X, int64_t p, const cs_mv_stcg_options* opt, double* Vg,
                     double* Ve, cs_mv_stcg_result* res) {
    return guarded([&] {
        require(op != nullptr && res != nullptr, "null argument");
        cs::mv_stcg_solve(op, kinship_divisor, Y, d, X, p, opt, Vg, Ve, res);
    });
}

void cs_vce_default_options(cs_vce_options* opt) {
    if (opt) cs::vce_default_options(opt);
}

int cs_vce_create(cs_vce** out) {
    return guarded([&] {
        require(out != nullptr, "null output handle");
        *out = cs::vce_create();
    });
}

int cs_vce_solve_stcg(cs_vce* vce, cs_kinship* op, double kinship_divisor,
                      const int32_t* rec_to_row, int64_t n_records, int with_pe, const double* y,
                      const double* X, int64_t p, const cs_vce_options* opt, cs_vce_result* res) {
    return guarded([&] {
        require(vce != nullptr && op != nullptr && res != nullptr, "null argument");
        cs::vce_solve_stcg(vce, op, kinship_divisor, rec_to_row, n_records, with_pe, y, X, p, opt,
                           res);
    });
}

int cs_vce_solution(const cs_vce* vce, double* beta, double* a_rows, double* pe_rows) {
    return guarded([&] {
        require(vce != nullptr, "null vce handle");
        cs::vce_solution(vce, beta, a_rows, pe_rows);
    });
}

int cs_vce_history(const cs_vce* vce, double* out, int64_t* n_iterations) {
    return guarded([&] {
        require(vce != nullptr, "null vce handle");
        cs::vce_history(vce, out, n_iterations);
    });
}

void cs_vce_destroy(cs_vce* vce) { cs::vce_destroy(vce); }

int cs_stcg_scan(const cs_genotypes* g, const double* G, int64_t q, const int32_t* subject_rows,
                 const int32_t* obs_to_subject, int64_t n_obs, const double* y, const double* X,
                 int64_t p, double vg, double vpe, double ve, double min_maf, int64_t snp_begin,
                 int64_t snp_end, double* beta, double* se, double* pvalue, double* log10p,
                 double* maf, int32_t* tested) {
    return guarded([&] {
        cs::stcg_scan(g, G, q, subject_rows, obs_to_subject, n_obs, y, X, p, vg, vpe, ve, min_maf,
                      snp_begin, snp_end, beta, se, pvalue, log10p, maf, tested);
    });
}

int cs_mvlmm_scan(const cs_genotypes* g, const int32_t* keep, int64_t n, const double* W,
                  int64_t r, const double* D, const double* Uty, int64_t d, const double* UtX,
                  int64_t p, const double* Vg, const double* Ve, int64_t snp_begin,
                  int64_t snp_end, int precision, double* beta, double* cov, double* wald,
                  double* pvalue, double* freq, int32_t* status) {
    return guarded([&] {
        require(beta && wald && pvalue && freq && status, "null output");
        cs::mvlmm_scan(g, keep, n, W, r, D, Uty, d, UtX, p, Vg, Ve, snp_begin, snp_end, precision,
                       beta, cov, wald, pvalue, freq, status);
    });
}

void cs_server_default_options(cs_server_options* opt) {
    if (opt) cs::server_default_options(opt);
}

int cs_server_create(const cs_genotypes* g, const int32_t* variants, int64_t n_variants,
                     const cs_server_options* opt, cs_server** out) {
    return guarded([&] {
        require(out != nullptr, "null output handle");
        *out = cs::server_create(g, variants, n_variants, opt);
    });
}

int cs_server_submit(cs_server* server, const cs_serve_request* request, int64_t* id) {
    return guarded([&] {
        require(server != nullptr && id != nullptr, "null argument");
        *id = cs::server_submit(server, request);
    });
}

int cs_server_wait(cs_server* server, int64_t id, double timeout_s, cs_serve_status* status) {
    return guarded([&] {
        require(server != nullptr, "null server handle");
        cs::server_wait(server, id, timeout_s, status);
    });
}

int cs_server_result(cs_server* server, int64_t id, int32_t trait, double* sigma2, double* beta,
                     double* se, double* pvalue, double* log10p, double* freq, int32_t* tested) {
    return guarded([&] {
        require(server != nullptr, "null server handle");
        cs::server_result(server, id, trait, sigma2, beta, se, pvalue, log10p, freq, tested);
    });
}

int cs_server_release(cs_server* server, int64_t id) {
    return guarded([&] {
        require(server != nullptr, "null server handle");
        cs::server_release(server, id);
    });
}

int cs_server_stats(cs_server* server, cs_server_statistics* stats) {
    return guarded([&] {
        require(server != nullptr && stats != nullptr, "null argument");
        cs::server_stats(server, stats);
    });
}

void cs_server_destroy(cs_server* server) { cs::server_destroy(server); }

int cs_write_assoc_txt(const char* out_path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                       const double* freq, const double* beta, const double* se,
                       const double* pvalue, const double* log10p, const int32_t* tested,
                       int stcg_columns) {
    return guarded([&] {
        cs::write_assoc_txt(out_path, bim_path, n_snps, n_obs, freq, beta, se, pvalue, log10p,
                            tested, stcg_columns);
    });
}

int cs_write_assoc(const char* out_path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                   const double* freq, const double* beta, const double* se, const double* pvalue,
                   const double* log10p, const int32_t* tested, const int64_t* order,
                   int64_t n_order, int layout, int gzip) {
    return guarded([&] {
        cs::write_assoc(out_path, bim_path, n_snps, n_obs, freq, beta, se, pvalue, log10p, tested,
                        order, n_order, layout, gzip != 0);
    });
}

int cs_append_cosmic_sumstats(const char* path, const char* bim_path, int64_t n_snps,
                              int32_t n_obs, const double* freq, const double* beta,
                              const double* se, const double* pvalue, const double* log10p,
                              const int32_t* tested, const char* model, int append, int gzip,
                              const char* created) {
    return guarded([&] {
        cs::append_cosmic_sumstats(path, bim_path, n_snps, n_obs, freq, beta, se, pvalue, log10p,
                                   tested, model, append != 0, gzip != 0, created);
    });
}

int cs_append_scan_common_meta(const char* out_prefix, const char* model, int64_t n, int loco,
                               int covariate_projection, int vce_converged) {
    return guarded([&] {
        cs::append_scan_common_meta(out_prefix, model, n, loco != 0, covariate_projection != 0,
                                    vce_converged != 0);
    });
}

int cs_write_assoc_mv_txt(const char* out_path, const char* bim_path, int64_t n_snps, int32_t d,
                          const double* freq, const double* wald, const double* pvalue,
                          const double* beta, const double* cov) {
    return guarded([&] {
        cs::write_assoc_mv_txt(out_path, bim_path, n_snps, d, freq, wald, pvalue, beta, cov);
    });
}

int cs_write_scan_meta(const char* out_prefix, int32_t requested_rank, double trace_threshold) {
    return guarded([&] { cs::write_scan_meta(out_prefix, requested_rank, trace_threshold, false); });
}

int cs_write_scan_meta_full_eigen(const char* out_prefix) {
    return guarded([&] { cs::write_scan_meta(out_prefix, 0, 0.0, true); });
}

int cs_write_low_rank_meta(const char* out_prefix, int32_t n_rows, const char* const* scopes,
                           const cs_lowrank_diagnostics* diags, int64_t n, double error_tol,
                           const char* const* fallbacks) {
    return guarded([&] {
        cs::write_low_rank_meta(out_prefix, n_rows, scopes, diags, n, error_tol, fallbacks);
    });
}

int cs_fam_read(const char* fam_path, cs_samples** out) {
    return guarded([&] {
        if (!fam_path || !out) cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_fam_read: null argument");
        auto* s = new cs_samples();
        try {
            s->fam = cs::read_fam(fam_path);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

int cs_samples_count(const cs_samples* s, int64_t* n) {
    return guarded([&] {
        if (!s || !n) cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_samples_count: null argument");
        *n = (int64_t)s->fam.size();
    });
}

int cs_samples_id(const cs_samples* s, int64_t i, char* fid, size_t fid_len, char* iid, size_t iid_len) {
    return guarded([&] {
        if (!s || i < 0 || i >= (int64_t)s->fam.size())
            cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_samples_id: sample index out of range");
        auto put = [](const std::string& v, char* buf, size_t len) {
            if (!buf || len == 0) return;
            const size_t k = std::min(len - 1, v.size());
            std::memcpy(buf, v.data(), k);
            buf[k] = '\0';
        };
        put(s->fam[i].fid, fid, fid_len);
        put(s->fam[i].iid, iid, iid_len);
    });
}

int cs_samples_fam_phenotype(const cs_samples* s, double* y) {
    return guarded([&] {
        if (!s || !y) cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_samples_fam_phenotype: null argument");
        for (size_t i = 0; i < s->fam.size(); ++i) y[i] = s->fam[i].phenotype;
    });
}

void cs_samples_destroy(cs_samples* s) { delete s; }

int cs_pheno_load(const char* path, int32_t col_idx, double missing_code, cs_pheno** out) {
    return guarded([&] {
        if (!path || !out) cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_pheno_load: null argument");
        auto* p = new cs_pheno();
        try {
            p->table.load(path, col_idx, missing_code);
            p->table.n_traits = 1;
        } catch (...) {
            delete p;
            throw;
        }
        *out = p;
    });
}

int cs_pheno_load_matrix(const char* path, const int32_t* cols, int32_t n_cols, double missing_code,
                         cs_pheno** out) {
    return guarded([&] {
        if (!path || !out || n_cols < 0 || (n_cols > 0 && !cols))
            cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_pheno_load_matrix: null argument");
        auto* p = new cs_pheno();
        try {
            p->table.load_matrix(path, std::vector<int>(cols, cols + n_cols), missing_code);
        } catch (...) {
            delete p;
            throw;
        }
        *out = p;
    });
}

int cs_pheno_traits(const cs_pheno* p, int32_t* n_traits) {
    return guarded([&] {
        if (!p || !n_traits) cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_pheno_traits: null argument");
        *n_traits = p->table.n_traits;
    });
}

int cs_pheno_align(const cs_pheno* p, const cs_samples* s, double* y, int64_t* matched) {
    return guarded([&] {
        if (!p || !s || !y) cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_pheno_align: null argument");
        const int64_t m = p->table.align(s->fam, y);
        if (matched) *matched = m;
    });
}

int cs_pheno_align_matrix(const cs_pheno* p, const cs_samples* s, double* Y, int64_t ldy,
                          int64_t* matched) {
    return guarded([&] {
        if (!p || !s || !Y || ldy < (int64_t)s->fam.size())
            cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_pheno_align_matrix: bad argument");
        const int64_t m = p->table.align_matrix(s->fam, Y, ldy);
        if (matched) *matched = m;
    });
}

void cs_pheno_destroy(cs_pheno* p) { delete p; }

int cs_covar_load(const char* path, double missing_code, cs_covar** out) {
    return guarded([&] {
        if (!path || !out) cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_covar_load: null argument");
        auto* c = new cs_covar();
        try {
            c->table.load(path, missing_code);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

int cs_covar_load_categorical(const char* path, const char* missing_token, cs_covar** out) {
    return guarded([&] {
        if (!path || !out) cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_covar_load_categorical: null argument");
        auto* c = new cs_covar();
        try {
            c->table.load_categorical(path, missing_token ? missing_token : "-9");
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

int cs_covar_columns(const cs_covar* c, int32_t* p) {
    return guarded([&] {
        if (!c || !p) cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_covar_columns: null argument");
        *p = c->table.n_cols;
    });
}

int cs_covar_align(const cs_covar* c, const cs_samples* s, float* X, int64_t ldx, int64_t* matched) {
    return guarded([&] {
        if (!c || !s || (c->table.n_cols > 0 && (!X || ldx < (int64_t)s->fam.size())))
            cs::fail(CS_ERR_INVALID_ARGUMENT, "cs_covar_align: bad argument");
        const int64_t m = c->table.align(s->fam, X, ldx);
        if (matched) *matched = m;
    });
}

void cs_covar_destroy(cs_covar* c) { delete c; }

int cs_filter_samples(const double* y, int64_t n, const float* X, int64_t ldx, int32_t p,
                      int32_t* keep, int64_t* n_keep) {
    return guarded([&] {
        if (n < 0 || p < 0 || (n > 0 && (!y || !keep)) || (p > 0 && (!X || ldx < n)) || !n_keep)
            cs::fail(CS_ERR_INVALID_ARGUMENT, "DataFilter: X and y dimension mismatch");
        *n_keep = cs::filter_samples(y, n, X, ldx, p, keep);
    });
}

int cs_profile_enable(int on) {
    return guarded([&] { cs::prof::set_enabled(on != 0); });
}

int cs_profile_summary(char* buf, size_t len, size_t* needed) {
    return guarded([&] {
        const std::string js = cs::prof::summary_json();
        if (needed) *needed = js.size() + 1;
        if (buf && len > 0) {
            const size_t n = std::min(len - 1, js.size());
            std::memcpy(buf, js.data(), n);
            buf[n] = 0;
        }
    });
}

int cs_launch_count(int64_t* count) {
    return guarded([&] {
        require(count != nullptr, "null argument");
        *count = cs::prof::launches();
    });
}

}  // extern "C"
