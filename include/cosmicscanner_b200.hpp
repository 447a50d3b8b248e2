// Header-only C++ facade over the C ABI of cosmicscanner_b200.h, shaped like the reference's
// interfaces so its call sites can swap in without semantic change:
//   cs::Genotypes        ~ cosmic::PlinkReader (libCosmicCore/src/plink_reader.h)
//   cs::KinshipOperator  ~ cosmic::KinshipOperator (src/kinship_operator.h:18-46)
//   cs::GenotypeMatrix   ~ cosmic::GenotypeMatrix (libCosmicCore/src/matrix_adapter.h:40-53)
//   cs::pcg_solve        ~ cosmic::MatrixFreePCG::solve (libCosmicCore/src/matrix_free_pcg.h)
//   cs::StcgVce          ~ cosmic::STCG_VCE (libCosmicCore/src/stcg_vce.h:7-54)
//   cs::LmmEngine        ~ LmmEngine::prepareLowRankMatrixFree / scan (src/lmm_engine.h)
// Status codes come back as std::runtime_error (std::invalid_argument for bad arguments)
// carrying the library's message, as the reference throws.  Types are Eigen-free: matrices
// are column-major std::vector<double> with explicit row counts.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cosmicscanner_b200.h"

namespace cs {

inline void check(int status) {
    if (status == CS_OK) return;
    const std::string msg = cs_last_error();
    if (status == CS_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

enum class Precision { FP64 = CS_PRECISION_FP64, Mixed = CS_PRECISION_MIXED };

class Genotypes {
   public:
    // PlinkReader::openBed on `prefix`.bed/.bim/.fam; the packed matrix becomes resident.
    static Genotypes open(const std::string& prefix) {
        cs_genotypes* h = nullptr;
        check(cs_genotypes_open_plink(prefix.c_str(), &h));
        return Genotypes(h);
    }
    // From the bytes of a .bed file (magic included).
    static Genotypes from_bed(const uint8_t* bed, size_t n_bytes, int64_t n_samples, int64_t n_snps) {
        cs_genotypes* h = nullptr;
        check(cs_genotypes_create(bed, n_bytes, n_samples, n_snps, &h));
        return Genotypes(h);
    }
    Genotypes(Genotypes&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
    Genotypes& operator=(Genotypes&& o) noexcept {
        std::swap(h_, o.h_);
        return *this;
    }
    Genotypes(const Genotypes&) = delete;
    Genotypes& operator=(const Genotypes&) = delete;
    ~Genotypes() { cs_genotypes_destroy(h_); }

    int64_t getNumSamples() const { return info().first; }
    int64_t getNumSnps() const { return info().second; }
    // PlinkReader::computeStats outputs (over all .fam samples).
    void stats(std::vector<double>& mean, std::vector<double>& inv_std) const {
        mean.resize(getNumSnps());
        inv_std.resize(getNumSnps());
        check(cs_genotypes_stats(h_, mean.data(), inv_std.data(), nullptr, nullptr));
    }
    cs_genotypes* handle() const { return h_; }

   private:
    explicit Genotypes(cs_genotypes* h) : h_(h) {}
    std::pair<int64_t, int64_t> info() const {
        int64_t n = 0, m = 0;
        check(cs_genotypes_info(h_, &n, &m, nullptr));
        return {n, m};
    }
    cs_genotypes* h_ = nullptr;
};

class KinshipOperator {
   public:
    // createKinshipOperator(reader, keep_indices, variant_indices) (kinship_operator.cpp:370-374);
    // empty vectors mean all samples / all variants.  `g` must outlive the operator.
    KinshipOperator(const Genotypes& g, const std::vector<int>& keep = {},
                    const std::vector<int>& variants = {}) {
        check(cs_kinship_create(g.handle(), keep.empty() ? nullptr : keep.data(), (int64_t)keep.size(),
                                variants.empty() ? nullptr : variants.data(),
                                (int64_t)variants.size(), &h_));
        check(cs_kinship_info(h_, &rows_, &m_));
    }
    KinshipOperator(const KinshipOperator&) = delete;
    KinshipOperator& operator=(const KinshipOperator&) = delete;
    ~KinshipOperator() { cs_kinship_destroy(h_); }

    int rows() const { return (int)rows_; }
    int cols() const { return (int)rows_; }
    int numVariants() const { return (int)m_; }
    bool isDense() const { return false; }

    // apply(const MatrixXd& X, MatrixXd& out): X is rows() x k column-major (host).
    void apply(const std::vector<double>& X, int64_t k, std::vector<double>& out,
               Precision p = Precision::FP64) const {
        if ((int64_t)X.size() != rows_ * k)
            throw std::runtime_error("PlinkKinshipOperator::apply: dimension mismatch");
        out.resize(rows_ * k);
        check(cs_kinship_apply_host(h_, X.data(), rows_, k, out.data(), rows_, (int)p));
    }
    void applyTranspose(const std::vector<double>& X, int64_t k, std::vector<double>& out,
                        Precision p = Precision::FP64) const {
        apply(X, k, out, p);  // K is symmetric
    }
    // Device form: X, Y device pointers, column-major with leading dimensions.
    void apply_device(const double* X, int64_t ldx, int64_t k, double* Y, int64_t ldy,
                      Precision p = Precision::FP64, void* stream = nullptr) const {
        check(cs_kinship_apply(h_, X, ldx, k, Y, ldy, (int)p, stream));
    }
    double trace() const {
        double t = 0.0;
        check(cs_kinship_trace(h_, &t));
        return t;
    }
    void getDiagonal(std::vector<double>& d) const {
        d.resize(rows_);
        check(cs_kinship_diagonal(h_, d.data()));
    }
    cs_kinship* handle() const { return h_; }

   private:
    cs_kinship* h_ = nullptr;
    int64_t rows_ = 0, m_ = 0;
};

// GenotypeMatrix (matrix_adapter.h:40-53) over a kinship operator's selection: rows() samples x
// cols() selected variants, z = (dosage - mean) / sd with the all-sample statistics, missing
// calls 0 (PlinkReader::multiply_Z_v / multiply_Zt_v, plink_reader.cpp:241-438).  Host vectors;
// `n_threads` is accepted for signature parity and ignored (the GPU does the work).
class GenotypeMatrix {
   public:
    explicit GenotypeMatrix(const KinshipOperator& op, Precision p = Precision::FP64)
        : op_(&op), p_(p) {}
    int rows() const { return op_->rows(); }
    int cols() const { return op_->numVariants(); }
    // y = Z v: v has cols() entries, y gets rows()
    void multiply_Z_v(const std::vector<double>& v, std::vector<double>& y, int n_threads = 1) const {
        (void)n_threads;
        if ((int64_t)v.size() != cols()) throw std::runtime_error("Dimension mismatch in multiply_Z_v");
        y.resize(rows());
        check(cs_genotype_multiply_z_host(op_->handle(), v.data(), cols(), 1, y.data(), rows(),
                                          (int)p_));
    }
    // y = Z^T v: v has rows() entries, y gets cols()
    void multiply_Zt_v(const std::vector<double>& v, std::vector<double>& y, int n_threads = 1) const {
        (void)n_threads;
        if ((int64_t)v.size() != rows()) throw std::runtime_error("Dimension mismatch in multiply_Zt_v");
        y.resize(cols());
        check(cs_genotype_multiply_zt_host(op_->handle(), v.data(), rows(), 1, y.data(), cols(),
                                           (int)p_));
    }

   private:
    const KinshipOperator* op_;
    Precision p_;
};

// MatrixFreePCG::solve on (sigma2_g K + sigma2_e I) X = B, device column-major blocks.
inline std::vector<int32_t> pcg_solve(const KinshipOperator& op, double sigma2_g, double sigma2_e,
                                      const double* B, int64_t ldb, int64_t k, double* X,
                                      int64_t ldx, double tol = 1e-8, int max_iter = 1000,
                                      bool relative = false, Precision p = Precision::FP64,
                                      double kinship_divisor = 0.0, void* stream = nullptr) {
    std::vector<int32_t> it(k > 0 ? k : 1);
    check(cs_pcg_solve(op.handle(), kinship_divisor, sigma2_g, sigma2_e, B, ldb, k, X, ldx, tol,
                       relative ? 1 : 0, max_iter, (int)p, it.data(), stream));
    it.resize(k);
    return it;
}

// MatrixFreePCG::solve on STCG_VCE's record-level covariance (stcg_vce.cpp:80-126):
// V = sigma2_g Zr K Zr^T + sigma2_pe Zr Zr^T + sigma2_e I, records mapped by rec_to_row (empty:
// one record per operator row).  Device column-major blocks of n_records rows.
inline std::vector<int32_t> pcg_solve_records(const KinshipOperator& op,
                                              const std::vector<int32_t>& rec_to_row,
                                              int64_t n_records, bool with_pe, double sigma2_g,
                                              double sigma2_pe, double sigma2_e, const double* B,
                                              int64_t ldb, int64_t k, double* X, int64_t ldx,
                                              double tol = 1e-10, int max_iter = 2000,
                                              bool relative = false, Precision p = Precision::FP64,
                                              double kinship_divisor = 0.0, void* stream = nullptr) {
    std::vector<int32_t> it(k > 0 ? k : 1);
    check(cs_pcg_solve_records(op.handle(), kinship_divisor,
                               rec_to_row.empty() ? nullptr : rec_to_row.data(), n_records,
                               with_pe ? 1 : 0, sigma2_g, sigma2_pe, sigma2_e, B, ldb, k, X, ldx,
                               tol, relative ? 1 : 0, max_iter, (int)p, it.data(), stream));
    it.resize(k);
    return it;
}

class StcgVce {
   public:
    StcgVce() { check(cs_vce_create(&h_)); }
    StcgVce(const StcgVce&) = delete;
    StcgVce& operator=(const StcgVce&) = delete;
    ~StcgVce() { cs_vce_destroy(h_); }

    static cs_vce_options default_options() {
        cs_vce_options o;
        cs_vce_default_options(&o);
        return o;
    }
    // STCG_VCE::solve(); X is n_records x p column-major; rec_to_row empty = one record per row.
    cs_vce_result solve(const KinshipOperator& op, const std::vector<double>& y,
                        const std::vector<double>& X, int64_t p,
                        const std::vector<int32_t>& rec_to_row = {}, bool with_pe = false,
                        double kinship_divisor = 0.0, const cs_vce_options& opt = default_options()) {
        cs_vce_result r{};
        check(cs_vce_solve_stcg(h_, op.handle(), kinship_divisor,
                                rec_to_row.empty() ? nullptr : rec_to_row.data(), (int64_t)y.size(),
                                with_pe ? 1 : 0, y.data(), X.empty() ? nullptr : X.data(), p, &opt,
                                &r));
        last_ = r;
        rows_ = op.rows();
        p_ = p;
        return r;
    }
    double getVarE() const { return last_.sigma2_e; }
    std::vector<double> getVarsU() const { return {last_.sigma2_g, last_.sigma2_pe}; }
    // final_solution pieces: beta (p), genetic values and pe effects over operator rows
    void solution(std::vector<double>& beta, std::vector<double>& a, std::vector<double>& pe) const {
        beta.resize(p_);
        a.resize(rows_);
        pe.resize(rows_);
        check(cs_vce_solution(h_, beta.data(), a.data(), pe.data()));
    }

   private:
    cs_vce* h_ = nullptr;
    cs_vce_result last_{};
    int64_t rows_ = 0, p_ = 0;
};

class LmmEngine {
   public:
    LmmEngine() { check(cs_lmm_create(&h_)); }
    LmmEngine(const LmmEngine&) = delete;
    LmmEngine& operator=(const LmmEngine&) = delete;
    ~LmmEngine() { cs_lmm_destroy(h_); }

    // prepareLowRankMatrixFree(y, X, op, rank, ...): X column-major n x p, already FP32-rounded
    // where the caller mirrors the reference's MatrixXf covariates.
    cs_lowrank_diagnostics prepareLowRankMatrixFree(const std::vector<double>& y,
                                                    const std::vector<double>& X, int64_t p,
                                                    KinshipOperator& op, int rank = 256,
                                                    int oversample = 10, int64_t seed = 42,
                                                    double trace_threshold = 0.95, int min_rank = 1,
                                                    Precision prec = Precision::FP64) {
        cs_lowrank_diagnostics d{};
        check(cs_lmm_prepare_lowrank_matrix_free(h_, op.handle(), y.data(),
                                                 X.empty() ? nullptr : X.data(), p, rank,
                                                 oversample, seed, trace_threshold, min_rank,
                                                 (int)prec, &d));
        return d;
    }

    struct ScanResult {
        std::vector<double> beta, se, p, log10p, freq;
        std::vector<int32_t> tested;
    };
    // scan(PlinkReader, ...) -> scanLowRank for every SNP, keep = analysed samples in y order.
    ScanResult scan(const Genotypes& g, const std::vector<int32_t>& keep, double min_maf = 0.01,
                    Precision prec = Precision::FP64) {
        const int64_t m = g.getNumSnps();
        ScanResult r;
        for (auto* v : {&r.beta, &r.se, &r.p, &r.log10p, &r.freq}) v->resize(m);
        r.tested.resize(m);
        check(cs_lmm_scan(h_, g.handle(), keep.data(), (int64_t)keep.size(), min_maf, (int)prec,
                          r.beta.data(), r.se.data(), r.p.data(), r.log10p.data(), r.freq.data(),
                          r.tested.data()));
        return r;
    }

    // scan() over SNPs [begin, end) (a LOCO chromosome's run).
    ScanResult scanWindow(const Genotypes& g, const std::vector<int32_t>& keep, int64_t begin,
                          int64_t end, double min_maf = 0.01, Precision prec = Precision::FP64) {
        ScanResult r;
        const int64_t m = end - begin;
        for (auto* v : {&r.beta, &r.se, &r.p, &r.log10p, &r.freq}) v->resize(m > 0 ? m : 0);
        r.tested.resize(m > 0 ? m : 0);
        check(cs_lmm_scan_window(h_, g.handle(), keep.data(), (int64_t)keep.size(), begin, end,
                                 min_maf, (int)prec, r.beta.data(), r.se.data(), r.p.data(),
                                 r.log10p.data(), r.freq.data(), r.tested.data()));
        return r;
    }

    // prepareFromVce(vce): the exact scan on EigenVce's basis and null model.
    void prepareFromVce(const class EigenVce& vce, bool use_residuals = false);

    cs_lmm* handle() { return h_; }

   private:
    cs_lmm* h_ = nullptr;
};

// ---- dense exact tier: GrmBuilder (libCosmicCore/src/grm_builder.h), EigenVce and MvEigenVce
// (libCosmicCore/src/eigen_vce.h); every N x N matrix stays on the device.
class GrmBuilder {
   public:
    explicit GrmBuilder(double min_maf = 0.01, int algorithm = 1) {
        cs_grm_default_options(&opt_);
        opt_.min_maf = min_maf;
        opt_.algorithm = algorithm;
    }
    GrmBuilder(const GrmBuilder&) = delete;
    GrmBuilder& operator=(const GrmBuilder&) = delete;
    ~GrmBuilder() { cs_grm_destroy(h_); }
    // compute(reader) over the given SNPs (empty: all) of every sample.
    void compute(const Genotypes& g, const std::vector<int32_t>& variants = {}) {
        cs_grm_destroy(h_);
        h_ = nullptr;
        check(cs_grm_create(g.handle(), variants.empty() ? nullptr : variants.data(),
                            (int64_t)variants.size(), &opt_, &h_));
    }
    int64_t getTotalSnps() const {
        int64_t v = 0;
        check(cs_grm_info(h_, nullptr, &v, nullptr));
        return v;
    }
    double getSum2pq() const {
        double v = 0;
        check(cs_grm_info(h_, nullptr, nullptr, &v));
        return v;
    }
    // getGrm(), or G[keep, keep] (column-major).
    std::vector<double> getGrm(const std::vector<int32_t>& keep = {}) const {
        int64_t n = 0;
        check(cs_grm_info(h_, &n, nullptr, nullptr));
        const int64_t k = keep.empty() ? n : (int64_t)keep.size();
        std::vector<double> out((size_t)(k * k));
        check(cs_grm_copy(h_, keep.empty() ? nullptr : keep.data(), k, out.data(), k));
        return out;
    }
    const cs_grm* handle() const { return h_; }

   private:
    cs_grm_options opt_{};
    cs_grm* h_ = nullptr;
};

class EigenVce {
   public:
    explicit EigenVce(bool use_covariate_projection = true) : proj_(use_covariate_projection) {}
    EigenVce(const EigenVce&) = delete;
    EigenVce& operator=(const EigenVce&) = delete;
    ~EigenVce() { cs_eigen_vce_destroy(h_); }
    // prepare(y, X, G[keep, keep]); X column-major n x p (FP32-rounded values).
    void prepare(const std::vector<double>& y, const std::vector<double>& X, int64_t p,
                 const GrmBuilder& grm, const std::vector<int32_t>& keep = {}) {
        cs_eigen_vce_destroy(h_);
        h_ = nullptr;
        check(cs_eigen_vce_prepare(grm.handle(), keep.empty() ? nullptr : keep.data(),
                                   (int64_t)keep.size(), y.data(), X.empty() ? nullptr : X.data(),
                                   p, proj_ ? 1 : 0, &h_));
    }
    // runNullModel() (Brent); the estimates and diagnostics.
    cs_eigen_vce_result runNullModel() {
        cs_eigen_vce_result r{};
        check(cs_eigen_vce_run_null(h_, &r));
        return r;
    }
    const cs_eigen_vce* handle() const { return h_; }

   private:
    bool proj_;
    cs_eigen_vce* h_ = nullptr;
};

inline void LmmEngine::prepareFromVce(const EigenVce& vce, bool use_residuals) {
    check(cs_lmm_prepare_from_vce(h_, vce.handle(), use_residuals ? 1 : 0));
}

class MvEigenVce {
   public:
    MvEigenVce() { cs_mv_vce_default_options(&opt_); }
    MvEigenVce(const MvEigenVce&) = delete;
    MvEigenVce& operator=(const MvEigenVce&) = delete;
    ~MvEigenVce() { cs_mv_eigen_vce_destroy(h_); }
    cs_mv_vce_options& options() { return opt_; }
    // prepare(Y, X, G[keep, keep]): Y column-major n x d (d <= 8), X n x p.
    void prepare(const std::vector<double>& Y, int64_t d, const std::vector<double>& X, int64_t p,
                 const GrmBuilder& grm, const std::vector<int32_t>& keep = {}) {
        cs_mv_eigen_vce_destroy(h_);
        h_ = nullptr;
        check(cs_mv_eigen_vce_prepare(grm.handle(), keep.empty() ? nullptr : keep.data(),
                                      (int64_t)keep.size(), Y.data(), d,
                                      X.empty() ? nullptr : X.data(), p, 1, &h_));
    }
    // runNullModel(): false when EM did not converge (the multivariate driver then stops).
    bool runNullModel() {
        int32_t conv = 0;
        check(cs_mv_eigen_vce_run_null(h_, &opt_, &conv, nullptr, nullptr));
        return conv != 0;
    }
    const cs_mv_eigen_vce* handle() const { return h_; }

   private:
    cs_mv_vce_options opt_{};
    cs_mv_eigen_vce* h_ = nullptr;
};

// ---- input side: the .fam samples, phenotype / covariate tables aligned to them and the keep
// list (PlinkReader::readFam, PhenoReader, CovarReader, DataFilter).  Matrices are
// column-major, NaN marks missing values.
class Samples {
   public:
    explicit Samples(const std::string& fam_path) { check(cs_fam_read(fam_path.c_str(), &h_)); }
    ~Samples() { cs_samples_destroy(h_); }
    Samples(const Samples&) = delete;
    Samples& operator=(const Samples&) = delete;
    int64_t size() const {
        int64_t n = 0;
        check(cs_samples_count(h_, &n));
        return n;
    }
    std::vector<double> famPhenotype() const {
        std::vector<double> y(size());
        check(cs_samples_fam_phenotype(h_, y.data()));
        return y;
    }
    const cs_samples* handle() const { return h_; }

   private:
    cs_samples* h_ = nullptr;
};

class PhenoReader {
   public:
    PhenoReader() = default;
    ~PhenoReader() { cs_pheno_destroy(h_); }
    PhenoReader(const PhenoReader&) = delete;
    PhenoReader& operator=(const PhenoReader&) = delete;
    void load(const std::string& path, int col_idx = 1, double missing_val = -9.0) {
        cs_pheno_destroy(h_);
        h_ = nullptr;
        check(cs_pheno_load(path.c_str(), col_idx, missing_val, &h_));
    }
    void loadMatrix(const std::string& path, const std::vector<int32_t>& cols, double missing_val = -9.0) {
        cs_pheno_destroy(h_);
        h_ = nullptr;
        check(cs_pheno_load_matrix(path.c_str(), cols.empty() ? nullptr : cols.data(),
                                   (int32_t)cols.size(), missing_val, &h_));
    }
    // y in .fam order; returns the matched count
    int64_t align(const Samples& s, std::vector<double>& y) const {
        y.assign(s.size(), 0.0);
        int64_t m = 0;
        check(cs_pheno_align(h_, s.handle(), y.data(), &m));
        return m;
    }
    int64_t alignMatrix(const Samples& s, std::vector<double>& Y, int32_t& n_traits) const {
        check(cs_pheno_traits(h_, &n_traits));
        Y.assign(s.size() * n_traits, 0.0);
        int64_t m = 0;
        check(cs_pheno_align_matrix(h_, s.handle(), Y.data(), s.size(), &m));
        return m;
    }

   private:
    cs_pheno* h_ = nullptr;
};

class CovarReader {
   public:
    CovarReader() = default;
    ~CovarReader() { cs_covar_destroy(h_); }
    CovarReader(const CovarReader&) = delete;
    CovarReader& operator=(const CovarReader&) = delete;
    void load(const std::string& path, double missing_val = -9.0) {
        cs_covar_destroy(h_);
        h_ = nullptr;
        check(cs_covar_load(path.c_str(), missing_val, &h_));
    }
    void loadCategorical(const std::string& path, const std::string& missing_val = "-9") {
        cs_covar_destroy(h_);
        h_ = nullptr;
        check(cs_covar_load_categorical(path.c_str(), missing_val.c_str(), &h_));
    }
    // X (n x p, column-major, float) in .fam order; returns the matched count
    int64_t align(const Samples& s, std::vector<float>& X, int32_t& p) const {
        check(cs_covar_columns(h_, &p));
        X.assign(s.size() * p, 0.0f);
        int64_t m = 0;
        check(cs_covar_align(h_, s.handle(), p ? X.data() : nullptr, s.size(), &m));
        return m;
    }

   private:
    cs_covar* h_ = nullptr;
};

// DataFilter::filterSamples: rows of y / X (n x p, column-major) without NaN, ascending
inline std::vector<int32_t> filterSamples(const std::vector<double>& y, const std::vector<float>& X,
                                          int32_t p) {
    std::vector<int32_t> keep(y.size());
    int64_t n_keep = 0;
    check(cs_filter_samples(y.data(), (int64_t)y.size(), p ? X.data() : nullptr, (int64_t)y.size(),
                            p, keep.data(), &n_keep));
    keep.resize(n_keep);
    return keep;
}

}  // namespace cs
