// Association result files, column for column as the reference writes them.
//
// `.assoc.txt`: src/gwas_output_schema.h:14-37 (kUnifiedHeader, writeAdditiveRow) through
// GwasScanner::flushAssocResults (src/gwas_output.cpp:123-183): rows whose P is NaN are
// skipped; numbers use the stream's default formatting (6 significant digits); the additive
// row carries NA for the six dominance / joint fields.  CHR, SNP, BP, A1 (.bim column 5) and
// A2 (.bim column 6) come from the .bim as PlinkReader::readBim parses it
// (libCosmicCore/src/plink_reader.cpp:52-65); FREQ is the A1 frequency over the analysed
// samples, N the analysed sample count (src/lmm_engine.cpp:1315-1326).
// `.stcg.assoc.txt`: src/models/repeatability_scan_stcg.cpp:190-193 header and :138-140 rows
// (FREQ there is the folded minor-allele frequency, N the subject count).
// `.assoc.mv.txt`: src/models/multivariate_model.cpp:943-951 header and
// src/models/multivariate_output.cpp:40-70 rows (WALD_STAT, P, then BETA_t / SE_t per trait,
// SE = sqrt of the Var(beta) diagonal; a negative or non-finite variance is an error).
// `--out-ssf`: the GWAS-SSF header and rows of flushAssocResults (src/gwas_output.cpp:81-82,
// 149-153).  `.cosmic.sumstats`: GwasScanner::appendCosmicSumstats (src/gwas_output.cpp:
// 186-234; version "1.0" from src/association/sumstats/sumstats.h:53): a header with the
// creation time on the first call, then per call (one per chromosome under LOCO) one row per
// tested SNP with per-field precisions.  `--out-gz`: the same text through zlib's gz* writer
// (src/gzip_writer.cpp:12-55); appends add a gzip member.
#include <zlib.h>

#include <chrono>
#include <cmath>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "cs_internal.h"

namespace cs {

namespace {

struct BimRow {
    std::string chrom, id, a1, a2;
    long long bp = 0;
};

std::vector<BimRow> read_bim(const std::string& path) {
    std::ifstream ifs(path);
    if (!ifs) fail(CS_ERR_IO, "Cannot open .bim file: " + path);
    std::vector<BimRow> rows;
    std::string line;
    while (std::getline(ifs, line)) {
        if (line.empty()) continue;
        std::stringstream ss(line);
        BimRow r;
        double cm = 0.0;
        ss >> r.chrom >> r.id >> cm >> r.bp >> r.a1 >> r.a2;
        rows.push_back(std::move(r));
    }
    return rows;
}

// gzip sink with an 8 KiB put area: whole buffers go to gzwrite, the rest on flush.  The
// mode string is formed from Z_DEFAULT_COMPRESSION as the reference forms it ("wb-1" /
// "ab-1"): zlib's mode parser skips the '-' and takes the digit, so the files are written at
// level 1, which the gzip header records (XFL = 4).
class GzipBuf : public std::streambuf {
public:
    GzipBuf(const std::string& path, bool append) {
        const std::string mode = std::string(append ? "ab" : "wb") + std::to_string(Z_DEFAULT_COMPRESSION);
        file_ = gzopen(path.c_str(), mode.c_str());
        if (!file_) fail(CS_ERR_IO, "Failed to open gzip file for writing: " + path);
        setp(buf_, buf_ + sizeof(buf_));
    }
    ~GzipBuf() override { close(); }
    bool close() {
        if (!file_) return true;
        const bool flushed = sync() == 0;
        const int status = gzclose(file_);
        file_ = nullptr;
        return flushed && status == Z_OK;
    }

protected:
    int sync() override {
        if (!file_) return -1;
        const int n = (int)(pptr() - pbase());
        if (n > 0) {
            if (gzwrite(file_, pbase(), (unsigned)n) != n) return -1;
            setp(buf_, buf_ + sizeof(buf_));
        }
        return 0;
    }
    int_type overflow(int_type c) override {
        if (sync() != 0) return traits_type::eof();
        if (traits_type::eq_int_type(c, traits_type::eof())) return traits_type::not_eof(c);
        *pptr() = traits_type::to_char_type(c);
        pbump(1);
        return c;
    }

private:
    gzFile file_ = nullptr;
    char buf_[8192];
};

// One output file of the association writers: plain (truncate or append) or gzip.
class AssocOut {
public:
    AssocOut(const std::string& path, bool gzip, bool append) : path_(path), os_(nullptr) {
        if (gzip) {
            gz_ = std::make_unique<GzipBuf>(path, append);
            os_.rdbuf(gz_.get());
        } else {
            if (!file_.open(path, std::ios::out | (append ? std::ios::app : std::ios::trunc)))
                fail(CS_ERR_IO, "Cannot open association output: " + path);
            os_.rdbuf(&file_);
        }
    }
    std::ostream& os() { return os_; }
    void finish() {
        os_.flush();
        if (!os_) fail(CS_ERR_IO, "Failed while writing association output: " + path_);
        const bool closed = gz_ ? gz_->close() : file_.close() != nullptr;
        if (!closed) fail(CS_ERR_IO, "Failed closing association output: " + path_);
    }

private:
    std::string path_;
    std::filebuf file_;
    std::unique_ptr<GzipBuf> gz_;
    std::ostream os_;
};

std::vector<BimRow> bim_for(const char* bim_path, int64_t n_snps, const char* who) {
    std::vector<BimRow> bim = read_bim(bim_path);
    if ((int64_t)bim.size() != n_snps)
        fail(CS_ERR_INVALID_ARGUMENT, std::string(who) + ": .bim has " + std::to_string(bim.size()) +
                                          " variants, results have " + std::to_string(n_snps));
    return bim;
}

}  // namespace

void write_assoc(const char* out_path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                 const double* freq, const double* beta, const double* se, const double* p,
                 const double* log10p, const int32_t* tested, const int64_t* order,
                 int64_t n_order, int layout, bool gzip) {
    if (!out_path || !bim_path || n_snps < 0 || !freq || !beta || !se || !p || !log10p ||
        (order && n_order < 0))
        fail(CS_ERR_INVALID_ARGUMENT, "write_assoc: null argument");
    if (layout < CS_ASSOC_UNIFIED || layout > CS_ASSOC_SSF)
        fail(CS_ERR_INVALID_ARGUMENT, "write_assoc: unknown layout");
    const std::vector<BimRow> bim = bim_for(bim_path, n_snps, "write_assoc");
    std::vector<int64_t> rows;
    if (order) {
        std::vector<uint8_t> seen(n_snps, 0);
        rows.assign(order, order + n_order);
        for (int64_t j : rows) {
            if (j < 0 || j >= n_snps || seen[j])
                fail(CS_ERR_INVALID_ARGUMENT, "write_assoc: order must list distinct SNP indices");
            seen[j] = 1;
        }
    } else {
        rows.resize(n_snps);
        for (int64_t j = 0; j < n_snps; ++j) rows[j] = j;
    }
    AssocOut out(out_path, gzip, false);
    std::ostream& ofs = out.os();
    if (layout == CS_ASSOC_STCG)
        ofs << "CHR\tSNP\tBP\tA1\tA2\tFREQ\tN\tBETA\tSE\tP\tLOG10P\n";
    else if (layout == CS_ASSOC_SSF)
        ofs << "chromosome\tbase_pair_location\teffect_allele\tother_allele"
               "\teffect_allele_frequency\tsample_size\tbeta\tstandard_error\tp_value\tvariant_id\n";
    else
        ofs << "CHR\tSNP\tBP\tA1\tA2\tFREQ\tN"
               "\tBETA_A\tSE_A\tP_A\tLOG10P_A"
               "\tBETA_D\tSE_D\tP_D\tLOG10P_D"
               "\tP_JOINT\tLOG10P_JOINT\n";
    for (const int64_t j : rows) {
        if (tested && !tested[j]) continue;
        if (std::isnan(p[j])) continue;
        const BimRow& b = bim[j];
        if (layout == CS_ASSOC_SSF) {
            ofs << b.chrom << '\t' << b.bp << '\t' << b.a1 << '\t' << b.a2 << '\t' << freq[j]
                << '\t' << n_obs << '\t' << beta[j] << '\t' << se[j] << '\t' << p[j] << '\t'
                << b.id << '\n';
            continue;
        }
        ofs << b.chrom << '\t' << b.id << '\t' << b.bp << '\t' << b.a1 << '\t' << b.a2 << '\t'
            << freq[j] << '\t' << n_obs << '\t' << beta[j] << '\t' << se[j] << '\t' << p[j]
            << '\t' << log10p[j];
        if (layout == CS_ASSOC_STCG)
            ofs << '\n';
        else
            ofs << "\tNA\tNA\tNA\tNA\tNA\tNA\n";
    }
    out.finish();
}

void append_cosmic_sumstats(const char* path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                            const double* freq, const double* beta, const double* se,
                            const double* p, const double* log10p, const int32_t* tested,
                            const char* model, bool append, bool gzip, const char* created) {
    if (!path || !bim_path || n_snps < 0 || !freq || !beta || !se || !p || !log10p || !model)
        fail(CS_ERR_INVALID_ARGUMENT, "append_cosmic_sumstats: null argument");
    const std::vector<BimRow> bim = bim_for(bim_path, n_snps, "append_cosmic_sumstats");
    AssocOut out(path, gzip, append);
    std::ostream& ofs = out.os();
    if (!append) {
        std::string date;
        if (created) {
            date = created;
        } else {
            const std::time_t now = std::chrono::system_clock::to_time_t(std::chrono::system_clock::now());
            std::tm utc{};
            gmtime_r(&now, &utc);
            std::ostringstream ss;
            ss << std::put_time(&utc, "%Y-%m-%d %H:%M:%S UTC");
            date = ss.str();
        }
        ofs << "# CosmicScanner Summary Statistics v1.0\n"
            << "# Created: " << date << "\n";
        if (model[0]) ofs << "# Model: " << model << "\n";
        ofs << "#\n"
            << "CHR\tSNP\tPOS\tA1\tA2\tBETA\tSE\tP\tN\tAF\tLOG10P\tMODEL"
            << "\tZ\tWEIGHT\tINFO\tWARNING\n";
    }
    for (int64_t j = 0; j < n_snps; ++j) {
        if (tested && !tested[j]) continue;
        if (std::isnan(p[j])) continue;
        const BimRow& b = bim[j];
        ofs << b.chrom << '\t' << b.id << '\t' << b.bp << '\t' << b.a1 << '\t' << b.a2 << '\t'
            << std::setprecision(10) << beta[j] << '\t' << se[j] << '\t' << p[j] << '\t' << n_obs
            << '\t' << std::setprecision(6) << freq[j] << '\t' << log10p[j] << '\t' << model
            << '\t' << (se[j] > 0 ? beta[j] / se[j] : 0.0) << '\t'
            << (se[j] > 0 ? 1.0 / (se[j] * se[j]) : 0.0) << '\t' << std::setprecision(4) << 1.0
            << "\t.\n";
    }
    out.finish();
}

void write_assoc_txt(const char* out_path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                     const double* freq, const double* beta, const double* se, const double* p,
                     const double* log10p, const int32_t* tested, int stcg_columns) {
    write_assoc(out_path, bim_path, n_snps, n_obs, freq, beta, se, p, log10p, tested, nullptr, 0,
                stcg_columns ? CS_ASSOC_STCG : CS_ASSOC_UNIFIED, false);
}

void write_assoc_mv_txt(const char* out_path, const char* bim_path, int64_t n_snps, int32_t d,
                        const double* freq, const double* wald, const double* p, const double* beta,
                        const double* cov) {
    if (!out_path || !bim_path || n_snps < 0 || d < 1 || !freq || !wald || !p || !beta || !cov)
        fail(CS_ERR_INVALID_ARGUMENT, "write_assoc_mv_txt: null argument");
    const std::vector<BimRow> bim = read_bim(bim_path);
    if ((int64_t)bim.size() != n_snps)
        fail(CS_ERR_INVALID_ARGUMENT, "write_assoc_mv_txt: .bim has " + std::to_string(bim.size()) +
                                          " variants, results have " + std::to_string(n_snps));
    std::ofstream ofs(out_path);
    if (!ofs) fail(CS_ERR_IO, "Cannot open output file: " + std::string(out_path));
    ofs << "CHR\tSNP\tBP\tA1\tA2\tFREQ\tWALD_STAT\tP";
    for (int t = 0; t < d; ++t) ofs << "\tBETA_" << (t + 1) << "\tSE_" << (t + 1);
    ofs << "\n";
    for (int64_t j = 0; j < n_snps; ++j) {
        if (std::isnan(p[j])) continue;
        const BimRow& b = bim[j];
        ofs << b.chrom << '\t' << b.id << '\t' << b.bp << '\t' << b.a1 << '\t' << b.a2 << '\t'
            << freq[j] << '\t' << wald[j] << '\t' << p[j];
        for (int t = 0; t < d; ++t) {
            const double var = cov[j * d * d + t + (int64_t)t * d];
            if (!std::isfinite(var) || var < 0.0)
                fail(CS_ERR_NUMERIC, "mvLMM covariance TRUE_SINGULARITY for SNP " + b.id +
                                         ": invalid trait variance");
            ofs << '\t' << beta[j * d + t] << '\t' << std::sqrt(var);
        }
        ofs << '\n';
    }
    ofs.flush();
    if (!ofs) fail(CS_ERR_IO, "Error writing output file: " + std::string(out_path));
}

void write_scan_meta(const char* out_prefix, int32_t requested_rank, double trace_threshold,
                     bool full_eigen) {
    if (!out_prefix) fail(CS_ERR_INVALID_ARGUMENT, "write_scan_meta: null argument");
    const std::string path = std::string(out_prefix) + ".scan.meta.txt";
    std::ofstream meta(path);
    if (!meta) fail(CS_ERR_IO, "Cannot open output file: " + path);
    meta << "Item\tValue\n"
         << "analysis_model\tunivariate_lmm\n"
         << "requested_scan_tier\tlegacy_default\n"
         << "resolved_scan_tier\tapprox\n"
         << "snp_vc_strategy\tfixed_null\n"
         << "SNP_MODEL\tadditive\n"
         << "HWE_APPLIED\tfalse\n"
         << "HWE_METHOD\tNONE\n"
         << "HWE_REASON_IF_SKIPPED\tFILTER_DISABLED\n"
         << "matrix_approximation\t" << (full_eigen ? "full_eigen" : "fastlmm_auto_trace") << "\n"
         << "requested_rank\t" << (full_eigen ? 0 : requested_rank) << "\n"
         << "trace_threshold\t" << (full_eigen ? 0.0 : trace_threshold) << "\n"
         << "RANK_SELECTION\t" << (full_eigen ? "FULL" : "AUTO_TRACE") << "\n";
    meta.flush();
    if (!meta) fail(CS_ERR_IO, "Error writing output file: " + path);
}

void append_scan_common_meta(const char* out_prefix, const char* model, int64_t n, bool loco,
                             bool covariate_projection, bool vce_converged) {
    if (!out_prefix || !model) fail(CS_ERR_INVALID_ARGUMENT, "append_scan_common_meta: null argument");
    const std::string path = std::string(out_prefix) + ".scan.meta.txt";
    std::ofstream meta(path, std::ios::app);
    if (!meta) fail(CS_ERR_IO, "Cannot append GWAS scan metadata: " + path);
    meta << "MODEL\t" << model << "\n"
         << "N\t" << n << "\n"
         << "N_SEMANTICS\tanalysis_samples_after_phenotype_and_covariate_filtering;"
            "per-SNP_missing_genotypes_mean-imputed\n"
         << "FREQ_SEMANTICS\tA1_allele_frequency_(not_MAF)\n"
         << "LOCO\t" << (loco ? "true" : "false") << "\n"
         << "COVARIATE_PROJECTION\t" << (covariate_projection ? "true" : "false") << "\n"
         << "VCE_CONVERGED\t" << (vce_converged ? "true" : "false") << "\n";
    meta.flush();
    if (!meta) fail(CS_ERR_IO, "Error writing output file: " + path);
}

void write_low_rank_meta(const char* out_prefix, int32_t n_rows, const char* const* scopes,
                         const cs_lowrank_diagnostics* diags, int64_t n, double error_tol,
                         const char* const* fallbacks) {
    if (!out_prefix || n_rows < 0 || (n_rows > 0 && (!scopes || !diags)))
        fail(CS_ERR_INVALID_ARGUMENT, "write_low_rank_meta: null argument");
    const std::string path = std::string(out_prefix) + ".low_rank.meta.tsv";
    std::ofstream meta(path);
    if (!meta) fail(CS_ERR_IO, "Cannot open output file: " + path);
    meta << "SCOPE\tALGORITHM\tREQUESTED_RANK\tEFFECTIVE_RANK\tSKETCH_SIZE"
         << "\tRESIDUAL_EIGENVALUE\tRELATIVE_FROBENIUS_ERROR\tERROR_TOLERANCE"
         << "\tDECOMPOSITION_SECONDS\tESTIMATED_PEAK_BYTES"
         << "\tFULL_EIGEN_ESTIMATED_PEAK_BYTES\tSELECTED_RANK\tTOTAL_RANK"
         << "\tTRACE_FRACTION\tRANK_SELECTION\tFALLBACK\n";
    for (int32_t r = 0; r < n_rows; ++r) {
        const cs_lowrank_diagnostics& d = diags[r];
        const long long rank = d.effective_rank, sk = d.sketch_size;
        const long long peak = 8LL * (2LL * n * sk + (long long)n * rank + sk * sk);
        // one stream: the precision set before RESIDUAL_EIGENVALUE stays for the rest of the
        // row and for the following rows, as in the reference
        meta << (scopes[r] ? scopes[r] : "GLOBAL") << "\trandomized_subspace_iteration_tail_mean_woodbury"
             << "\t" << d.effective_rank << "\t" << d.effective_rank << "\t" << d.sketch_size
             << "\t" << std::setprecision(12) << d.residual_eigenvalue << "\t"
             << d.relative_frobenius_error << "\t" << error_tol << "\t" << d.seconds << "\t" << peak
             << "\t" << (24LL * n * n) << "\t" << d.effective_rank << "\t" << n << "\t"
             << d.trace_fraction << "\tMATRIX_FREE_AUTO_TRACE\t"
             << (fallbacks && fallbacks[r] ? fallbacks[r] : "none")
             << "\n";
    }
    meta.flush();
    if (!meta) fail(CS_ERR_IO, "Error writing output file: " + path);
}

}  // namespace cs
