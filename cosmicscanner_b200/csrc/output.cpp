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
#include <cmath>
#include <fstream>
#include <iomanip>
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

}  // namespace

void write_assoc_txt(const char* out_path, const char* bim_path, int64_t n_snps, int32_t n_obs,
                     const double* freq, const double* beta, const double* se, const double* p,
                     const double* log10p, const int32_t* tested, int stcg_columns) {
    if (!out_path || !bim_path || n_snps < 0 || !freq || !beta || !se || !p || !log10p)
        fail(CS_ERR_INVALID_ARGUMENT, "write_assoc_txt: null argument");
    const std::vector<BimRow> bim = read_bim(bim_path);
    if ((int64_t)bim.size() != n_snps)
        fail(CS_ERR_INVALID_ARGUMENT, "write_assoc_txt: .bim has " + std::to_string(bim.size()) +
                                          " variants, results have " + std::to_string(n_snps));
    std::ofstream ofs(out_path);
    if (!ofs) fail(CS_ERR_IO, "Cannot open output file: " + std::string(out_path));
    if (stcg_columns)
        ofs << "CHR\tSNP\tBP\tA1\tA2\tFREQ\tN\tBETA\tSE\tP\tLOG10P\n";
    else
        ofs << "CHR\tSNP\tBP\tA1\tA2\tFREQ\tN"
               "\tBETA_A\tSE_A\tP_A\tLOG10P_A"
               "\tBETA_D\tSE_D\tP_D\tLOG10P_D"
               "\tP_JOINT\tLOG10P_JOINT\n";
    for (int64_t j = 0; j < n_snps; ++j) {
        if (tested && !tested[j]) continue;
        if (std::isnan(p[j])) continue;
        const BimRow& b = bim[j];
        ofs << b.chrom << '\t' << b.id << '\t' << b.bp << '\t' << b.a1 << '\t' << b.a2 << '\t'
            << freq[j] << '\t' << n_obs << '\t' << beta[j] << '\t' << se[j] << '\t' << p[j]
            << '\t' << log10p[j];
        if (stcg_columns)
            ofs << '\n';
        else
            ofs << "\tNA\tNA\tNA\tNA\tNA\tNA\n";
    }
    ofs.flush();
    if (!ofs) fail(CS_ERR_IO, "Error writing output file: " + std::string(out_path));
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

void write_scan_meta(const char* out_prefix, int32_t requested_rank, double trace_threshold) {
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
         << "matrix_approximation\tfastlmm_auto_trace\n"
         << "requested_rank\t" << requested_rank << "\n"
         << "trace_threshold\t" << trace_threshold << "\n"
         << "RANK_SELECTION\tAUTO_TRACE\n";
    meta.flush();
    if (!meta) fail(CS_ERR_IO, "Error writing output file: " + path);
}

void write_low_rank_meta(const char* out_prefix, int32_t n_rows, const char* const* scopes,
                         const cs_lowrank_diagnostics* diags, int64_t n, double error_tol,
                         const char* fallback) {
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
             << d.trace_fraction << "\tMATRIX_FREE_AUTO_TRACE\t" << (fallback ? fallback : "none")
             << "\n";
    }
    meta.flush();
    if (!meta) fail(CS_ERR_IO, "Error writing output file: " + path);
}

}  // namespace cs
