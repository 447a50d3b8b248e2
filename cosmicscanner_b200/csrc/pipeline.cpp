// The matrix-free LMM job orchestrated in C++ behind the C ABI, as GwasScanner::runLocoScan
// runs its PLINK matrix-free branch (src/gwas_scanner.cpp:74-509):
//   * GRM variant selection from the all-sample statistics (:258-277): 1/sd != 0 and
//     MAF >= --maf (and not numerically 0);
//   * one null model over every selected variant (--no-loco or a single chromosome), or the
//     leave-one-chromosome-out loop (:299-314, 464-472): per chromosome in sort_chrom_labels
//     order (:62-72), an operator without that chromosome's GRM variants, its own null model,
//     and the scan of that chromosome's SNPs (contiguous runs of the .bim order);
//   * each null model the low-rank sketch with trace-fraction rank selection; a sketch that
//     misses the trace threshold (unless --fastlmm-no-fallback) or whose relative Frobenius
//     error exceeds --lmm-low-rank-error-tol falls back to the same sketch at the fixed
//     requested rank (MatrixFreeVce, :347-383, src/matrix_free_vce.cpp:32-236), keeping the
//     first sketch's diagnostics with the fallback label;
//   * cs_run_gwas_lmm adds the input side (.fam, phenotype, covariates, keep list:
//     src/models/univariate_model.cpp:389-426) and the result files (.assoc.txt,
//     .cosmic.sumstats, .scan.meta.txt, .low_rank.meta.tsv).
// Everything goes through the library's own C ABI; a failing call ends the job with its
// status and message.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "cs_internal.h"

namespace {

void ok(int status) {
    if (status != CS_OK) cs::fail(status, cs_last_error());
}

std::vector<std::string> sort_chrom_labels(const std::set<std::string>& labels) {
    std::vector<std::string> out(labels.begin(), labels.end());
    std::sort(out.begin(), out.end(), [](const std::string& a, const std::string& b) {
        try {
            return std::stoi(a) < std::stoi(b);
        } catch (...) {
            return a < b;
        }
    });
    return out;
}

struct Handles {
    cs_kinship* op = nullptr;
    cs_lmm* lmm = nullptr;
    ~Handles() {
        if (lmm) cs_lmm_destroy(lmm);
        if (op) cs_kinship_destroy(op);
    }
};

// The null model of one scope with the reference's fall-back rule.
cs_lmm_run_scope prepare_with_fallback(cs_lmm* lmm, cs_kinship* op, int64_t n, const double* y,
                                       const double* X, int64_t p, const cs_lmm_run_options& o) {
    const int rank = (int)std::max<int64_t>(1, std::min<int64_t>(o.rank, n - 1));
    cs_lmm_run_scope sc{};
    ok(cs_lmm_prepare_lowrank_matrix_free(lmm, op, y, X, p, rank, o.oversample, o.seed,
                                          o.trace_threshold, o.min_rank, o.precision, &sc.diag));
    bool accepted = sc.diag.relative_frobenius_error <= o.error_tol;
    sc.fallback = CS_FALLBACK_NONE;
    if (!sc.diag.trace_threshold_met) {
        if (!o.no_fallback) {
            accepted = false;
            sc.fallback = CS_FALLBACK_TRACE_THRESHOLD;
        }
    } else if (!accepted) {
        sc.fallback = CS_FALLBACK_ERROR_TOLERANCE;
    }
    if (!accepted) {
        cs_lowrank_diagnostics refit{};
        ok(cs_lmm_prepare_lowrank_matrix_free(lmm, op, y, X, p, rank, o.oversample, o.seed, 0.0,
                                              o.min_rank, o.precision, &refit));
        sc.diag.sigma2_g = refit.sigma2_g;
        sc.diag.sigma2_e = refit.sigma2_e;
        sc.diag.delta = refit.delta;
        sc.diag.log_eta = refit.log_eta;
        sc.diag.reml_objective = refit.reml_objective;
    }
    return sc;
}

void set_label(cs_lmm_run_scope& sc, const std::string& label) {
    std::memset(sc.label, 0, sizeof(sc.label));
    std::strncpy(sc.label, label.c_str(), sizeof(sc.label) - 1);
}

// The job over host arrays; returns the scopes (one, or one per chromosome under LOCO).
std::vector<cs_lmm_run_scope> run_matrix_free(const cs_genotypes* g, const int32_t* keep,
                                              int64_t n_keep, const double* y, const double* X,
                                              int64_t p, const char* const* chrom,
                                              const cs_lmm_run_options& o, double* beta,
                                              double* se, double* pvalue, double* log10p,
                                              double* freq, int32_t* tested) {
    int64_t N = 0, M = 0;
    ok(cs_genotypes_info(g, &N, &M, nullptr));
    std::vector<int32_t> all_keep;
    if (!keep || n_keep <= 0) {
        all_keep.resize(N);
        for (int64_t i = 0; i < N; ++i) all_keep[i] = (int32_t)i;
        keep = all_keep.data();
        n_keep = N;
    }
    const bool subset = all_keep.empty();  // the caller's keep list (may still be 0..N-1)
    // GRM variant selection (src/gwas_scanner.cpp:258-277)
    std::vector<double> mean(M), inv_std(M);
    ok(cs_genotypes_stats(g, mean.data(), inv_std.data(), nullptr, nullptr));
    std::vector<int32_t> variants;
    for (int64_t j = 0; j < M; ++j) {
        const double f = mean[j] / 2.0, maf = std::min(f, 1.0 - f);
        if (inv_std[j] != 0.0 && !(maf < o.min_maf) && !(std::abs(maf) < 1e-8))
            variants.push_back((int32_t)j);
    }
    if (variants.empty()) cs::fail(CS_ERR_INVALID_ARGUMENT, "Matrix-free GRM selection produced no variants");
    for (int64_t j = 0; j < M; ++j) {
        if (beta) beta[j] = NAN;
        if (se) se[j] = NAN;
        if (pvalue) pvalue[j] = NAN;
        if (log10p) log10p[j] = NAN;
        if (freq) freq[j] = NAN;
        if (tested) tested[j] = 0;
    }
    auto label_of = [&](int64_t j) { return std::string(chrom && chrom[j] ? chrom[j] : ""); };
    std::set<std::string> labels;
    if (chrom)
        for (int64_t j = 0; j < M; ++j) labels.insert(label_of(j));
    std::vector<cs_lmm_run_scope> scopes;
    if (!(o.loco && labels.size() > 1)) {
        Handles h;
        ok(cs_kinship_create(g, subset ? keep : nullptr, subset ? n_keep : 0, variants.data(),
                             (int64_t)variants.size(), &h.op));
        ok(cs_lmm_create(&h.lmm));
        cs_lmm_run_scope sc = prepare_with_fallback(h.lmm, h.op, n_keep, y, X, p, o);
        set_label(sc, "GLOBAL");
        ok(cs_lmm_scan(h.lmm, g, keep, n_keep, o.min_maf, o.precision, beta, se, pvalue, log10p,
                       freq, tested));
        scopes.push_back(sc);
        return scopes;
    }
    for (const std::string& c : sort_chrom_labels(labels)) {
        std::vector<int32_t> loco;
        for (int32_t j : variants)
            if (c != label_of(j)) loco.push_back(j);
        if (loco.empty())
            cs::fail(CS_ERR_INVALID_ARGUMENT, "Matrix-free LOCO left no GRM variants for chromosome " + c);
        Handles h;
        ok(cs_kinship_create(g, subset ? keep : nullptr, subset ? n_keep : 0, loco.data(),
                             (int64_t)loco.size(), &h.op));
        ok(cs_lmm_create(&h.lmm));
        cs_lmm_run_scope sc = prepare_with_fallback(h.lmm, h.op, n_keep, y, X, p, o);
        set_label(sc, c);
        // the chromosome's SNPs as contiguous runs of the .bim order
        int64_t j = 0;
        while (j < M) {
            if (c != label_of(j)) {
                ++j;
                continue;
            }
            int64_t e = j + 1;
            while (e < M && c == label_of(e)) ++e;
            auto at = [&](double* a) { return a ? a + j : nullptr; };
            ok(cs_lmm_scan_window(h.lmm, g, keep, n_keep, j, e, o.min_maf, o.precision, at(beta),
                                  at(se), at(pvalue), at(log10p), at(freq),
                                  tested ? tested + j : nullptr));
            j = e;
        }
        scopes.push_back(sc);
    }
    return scopes;
}

const char* fallback_name(int32_t f) {
    return f == CS_FALLBACK_TRACE_THRESHOLD ? "trace_threshold"
           : f == CS_FALLBACK_ERROR_TOLERANCE ? "error_tolerance"
                                              : "none";
}

std::vector<std::string> read_bim_chrom(const std::string& path) {
    std::ifstream f(path);
    if (!f) cs::fail(CS_ERR_IO, "Cannot open BIM file: " + path);
    std::vector<std::string> out;
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        std::string c;
        if (ss >> c) out.push_back(c);
    }
    return out;
}

}  // namespace

extern "C" {

void cs_lmm_run_default_options(cs_lmm_run_options* o) {
    if (!o) return;
    o->rank = 256;
    o->oversample = 10;
    o->seed = 42;
    o->trace_threshold = 0.95;
    o->min_rank = 1;
    o->min_maf = 0.01;
    o->precision = CS_PRECISION_MIXED;
    o->loco = 1;
    o->no_fallback = 1;
    o->error_tol = 1.0;
}

int cs_run_lmm_matrix_free(const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                           const double* y, const double* X, int64_t p, const char* const* chrom,
                           const cs_lmm_run_options* opt, double* beta, double* se,
                           double* pvalue, double* log10p, double* freq, int32_t* tested,
                           cs_lmm_run_scope* scopes, int32_t max_scopes, int32_t* n_scopes) {
    try {
        if (!g || !y || (p > 0 && !X)) cs::fail(CS_ERR_INVALID_ARGUMENT, "null argument");
        cs_lmm_run_options o;
        if (opt) o = *opt;
        else cs_lmm_run_default_options(&o);
        const auto sc = run_matrix_free(g, keep, n_keep, y, X, p, chrom, o, beta, se, pvalue,
                                        log10p, freq, tested);
        if (n_scopes) *n_scopes = (int32_t)sc.size();
        if (scopes)
            for (size_t i = 0; i < sc.size() && (int32_t)i < max_scopes; ++i) scopes[i] = sc[i];
        return CS_OK;
    } catch (const cs::Error& e) {
        cs::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        cs::set_last_error(e.what());
        return CS_ERR_CUDA;
    }
}

void cs_gwas_lmm_default_options(cs_gwas_lmm_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->mpheno = 1;
    o->missing_code = -9.0;
    cs_lmm_run_default_options(&o->run);
}

int cs_run_gwas_lmm(const cs_gwas_lmm_options* opt, int64_t* n_kept, int32_t* n_scopes) {
    try {
        if (!opt || !opt->bfile || !opt->out) cs::fail(CS_ERR_INVALID_ARGUMENT, "bfile and out are required");
        const std::string bfile = opt->bfile, out = opt->out;
        // ---- inputs (UnivariateModel::prepare with the DataLoader route)
        cs_samples* samples = nullptr;
        ok(cs_fam_read((bfile + ".fam").c_str(), &samples));
        struct SamplesGuard {
            cs_samples* s;
            ~SamplesGuard() { cs_samples_destroy(s); }
        } sg{samples};
        int64_t N = 0;
        ok(cs_samples_count(samples, &N));
        std::vector<double> y(N);
        if (opt->pheno) {
            cs_pheno* ph = nullptr;
            ok(cs_pheno_load(opt->pheno, opt->mpheno, opt->missing_code, &ph));
            int64_t matched = 0;
            const int rc = cs_pheno_align(ph, samples, y.data(), &matched);
            cs_pheno_destroy(ph);
            ok(rc);
        } else {
            ok(cs_samples_fam_phenotype(samples, y.data()));
        }
        std::vector<std::vector<float>> cols{std::vector<float>(N, 1.0f)};
        auto add_covar = [&](const char* path, bool categorical) {
            cs_covar* cv = nullptr;
            ok(categorical ? cs_covar_load_categorical(path, "NA", &cv)
                           : cs_covar_load(path, opt->missing_code, &cv));
            int32_t pc = 0;
            int rc = cs_covar_columns(cv, &pc);
            std::vector<float> Xc((size_t)N * std::max(pc, 1));
            int64_t matched = 0;
            if (rc == CS_OK) rc = cs_covar_align(cv, samples, Xc.data(), N, &matched);
            cs_covar_destroy(cv);
            ok(rc);
            for (int32_t a = 0; a < pc; ++a)
                cols.emplace_back(Xc.begin() + (int64_t)a * N, Xc.begin() + (int64_t)(a + 1) * N);
        };
        if (opt->qcovar) add_covar(opt->qcovar, false);
        if (opt->covar) add_covar(opt->covar, true);
        const int32_t p = (int32_t)cols.size();
        std::vector<float> Xf((size_t)N * p);
        for (int32_t a = 0; a < p; ++a) std::copy(cols[a].begin(), cols[a].end(), Xf.begin() + (int64_t)a * N);
        std::vector<int32_t> keep(N);
        int64_t nk = 0;
        ok(cs_filter_samples(y.data(), N, Xf.data(), N, p, keep.data(), &nk));
        keep.resize(nk);
        if (nk < 10) cs::fail(CS_ERR_INVALID_ARGUMENT, "Too few valid samples.");
        std::vector<double> yk(nk), Xk((size_t)nk * p);
        for (int64_t i = 0; i < nk; ++i) {
            yk[i] = y[keep[i]];
            for (int32_t a = 0; a < p; ++a) Xk[i + a * nk] = (double)Xf[keep[i] + (int64_t)a * N];
        }
        // ---- genotypes and the job
        cs_genotypes* g = nullptr;
        ok(cs_genotypes_open_plink(bfile.c_str(), &g));
        struct GenoGuard {
            cs_genotypes* g;
            ~GenoGuard() { cs_genotypes_destroy(g); }
        } gg{g};
        int64_t Ng = 0, M = 0;
        ok(cs_genotypes_info(g, &Ng, &M, nullptr));
        if (Ng != N) cs::fail(CS_ERR_INVALID_ARGUMENT, ".fam and .bed sample counts differ");
        const std::vector<std::string> chrom = read_bim_chrom(bfile + ".bim");
        if ((int64_t)chrom.size() != M) cs::fail(CS_ERR_FORMAT, ".bim and .bed SNP counts differ");
        std::vector<const char*> cptr(M);
        for (int64_t j = 0; j < M; ++j) cptr[j] = chrom[j].c_str();
        std::vector<double> beta(M), se(M), pv(M), l10(M), fr(M);
        std::vector<int32_t> tested(M);
        const auto scopes = run_matrix_free(g, keep.data(), nk, yk.data(), Xk.data(), p,
                                            cptr.data(), opt->run, beta.data(), se.data(),
                                            pv.data(), l10.data(), fr.data(), tested.data());
        const bool used_loco = scopes.size() > 1 || std::strcmp(scopes[0].label, "GLOBAL") != 0;
        // ---- result files (src/gwas_scanner.cpp:95-116, 408-428, 449-453, 499-509)
        ok(cs_write_scan_meta(out.c_str(), opt->run.rank, opt->run.trace_threshold));
        std::vector<const char*> labels, fallbacks;
        std::vector<cs_lowrank_diagnostics> diags;
        for (const auto& sc : scopes) {
            labels.push_back(sc.label);
            fallbacks.push_back(fallback_name(sc.fallback));
            diags.push_back(sc.diag);
        }
        ok(cs_write_low_rank_meta(out.c_str(), (int32_t)scopes.size(), labels.data(), diags.data(),
                                  nk, opt->run.error_tol, fallbacks.data()));
        std::vector<int64_t> order;
        for (size_t s = 0; s < scopes.size(); ++s) {
            std::vector<int32_t> part(M, 0);
            for (int64_t j = 0; j < M; ++j)
                if (!used_loco || chrom[j] == scopes[s].label) {
                    part[j] = tested[j];
                    order.push_back(j);
                }
            ok(cs_append_cosmic_sumstats((out + ".cosmic.sumstats").c_str(), (bfile + ".bim").c_str(),
                                         M, (int32_t)nk, fr.data(), beta.data(), se.data(), pv.data(),
                                         l10.data(), part.data(), "LMM", s > 0 ? 1 : 0,
                                         opt->out_gz ? 1 : 0, opt->created));
        }
        ok(cs_write_assoc((out + ".assoc.txt").c_str(), (bfile + ".bim").c_str(), M, (int32_t)nk,
                          fr.data(), beta.data(), se.data(), pv.data(), l10.data(), tested.data(),
                          order.data(), (int64_t)order.size(),
                          opt->out_ssf ? CS_ASSOC_SSF : CS_ASSOC_UNIFIED, opt->out_gz ? 1 : 0));
        ok(cs_append_scan_common_meta(out.c_str(), "additive", nk, used_loco ? 1 : 0, 1, 1));
        if (n_kept) *n_kept = nk;
        if (n_scopes) *n_scopes = (int32_t)scopes.size();
        return CS_OK;
    } catch (const cs::Error& e) {
        cs::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        cs::set_last_error(e.what());
        return CS_ERR_CUDA;
    }
}

}  // extern "C"
