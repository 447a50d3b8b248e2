// Input side of the association path: .fam samples, phenotype and covariate tables aligned
// to them, and the keep list of samples with complete data.  Host code with the reference's
// parsing rules, so that a caller can feed the engines exactly what the reference would:
//  * .fam: PlinkReader::readFam (libCosmicCore/src/plink_reader.cpp:34-48): whitespace
//    fields FID IID father mother sex phenotype; empty lines skipped; none -> error.
//  * phenotypes: PhenoReader::load / align (libCosmicCore/src/pheno_reader.cpp:13-61,
//    138-187): rows keyed "FID:IID", the col_idx-th value after FID IID, NA spellings and
//    the missing code (|v - code| < 1e-6) -> NaN, unparsable -> NaN, later duplicates win;
//    align refuses a constant trait (zero variance over >= 2 finite matched values).
//    loadMatrix / alignMatrix (:63-125, 189-215): every value after FID IID read as double
//    until the first non-number, missing code within 1e-8 -> NaN, 1-based column selection
//    (absent column -> NaN), rows with a different count than the first are skipped.
//  * quantitative covariates: CovarReader::load (libCosmicCore/src/covar_reader.cpp:19-62):
//    values read as float until the first non-number (FP32 semantics), missing code within
//    1e-8 -> NaN, rows with a different count than the first are skipped.
//  * categorical covariates: CovarReader::loadCategorical (:64-176): per column the sorted
//    set of levels (missing token excluded); the first level is the reference and every
//    other level gets a 0/1 dummy column; a missing token makes the column's dummies NaN;
//    one-level columns give no column.
//  * covariate alignment: CovarReader::align (:468-500): NaN for unmatched samples.
//  * design: DataLoader::loadCovariates (src/data_loader.h:219-261): [1 | quantitative |
//    categorical dummies] as float.
//  * keep list: DataFilter::filterSamples (libCosmicCore/src/data_filter.h:21-41): samples
//    whose phenotype is NaN or any covariate is NaN are dropped.
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "cs_internal.h"
#include "input_internal.h"

namespace cs {

namespace {

std::string key_of(const std::string& fid, const std::string& iid) { return fid + ":" + iid; }

// std::stod semantics: a leading number (whitespace skipped, trailing text ignored), or no
// conversion at all
bool parse_double(const std::string& s, double& v) {
    const char* b = s.c_str();
    char* e = nullptr;
    v = std::strtod(b, &e);
    return e != b;
}

}  // namespace

std::vector<FamRecord> read_fam(const std::string& path) {
    std::ifstream ifs(path);
    if (!ifs) fail(CS_ERR_IO, "Cannot open .fam file: " + path);
    std::vector<FamRecord> out;
    std::string line;
    while (std::getline(ifs, line)) {
        if (line.empty()) continue;
        std::stringstream ss(line);
        FamRecord r;
        // a field that does not parse leaves the stream failed: sex / phenotype read as 0
        ss >> r.fid >> r.iid >> r.father >> r.mother >> r.sex >> r.phenotype;
        out.push_back(std::move(r));
    }
    if (out.empty()) fail(CS_ERR_INVALID_ARGUMENT, "No samples found in .fam file");
    return out;
}

void PhenoTable::load(const std::string& path, int col_idx, double missing) {
    values.clear();
    std::ifstream ifs(path);
    if (!ifs) fail(CS_ERR_IO, "Cannot open phenotype file: " + path);
    std::string line;
    while (std::getline(ifs, line)) {
        if (line.empty()) continue;
        std::stringstream ss(line);
        std::string fid, iid;
        ss >> fid >> iid;
        if (fid.empty() || iid.empty()) continue;
        std::string tok;
        bool found = false;
        for (int i = 0; i < col_idx; ++i) {
            if (!(ss >> tok)) {
                found = false;
                break;
            }
            found = true;
        }
        if (!found) continue;
        double v = NAN;
        if (tok == "NA" || tok == "na" || tok == "NaN" || tok == "nan" || tok == "NAN") {
            v = NAN;
        } else if (!parse_double(tok, v)) {
            v = NAN;
        }
        if (std::isnan(v) || std::abs(v - missing) < 1e-6) v = NAN;
        values[key_of(fid, iid)] = v;
    }
}

int64_t PhenoTable::align(const std::vector<FamRecord>& fam, double* y) const {
    int64_t matched = 0;
    for (size_t i = 0; i < fam.size(); ++i) {
        auto it = values.find(key_of(fam[i].fid, fam[i].iid));
        y[i] = it == values.end() ? NAN : it->second;
        if (!std::isnan(y[i])) ++matched;
    }
    double sum = 0.0, sum_sq = 0.0;
    int64_t finite = 0;
    for (size_t i = 0; i < fam.size(); ++i) {
        if (!std::isfinite(y[i])) continue;
        sum += y[i];
        sum_sq += y[i] * y[i];
        ++finite;
    }
    if (finite >= 2) {
        const double mean = sum / (double)finite, mean_sq = sum_sq / (double)finite;
        if (!(mean_sq - mean * mean > 1e-12))
            fail(CS_ERR_INVALID_ARGUMENT,
                 "Phenotype has zero variance across " + std::to_string(finite) +
                     " finite matched samples (every observed value is identical to " +
                     std::to_string(mean) +
                     "). Association tests are not estimable for a constant trait; check the "
                     "phenotype column (--mpheno) and the sample matching.");
    }
    return matched;
}

void PhenoTable::load_matrix(const std::string& path, const std::vector<int>& cols, double missing) {
    rows.clear();
    n_traits = 0;
    std::ifstream ifs(path);
    if (!ifs) fail(CS_ERR_IO, "Cannot open phenotype file: " + path);
    std::string line;
    while (std::getline(ifs, line)) {
        if (line.empty()) continue;
        std::stringstream ss(line);
        std::string fid, iid;
        ss >> fid >> iid;
        if (fid.empty() || iid.empty()) continue;
        std::vector<double> all, vals;
        double v;
        while (ss >> v) all.push_back(std::abs(v - missing) < 1e-8 ? NAN : v);
        if (cols.empty()) {
            vals = all;
        } else {
            for (int c : cols) {
                const int idx = c - 1;
                vals.push_back(idx >= 0 && idx < (int)all.size() ? all[idx] : NAN);
            }
        }
        if (n_traits == 0) {
            n_traits = (int)vals.size();
        } else if ((int)vals.size() != n_traits) {
            continue;  // a row with a different column count is skipped
        }
        rows[key_of(fid, iid)] = vals;
    }
}

int64_t PhenoTable::align_matrix(const std::vector<FamRecord>& fam, double* Y, int64_t ld) const {
    int64_t matched = 0;
    for (size_t i = 0; i < fam.size(); ++i) {
        auto it = rows.find(key_of(fam[i].fid, fam[i].iid));
        const bool found = it != rows.end() && (int)it->second.size() == n_traits;
        bool complete = found;
        for (int t = 0; t < n_traits; ++t) {
            const double v = found ? it->second[t] : NAN;
            Y[i + (int64_t)t * ld] = v;
            if (std::isnan(v)) complete = false;
        }
        if (complete) ++matched;
    }
    return matched;
}

void CovarTable::load(const std::string& path, double missing) {
    rows.clear();
    n_cols = 0;
    std::ifstream ifs(path);
    if (!ifs) fail(CS_ERR_IO, "Cannot open covariate file: " + path);
    std::string line;
    while (std::getline(ifs, line)) {
        if (line.empty()) continue;
        std::stringstream ss(line);
        std::string fid, iid;
        ss >> fid >> iid;
        if (fid.empty() || iid.empty()) continue;
        std::vector<float> vals;
        float v;
        while (ss >> v) vals.push_back(std::abs(v - missing) < 1e-8 ? NAN : v);
        // the count comes from the first row with any value (a header row has none)
        if (n_cols == 0) {
            n_cols = (int)vals.size();
        } else if ((int)vals.size() != n_cols) {
            continue;  // a row with a different column count is skipped
        }
        rows[key_of(fid, iid)] = vals;
    }
}

void CovarTable::load_categorical(const std::string& path, const std::string& missing) {
    rows.clear();
    n_cols = 0;
    std::ifstream ifs(path);
    if (!ifs) fail(CS_ERR_IO, "Cannot open covariate file: " + path);
    std::vector<std::map<std::string, int>> levels;
    std::vector<std::vector<std::string>> raw;
    std::vector<std::string> keys;
    std::string line;
    while (std::getline(ifs, line)) {
        if (line.empty()) continue;
        std::stringstream ss(line);
        std::string fid, iid;
        ss >> fid >> iid;
        if (fid.empty() || iid.empty()) continue;
        std::vector<std::string> toks;
        std::string tok;
        while (ss >> tok) toks.push_back(tok);
        if (levels.empty()) {
            levels.resize(toks.size());
        } else if (toks.size() != levels.size()) {
            continue;  // a row with a different column count is skipped
        }
        for (size_t c = 0; c < toks.size(); ++c)
            if (toks[c] != missing) levels[c][toks[c]]++;
        raw.push_back(std::move(toks));
        keys.push_back(key_of(fid, iid));
    }
    std::vector<int> offset(levels.size(), 0);
    int acc = 0;
    for (size_t c = 0; c < levels.size(); ++c) {
        offset[c] = acc;
        const int k = (int)levels[c].size();
        if (k > 1) acc += k - 1;
    }
    n_cols = acc;
    for (size_t r = 0; r < raw.size(); ++r) {
        std::vector<float> enc(n_cols, 0.0f);
        for (size_t c = 0; c < raw[r].size(); ++c) {
            const int k = (int)levels[c].size();
            if (k <= 1) continue;
            const std::string& v = raw[r][c];
            if (v == missing) {
                for (int d = 0; d < k - 1; ++d) enc[offset[c] + d] = NAN;
                continue;
            }
            auto it = levels[c].begin();
            if (v == it->first) continue;  // the reference level: all dummies 0
            ++it;
            for (int idx = 0; it != levels[c].end(); ++it, ++idx)
                if (it->first == v) {
                    enc[offset[c] + idx] = 1.0f;
                    break;
                }
        }
        rows[keys[r]] = std::move(enc);
    }
}

int64_t CovarTable::align(const std::vector<FamRecord>& fam, float* X, int64_t ld) const {
    int64_t matched = 0;
    for (size_t i = 0; i < fam.size(); ++i) {
        auto it = rows.find(key_of(fam[i].fid, fam[i].iid));
        // a row stored before the column count was known (no values) matches nothing
        const bool found = it != rows.end() && (int)it->second.size() == n_cols;
        bool complete = found;
        for (int c = 0; c < n_cols; ++c) {
            const float v = found ? it->second[c] : NAN;
            X[i + (int64_t)c * ld] = v;
            if (std::isnan(v)) complete = false;
        }
        if (complete && n_cols > 0) ++matched;
    }
    return matched;
}

int64_t filter_samples(const double* y, int64_t n, const float* X, int64_t ldx, int32_t p,
                       int32_t* keep) {
    int64_t kept = 0;
    for (int64_t i = 0; i < n; ++i) {
        bool ok = !std::isnan(y[i]);
        for (int32_t j = 0; ok && j < p; ++j)
            if (std::isnan(X[i + (int64_t)j * ldx])) ok = false;
        if (ok) keep[kept++] = (int32_t)i;
    }
    return kept;
}

}  // namespace cs
