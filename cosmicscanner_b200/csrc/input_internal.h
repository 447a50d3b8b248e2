// Host-side tables of the input stage (input.cpp): .fam records, phenotype and covariate
// tables keyed "FID:IID", aligned to the .fam order.
#pragma once
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

namespace cs {

struct FamRecord {
    std::string fid, iid, father, mother;
    int sex = 0;
    double phenotype = 0.0;
};
std::vector<FamRecord> read_fam(const std::string& path);

struct PhenoTable {
    std::unordered_map<std::string, double> values;             // single trait (load)
    std::unordered_map<std::string, std::vector<double>> rows;  // several traits (load_matrix)
    int n_traits = 0;
    void load(const std::string& path, int col_idx, double missing);
    int64_t align(const std::vector<FamRecord>& fam, double* y) const;
    void load_matrix(const std::string& path, const std::vector<int>& cols, double missing);
    int64_t align_matrix(const std::vector<FamRecord>& fam, double* Y, int64_t ld) const;
};

struct CovarTable {
    std::unordered_map<std::string, std::vector<float>> rows;
    int n_cols = 0;
    void load(const std::string& path, double missing);
    void load_categorical(const std::string& path, const std::string& missing);
    int64_t align(const std::vector<FamRecord>& fam, float* X, int64_t ld) const;
};

int64_t filter_samples(const double* y, int64_t n, const float* X, int64_t ldx, int32_t p,
                       int32_t* keep);

}  // namespace cs

struct cs_samples {
    std::vector<cs::FamRecord> fam;
};
struct cs_pheno {
    cs::PhenoTable table;
};
struct cs_covar {
    cs::CovarTable table;
};
