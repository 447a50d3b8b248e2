// Dense exact tier (dense.cu): the genomic relationship matrix built from the packed
// genotypes (GrmBuilder), its eigenbasis with the covariates projected out (EigenVce) and
// the Brent null model (VCESolver::solveDiagonal), shared with the exact scan of the LMM
// engine (lowrank.cu).
#pragma once
#include <cstdint>
#include <memory>
#include <vector>

#include "cs_internal.h"

namespace cs {

// EigenVce's outputs as LmmEngine::prepareFromVce takes them (src/lmm_engine.cpp:716-725).
struct DenseNull {
    int64_t n = 0;      // analysed samples
    int64_t n_eig = 0;  // n - p with the covariate projection, else n
    int64_t p = 0;      // columns of UtX (0 with the projection)
    bool projected = false;
    DeviceBuffer<double> W;           // W_proj: n x n_eig, column-major, ld n
    std::vector<double> D, Uty, UtX;  // n_eig; n_eig; n_eig x p column-major
    double sigma2_g = 0.0, sigma2_e = 0.0, delta = 0.0;
    bool solved = false;
};

}  // namespace cs

struct cs_grm {
    int64_t n = 0;        // samples (rows of the .fam for a built matrix)
    int64_t n_valid = 0;  // variants that passed the filters
    double sum_2pq = 0.0;  // GrmBuilder::getSum2pq
    double div = 1.0;      // the normalisation applied: G = (sum Z Z^T) / div
    int algorithm = 1;
    cs::DeviceBuffer<double> G;  // n x n, column-major, both triangles
};

struct cs_eigen_vce {
    std::shared_ptr<cs::DenseNull> d;
    cs_eigen_vce_result result{};
};
