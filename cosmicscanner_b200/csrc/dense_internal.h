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
    int64_t traits = 1;  // columns of Uty
    bool projected = false;
    DeviceBuffer<double> W;           // W_proj: n x n_eig, column-major, ld n
    std::vector<double> D, Uty, UtX;  // n_eig; n_eig x traits; n_eig x p (column-major)
    double sigma2_g = 0.0, sigma2_e = 0.0, delta = 0.0;
    bool solved = false;
};

// EigenVce::prepare's eigenbasis of G[keep, keep] with Uty = W^T Y for nt trait columns
// (dense.cu).
std::shared_ptr<DenseNull> eigen_basis(const cs_grm* grm, const int32_t* keep, int64_t n_keep,
                                       const double* Y, int64_t nt, const double* X, int64_t p,
                                       bool projection);

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

// MvEigenVce (mv_vce.cu): the eigenbasis with U'Y for d traits, the variance matrices and the
// device copies of D and U'Y that the EM / log-likelihood kernel reads.
struct cs_mv_eigen_vce {
    std::shared_ptr<cs::DenseNull> d;
    int64_t traits = 0;
    std::vector<double> Vg, Ve, Vg_se, Ve_se;  // d x d, column-major
    cs::DeviceBuffer<double> dD, dY, partial;
    int blocks = 0;
    int iterations = 0;
    bool converged = false;
    double logl = 0.0;
};
