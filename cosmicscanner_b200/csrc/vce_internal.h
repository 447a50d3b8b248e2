// Internal pieces of the matrix-free variance-component engine (pcg.cu, stcg.cu).
//
// Vectors are row-major blocks: row i of an (n x ld) block holds the k right-hand sides of
// sample (or record) i, so the kinship operator consumes them without a transpose.
#pragma once
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <vector>

#include "cs_internal.h"

namespace cs {

inline void check_blas_status(cublasStatus_t st, const char* what) {
    if (st != CUBLAS_STATUS_SUCCESS)
        fail(CS_ERR_CUDA, std::string(what) + ": cuBLAS status " + std::to_string((int)st));
}
#define CS_BLAS(call) ::cs::check_blas_status((call), #call)

inline void check_solver_status(cusolverStatus_t st, const char* what) {
    if (st != CUSOLVER_STATUS_SUCCESS)
        fail(CS_ERR_CUDA, std::string(what) + ": cuSOLVER status " + std::to_string((int)st));
}
#define CS_SOLVER(call) ::cs::check_solver_status((call), #call)

// One cuBLAS and one cuSOLVER handle per (thread, device), created on first use and kept for
// the process.
cublasHandle_t shared_blas();
cusolverDnHandle_t shared_solver();

// Records -> genotype rows (libCosmicCore/src/stcg_vce.cpp:17-38, 64-78).  Identity when
// every record is its own genotype row, in order.
struct RecordMap {
    int64_t n_rec = 0, n_rows = 0;
    bool identity = true;
    std::vector<int32_t> rec_to_row;                  // host copy, -1 = no genotype row
    DeviceBuffer<int32_t> d_rec_to_row, d_row_ptr, d_row_recs;  // CSR by row, records ascending
    void build(const int32_t* rec_to_row_host, int64_t n_rec, int64_t n_rows);
};

// V = vg * Zr K Zr^T + vpe * Zr Zr^T + ve * I on record-level blocks, with
// K = Z Z^T / divisor (stcg_vce.cpp:80-115).
struct VOperator {
    cs_kinship* op = nullptr;
    const RecordMap* rm = nullptr;
    double fac = 1.0;  // op->num_variants / divisor
    double vg = 0.0, vpe = 0.0, ve = 0.0;
    bool with_pe = false;
    int precision = CS_PRECISION_FP64;
    DeviceBuffer<double> u, ku;
    int64_t applies = 0;     // kinship applies issued
    int64_t apply_cols = 0;  // right-hand sides they carried

    // out (n_rec x ldo) = V * in (n_rec x ldi), k columns.
    void apply(const double* in, int64_t ldi, int64_t k, double* out, int64_t ldo, cudaStream_t s);
    // g_out = Zr K Zr^T in (dV/d sigma2_g); pe_out (optional) = Zr Zr^T in.
    void derivatives(const double* in, int64_t ldi, int64_t k, double* g_out, int64_t ldg,
                     double* pe_out, int64_t ldp, cudaStream_t s);
    // rows_out (n_rows x ldo) = K Zr^T in: the genetic solution at genotype rows.
    void genetic_rows(const double* in, int64_t ldi, int64_t k, double* rows_out, int64_t ldo,
                      double* zt_out, int64_t ldz, cudaStream_t s);

   private:
    const double* gather(const double* in, int64_t ldi, int64_t k, cudaStream_t s);
};

// Low-rank deflation preconditioner for V = vg K + ve I on single-record blocks: with the
// top r eigenpairs (U, lambda) of K from a randomized sketch and the tail mean r0 standing in
// for the rest of the spectrum, M = vg (U diag(lambda) U^T + r0 (I - U U^T)) + ve I and
//   M^-1 = base I + U diag(c) U^T,  base = 1 / (vg r0 + ve),  c_j = 1 / (vg lambda_j + ve) - base
// (the Woodbury form the low-rank LMM uses for V^-1, lmm_engine.cpp:1097-1105).  Applying it
// to a k-column block is two GEMMs of n x r x k; it removes the few large eigenvalues that
// population structure gives K, which set the iteration count of the scalar preconditioner.
struct LowRankPreconditioner {
    DeviceBuffer<double> U;       // n x r, row-major
    std::vector<double> lambda;   // r eigenvalues of K
    double r0 = 0.0, base = 0.0;
    int64_t n = 0, r = 0;
    DeviceBuffer<double> c, T;
    void set_components(double vg, double ve, cudaStream_t s);
    // Z (n x ldz, row-major) = M^-1 R (n x ldr), k columns; Z must not alias R.
    void apply(const double* R, int64_t ldr, int64_t k, double* Z, int64_t ldz, cudaStream_t s);
};

struct PcgWorkspace {
    DeviceBuffer<double> R, P, AP, T, Zp, partial_a, partial_b;
    DeviceBuffer<double> alpha, beta, rsold, rr, rz;
    DeviceBuffer<int32_t> map, idx;
};

struct PcgStats {
    std::vector<int32_t> iterations;  // per column
    int64_t sweeps = 0;               // operator applies (each over the active columns)
    int64_t column_iterations = 0;
};

// libCosmicCore/src/matrix_free_pcg.h:20-68 on k right-hand sides at once (x0 = 0): every
// column runs its own CG recurrence with the scalar preconditioner 1/diag and stops when
// ||r|| < tol (absolute; relative: tol * ||b||) or at max_iter.  Converged columns leave the
// operator applies.  B, X: row-major (n_rec x ld).
// With a preconditioner M, z = M^-1 r replaces r / diag.
void pcg_solve_block(VOperator& A, double diag, const double* B, int64_t ldb, int64_t k,
                     double* X, int64_t ldx, double tol, bool relative, int max_iter,
                     PcgWorkspace& ws, PcgStats& st, cudaStream_t s,
                     LowRankPreconditioner* M = nullptr);

// Column dot products of two row-major blocks: out[c] = sum_i A[i, c] * B[i, c] (host),
// in a fixed summation order.
void column_dots(const double* A, int64_t lda, const double* B, int64_t ldb, int64_t n, int64_t k,
                 double* out_host, PcgWorkspace& ws, cudaStream_t s);

// The mt19937_64 stream on the device (omega.cu).
void mt64_seed_device(uint64_t seed, uint64_t* d_state, cudaStream_t s);
void mt64_generate(uint64_t* d_state, int64_t n_out, uint64_t* d_out, cudaStream_t s);

// A continuing mt19937_64 stream mapped to Rademacher signs the way
// std::uniform_int_distribution<int>(0, 1) maps it (the top bit): probe t takes draws
// t*n .. t*n + n - 1 and lands in column t of a row-major block.
struct RademacherStream {
    DeviceBuffer<uint64_t> state, raw, carry;
    int64_t n_carry = 0;
    void seed(uint64_t seed, cudaStream_t s);
    void draw(int64_t n, int64_t cols, double* out, int64_t ld, cudaStream_t s);
};

}  // namespace cs
