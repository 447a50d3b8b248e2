// Low-rank matrix-free LMM engine:
//   prepare  = LmmEngine::prepareLowRankMatrixFree  (src/lmm_engine.cpp:897-1095)
//   scan     = LmmEngine::scanLowRank              (src/lmm_engine.cpp:1269-1361)
//
// Device work: the operator applies (the hot loop), the QR / projection GEMMs of the
// randomized subspace iteration, the per-SNP basis projection of the scan (a decode-GEMM
// over the packed genotypes) and its per-SNP statistics.  Host work: the mt19937_64
// stream of Omega (sequential by definition), the sk x sk eigendecomposition, and the
// REML search, which after projecting X and y onto the basis costs O(rank p^2) per
// evaluation.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <numeric>
#include <mutex>
#include <optional>
#include <random>

#include "cs_internal.h"
#include "dense_internal.h"
#include "linalg_host.h"
#include "vce_internal.h"

namespace cs {
// Workspace of the device Cholesky-QR: cuSOLVER buffers and the factorisation status.
struct QrWorkspace {
    DeviceBuffer<double> potrf_work;
    DeviceBuffer<char> trtri_work;
    std::vector<char> trtri_host;
    DeviceBuffer<int> info;
    int64_t k = -1;
};
}  // namespace cs

struct cs_lmm {
    int64_t n = 0, p = 0, rank = 0;
    bool prepared = false;
    bool sketched = false;
    cs_lowrank_diagnostics sketch_diag{};
    std::vector<double> lambda;
    double r0 = 0.0, sigma2_g = 0.0, sigma2_e = 0.0, delta = 0.0;
    std::vector<double> y, X;  // host, X column-major n x p
    cs::DeviceBuffer<double> d_U;  // n x rank, row-major
    cublasHandle_t blas = nullptr;
    cs::DeviceBuffer<double> d_a, d_b, d_c, d_d;
    // persistent work buffers (grown on demand, never freed between calls)
    cs::DeviceBuffer<double> omega, sample, q, scratch, gram, small;
    cs::OmegaWorkspace omega_ws;
    cs::QrWorkspace qr_ws;
    // device eigensolver of the sketch's projected matrix: eigenvalues, workspace, status
    cs::DeviceBuffer<double> eig_w, eig_work;
    cs::DeviceBuffer<int> eig_info;
    // scan: analysed-sample view of the genotypes and its tensor-core context, cached
    // for repeated scans of the same (genotypes, keep) pair
    uint64_t scan_g_uid = 0;
    int64_t scan_begin = -1, scan_end = -1;
    std::vector<int32_t> scan_keep;
    cs::DeviceBuffer<uint8_t> scan_own;
    cs_packed_view scan_view;
    std::vector<int32_t> scan_counts;
    cs::MixedScan* scan_mixed = nullptr;
    // The last sketch apply's rows pass, kept for the scan (mixed form, every sample): the
    // scan's U block is Z_c^T U = (Z_c^T Q) W_sel, so it needs no genotype pass.  d_ztq
    // holds s_t^2 (Z_c^T Q)[t, :] per operator row t (R x sketch, column-major); snp_row maps
    // a .bed row to its operator row (-1: none); d_s2inv = 1 / s_t^2 (0 where s_t = 0).
    // With the fused final apply the next p + 1 columns hold s_t^2 Z_c^T [X | y - ybar] for
    // the y / X recorded in fused_y / fused_X.
    uint64_t sketch_g_uid = 0;
    int64_t ztq_rows = 0, ztq_cols = 0, ztq_sk = 0, fused_p = -1;
    std::vector<double> fused_y, fused_X;
    cs::DeviceBuffer<double> d_ztq, d_wsel, d_s2inv, d_ztq_u, qx, sample_x, d_betax;
    std::vector<double> utz;  // U^T [X | y] of the last fit (rank x (p + 1), column-major)
    // Several traits of one request (the serving loop): their y columns (n x t), and the
    // projection [U | X | py | y_1 - ybar_1 .. y_t - ybar_t] of the first trait's scan, valid
    // for the sketch generation, covariates, precision and scan view it was made with.
    std::vector<double> trait_Y, tcache_X;
    int64_t trait_t = 0;
    uint64_t basis_gen = 0, tcache_gen = 0;
    int tcache_prec = -1;
    bool tcache_valid = false;
    cs::DeviceBuffer<double> d_bt, d_tc;
    // the per-SNP encoding of the cached scan view and MAF threshold, and whether d_lut /
    // d_gn2 / d_pass still hold it (a later trait of the same request reuses both)
    std::vector<double> enc_lut, enc_gn2, enc_fr, enc_row_mean;
    std::vector<uint8_t> enc_pass;
    double enc_maf = -1.0;
    bool enc_valid = false, enc_on_device = false;
    std::vector<int32_t> snp_row;
    cs::DeviceBuffer<int32_t> d_win_rows;
    // exact mode (LmmEngine::prepareFromVce): the dense eigenbasis and null model, and the
    // scan's per-chunk buffers
    std::shared_ptr<const cs::DenseNull> dense;
    bool dense_residuals = false;
    cs::DeviceBuffer<double> d_chunk, d_py, d_vinv, d_wutx, d_acc;
    cs::DeviceBuffer<int32_t> d_counts, d_tested;
    cs::DeviceBuffer<double> d_lut, d_T, d_gn2, d_cv, d_utx, d_inv, d_beta, d_se, d_p, d_l10;
    cs::DeviceBuffer<uint8_t> d_pass;
    // sketch eigenvectors: the rotated Q, the QL rotations, the selected columns
    cs::DeviceBuffer<double> d_eig, d_rot_cs;
    cs::DeviceBuffer<int32_t> d_rot_i, d_cols;
    ~cs_lmm() { cs::mixed_scan_destroy(scan_mixed); }
};

namespace cs {

namespace {


// ---------------------------------------------------------------- QR
// Strictly lower triangle of a k x k column-major matrix -> 0 (cuSOLVER leaves the Gram's
// lower half under the factor).
__global__ void k_zero_lower(double* __restrict__ A, int64_t k) {
    const int64_t total = k * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x)
        if (e % k > e / k) A[e] = 0.0;
}

// One pass with the factor on the host (shifted when the Gram is not numerically positive
// definite): R^{-1} -> Rinv_d.  Returns false when even the shifted Gram fails.
bool host_factor_pass(const double* G, int64_t n, int64_t k, double* Rinv_d, bool& shifted,
                      cudaStream_t s) {
    std::vector<double> g(k * k), R;
    CS_CUDA(cudaMemcpyAsync(g.data(), G, 8 * k * k, cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    shifted = false;
    if (!la::cholesky_upper(g, (int)k, R)) {
        // shifted Cholesky-QR: G + sigma I is safely positive definite
        double tr = 0.0;
        for (int64_t j = 0; j < k; ++j) tr += g[j + j * k];
        const double shift = 11.0 * (double)(n * k + k * (k + 1)) * 2.2e-16 * tr;
        for (int64_t j = 0; j < k; ++j) g[j + j * k] += shift;
        if (!la::cholesky_upper(g, (int)k, R)) return false;
        shifted = true;
    }
    const std::vector<double> Rinv = la::upper_inverse(R, (int)k);
    CS_CUDA(cudaMemcpyAsync(Rinv_d, Rinv.data(), 8 * k * k, cudaMemcpyHostToDevice, s));
    CS_CUDA(cudaStreamSynchronize(s));
    return true;
}

// Thin QR of Y (n x k row-major) by Cholesky-QR (`passes` passes, 2 = Cholesky-QR2) of
// G = Y^T Y, G = R^T R, Y <- Y R^{-1}, with the k x k factor and its triangular inverse
// formed on the device (cuSOLVER potrf + trtri) and applied as one DGEMM (a device
// triangular solve of this shape runs several times slower than the GEMM).  A pass whose
// Gram matrix is not numerically positive definite is factored on the host with a shift
// (shifted Cholesky-QR) and one more pass added.  Any orthonormal basis of span(Y) gives the
// same subspace iteration as the reference's HouseholderQR (lmm_engine.cpp:931-941): Q is
// unique up to column signs, which cancel in Q^T K Q and in U = Q W.  Y is used as scratch;
// the result is written to Q.
void cholesky_qr(cublasHandle_t blas, double* Y, int64_t n, int64_t k, double* Q,
                 DeviceBuffer<double>& d_gram, QrWorkspace& ws, cudaStream_t s, int passes = 2) {
    const double one = 1.0, zero = 0.0;
    d_gram.resize(k * k);
    double* G = d_gram.get();
    CS_BLAS(cublasSetStream(blas, s));
    cusolverDnHandle_t sol = shared_solver();
    CS_SOLVER(cusolverDnSetStream(sol, s));
    if (ws.k != k) {
        int lw = 0;
        CS_SOLVER(cusolverDnDpotrf_bufferSize(sol, CUBLAS_FILL_MODE_UPPER, (int)k, G, (int)k, &lw));
        ws.potrf_work.resize(std::max(lw, 1));
        size_t dbytes = 0, hbytes = 0;
        CS_SOLVER(cusolverDnXtrtri_bufferSize(sol, CUBLAS_FILL_MODE_UPPER, CUBLAS_DIAG_NON_UNIT, k,
                                              CUDA_R_64F, G, k, &dbytes, &hbytes));
        ws.trtri_work.resize(std::max<size_t>(dbytes, 1));
        ws.trtri_host.resize(std::max<size_t>(hbytes, 1));
        ws.info.resize(2);
        ws.k = k;
    }
    double* src = Y;
    double* dst = Q;
    for (int pass = 0; pass < passes; ++pass) {
        CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)k, (int)k, (int)n, &one, src,
                            (int)k, src, (int)k, &zero, G, (int)k));
        // G = R^T R on the device, then R^{-1} in place (upper triangle)
        CS_SOLVER(cusolverDnDpotrf(sol, CUBLAS_FILL_MODE_UPPER, (int)k, G, (int)k,
                                   ws.potrf_work.get(), (int)ws.potrf_work.count, ws.info.get()));
        int info = 0;
        CS_CUDA(cudaMemcpyAsync(&info, ws.info.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaStreamSynchronize(s));
        if (info == 0) {
            CS_SOLVER(cusolverDnXtrtri(sol, CUBLAS_FILL_MODE_UPPER, CUBLAS_DIAG_NON_UNIT, k, CUDA_R_64F,
                                       G, k, ws.trtri_work.get(), ws.trtri_work.count,
                                       ws.trtri_host.data(), ws.trtri_host.size(), ws.info.get() + 1));
            k_zero_lower<<<(unsigned)std::min<int64_t>((k * k + 255) / 256, 1024), 256, 0, s>>>(G, k);
            CS_LAUNCH("zero_lower");
        } else {
            // not numerically positive definite: recompute the Gram and factor it on the host
            CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)k, (int)k, (int)n, &one, src,
                                (int)k, src, (int)k, &zero, G, (int)k));
            bool shifted = false;
            if (!host_factor_pass(G, n, k, G, shifted, s))
                fail(CS_ERR_NUMERIC, "QR of the sketch failed (rank-deficient sketch)");
            if (shifted) passes = std::min(passes + 1, 4);
        }
        // row-major dst = src R^{-1}  <=>  column-major dst^c = R^{-T} src^c
        CS_BLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)k, (int)n, (int)k, &one, G,
                            (int)k, src, (int)k, &zero, dst, (int)k));
        // the last pass must land in Q
        const bool last = pass + 1 == passes;
        if (!last) {
            src = dst;
            dst = dst == Q ? Y : Q;
        } else if (dst != Q) {
            CS_CUDA(cudaMemcpyAsync(Q, dst, 8 * n * k, cudaMemcpyDeviceToDevice, s));
        }
    }
    int tinfo[2] = {0, 0};
    CS_CUDA(cudaMemcpyAsync(tinfo, ws.info.get(), 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    if (tinfo[1] != 0) fail(CS_ERR_NUMERIC, "QR of the sketch failed (singular triangular factor)");
}

// ---------------------------------------------------------------- eigenvectors
// Applies the recorded QL rotations to the columns of Q (n x n, column-major): block b owns
// rows 32 b .. 32 b + 31 in shared memory (one lane per row, bank-conflict free), a warp loads
// 32 rotations at a time and broadcasts them with shuffles, and the rotations are applied in
// order (each updates columns i and i + 1 of the lane's row).
__global__ void __launch_bounds__(32, 1)
k_rotate_rows(double* __restrict__ Q, int n, const int32_t* __restrict__ ri,
              const double2* __restrict__ rcs, int64_t nrot) {
    extern __shared__ double rows_s[];  // rows_s[c * 32 + lane]
    const int lane = threadIdx.x;
    const int r = blockIdx.x * 32 + lane;
    const bool live = r < n;
    for (int c = 0; c < n; ++c) rows_s[c * 32 + lane] = live ? Q[r + (int64_t)c * n] : 0.0;
    __syncwarp();
    // A QL sweep runs i downwards, so rotation (i - 1, i) usually follows (i, i + 1): the new
    // column i stays in a register for it instead of a store-load round trip.
    int prev_i = -2;
    double carry = 0.0;
    for (int64_t base = 0; base < nrot; base += 32) {
        const int64_t q = base + lane;
        const int my_i = q < nrot ? ri[q] : 0;
        const double2 my_cs = q < nrot ? rcs[q] : make_double2(1.0, 0.0);
        const int cnt = nrot - base < 32 ? (int)(nrot - base) : 32;
        for (int j = 0; j < cnt; ++j) {
            const int i = __shfl_sync(0xffffffffu, my_i, j);
            const double c = __shfl_sync(0xffffffffu, my_cs.x, j);
            const double sn = __shfl_sync(0xffffffffu, my_cs.y, j);
            const double a = rows_s[i * 32 + lane];
            const double b = (i + 1 == prev_i) ? carry : rows_s[(i + 1) * 32 + lane];
            const double na = c * a - sn * b;
            rows_s[(i + 1) * 32 + lane] = sn * a + c * b;
            rows_s[i * 32 + lane] = na;
            carry = na;
            prev_i = i;
        }
    }
    __syncwarp();
    if (live)
        for (int c = 0; c < n; ++c) Q[r + (int64_t)c * n] = rows_s[c * 32 + lane];
}

// out[:, j] = Q[:, cols[j]] (column-major, n rows)
__global__ void k_gather_columns(const double* __restrict__ Q, int64_t n,
                                 const int32_t* __restrict__ cols, int64_t k, double* __restrict__ out) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = e / n, a = e - j * n;
        out[e] = Q[a + (int64_t)cols[j] * n];
    }
}

// ---------------------------------------------------------------- REML (host)
// Objective of lmm_engine.cpp:990-1009 evaluated in the basis: with
// R^{-1}(eta) = b I + U diag(c) U^T, b = 1/(1 + eta r0), c_j = 1/(1 + eta l_j) - b,
// every N-length product reduces to X^T X, X^T y, U^T X, U^T y.
struct RemlData {
    int64_t n, p, rank;
    double r0;
    const double* lambda;
    std::vector<double> XtX, Xty, UtX, Uty;  // UtX rank x p col-major
    double yty = 0.0;
    const double* X;
    const double* y;
};

double reml_objective(const RemlData& d, double log_eta, double* quadratic) {
    const int64_t p = d.p, r = d.rank, n = d.n;
    const double eta = std::exp(log_eta);
    const double base = 1.0 / (1.0 + eta * d.r0);
    std::vector<double> c(r);
    for (int64_t j = 0; j < r; ++j) c[j] = 1.0 / (1.0 + eta * d.lambda[j]) - base;
    std::vector<double> info(p * p), xry(p);
    for (int64_t a = 0; a < p; ++a) {
        for (int64_t b = 0; b < p; ++b) {
            double acc = base * d.XtX[a + b * p];
            for (int64_t j = 0; j < r; ++j) acc += d.UtX[j + a * r] * c[j] * d.UtX[j + b * r];
            info[a + b * p] = acc;
        }
        double acc = base * d.Xty[a];
        for (int64_t j = 0; j < r; ++j) acc += d.UtX[j + a * r] * c[j] * d.Uty[j];
        xry[a] = acc;
    }
    std::vector<double> L, D;
    if (!la::ldlt(info, (int)p, L, D)) return std::numeric_limits<double>::infinity();
    std::vector<double> beta = xry;
    la::ldlt_solve(L, D, (int)p, beta.data());
    // residual r = y - X beta: r^T r = y^T y - 2 beta^T X^T y + beta^T X^T X beta
    double rr = d.yty;
    for (int64_t a = 0; a < p; ++a) {
        rr -= 2.0 * beta[a] * d.Xty[a];
        for (int64_t b = 0; b < p; ++b) rr += beta[a] * d.XtX[a + b * p] * beta[b];
    }
    (void)n;
    double qf = base * rr;
    for (int64_t j = 0; j < r; ++j) {
        double ur = d.Uty[j];
        for (int64_t a = 0; a < p; ++a) ur -= d.UtX[j + a * r] * beta[a];
        qf += c[j] * ur * ur;
    }
    if (!(qf > 0.0) || !std::isfinite(qf)) return std::numeric_limits<double>::infinity();
    if (quadratic) *quadratic = qf;
    double logdet_r = (double)(n - r) * std::log1p(eta * d.r0);
    for (int64_t j = 0; j < r; ++j) logdet_r += std::log(1.0 + eta * d.lambda[j]);
    double logdet_x = 0.0;
    for (int64_t a = 0; a < p; ++a) logdet_x += std::log(std::max(std::abs(D[a]), 1e-300));
    const double df = (double)(n - p);
    return logdet_r + logdet_x + df * std::log(qf / df);
}

// 81-point grid on log(eta) in [-12, 12] then <= 80 golden-section steps to 1e-8
// (lmm_engine.cpp:1010-1040).
void reml_search(const RemlData& d, double* best_log_eta, double* best_obj, double* quadratic) {
    const int grid = 81;
    int best_index = 0;
    double ble = -12.0;
    double bo = reml_objective(d, ble, nullptr);
    for (int i = 1; i < grid; ++i) {
        const double cand = -12.0 + 24.0 * i / static_cast<double>(grid - 1);
        const double v = reml_objective(d, cand, nullptr);
        if (v < bo) {
            bo = v;
            ble = cand;
            best_index = i;
        }
    }
    double left = -12.0 + 24.0 * std::max(0, best_index - 1) / static_cast<double>(grid - 1);
    double right = -12.0 + 24.0 * std::min(grid - 1, best_index + 1) / static_cast<double>(grid - 1);
    const double golden = (std::sqrt(5.0) - 1.0) / 2.0;
    double c = right - golden * (right - left), dd = left + golden * (right - left);
    double fc = reml_objective(d, c, nullptr), fd = reml_objective(d, dd, nullptr);
    for (int it = 0; it < 80 && right - left > 1e-8; ++it) {
        if (fc < fd) {
            right = dd; dd = c; fd = fc; c = right - golden * (right - left);
            fc = reml_objective(d, c, nullptr);
        } else {
            left = c; c = dd; fc = fd; dd = left + golden * (right - left);
            fd = reml_objective(d, dd, nullptr);
        }
    }
    ble = 0.5 * (left + right);
    double q = 0.0;
    bo = reml_objective(d, ble, &q);
    if (!std::isfinite(bo)) fail(CS_ERR_NUMERIC, "Low-rank REML optimization failed");
    *best_log_eta = ble;
    *best_obj = bo;
    *quadratic = q;
}

// U^T [cols] for host column-major matrices Z (n x m): returns rank x m column-major.
std::vector<double> project_on_basis(cs_lmm* l, const double* Z, int64_t m, cudaStream_t s) {
    const int64_t n = l->n, r = l->rank;
    std::vector<double> zr((size_t)n * m);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t c = 0; c < m; ++c) zr[i * m + c] = Z[i + c * n];
    l->d_a.resize(n * m);
    l->d_b.resize(r * m);
    CS_CUDA(cudaMemcpyAsync(l->d_a.get(), zr.data(), 8 * n * m, cudaMemcpyHostToDevice, s));
    const double one = 1.0, zero = 0.0;
    CS_BLAS(cublasSetStream(l->blas, s));
    // out (rank x m, col-major) = U^c (rank x n) * Z^c^T  with Z^c = (m x n)
    CS_BLAS(cublasDgemm(l->blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)r, (int)m, (int)n, &one,
                        l->d_U.get(), (int)r, l->d_a.get(), (int)m, &zero, l->d_b.get(), (int)r));
    std::vector<double> out((size_t)r * m);
    CS_CUDA(cudaMemcpyAsync(out.data(), l->d_b.get(), 8 * r * m, cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    return out;
}

// ---------------------------------------------------------------- scan kernels
// The py column of one trait from the cached projection C (row-major, ld ldc):
//   C[j, r + p] = b (C[j, ycol] - sum_a C[j, r + a] bX_a)  (the U-block term added afterwards).
__global__ void k_scan_py_from_y(double* __restrict__ C, int64_t ldc, int64_t r, int p,
                                 int64_t ycol, const double* __restrict__ betax, double base,
                                 int64_t M) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < M;
         j += (int64_t)gridDim.x * blockDim.x) {
        double* c = C + j * ldc;
        double fit = 0.0;
        for (int a = 0; a < p; ++a) fit += c[r + a] * betax[a];
        c[r + p] = base * (c[ycol] - fit);
    }
}

// The X and py columns of the scan's T from the fused sketch apply: with F (R x (p + 1),
// column-major, ld R) = s^2 o Z_c^T [X | y - ybar] and row = rows[j],
//   T[j, a] = F[row, a] / s^2 (a < p),  T[j, p] = b (F[row, p] / s^2 - sum_a T[j, a] bX_a),
// the U-block term of py added afterwards (0 where row < 0).
__global__ void k_scan_fused_cols(const double* __restrict__ F, int64_t ldf, int p,
                                  const int32_t* __restrict__ rows, const double* __restrict__ s2inv,
                                  const double* __restrict__ betax, double base, int64_t M,
                                  double* __restrict__ T, int64_t ldt) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < M;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int32_t row = rows[j];
        double* t = T + j * ldt;
        if (row < 0) {
            for (int a = 0; a <= p; ++a) t[a] = 0.0;
            continue;
        }
        const double si = s2inv[row];
        double fit = 0.0;
        for (int a = 0; a < p; ++a) {
            const double v = F[row + (int64_t)a * ldf] * si;
            t[a] = v;
            fit += v * betax[a];
        }
        t[p] = base * (F[row + (int64_t)p * ldf] * si - fit);
    }
}

// T[j ldt + c] (c < r) = C[c + row_j r] / s_row^2, row_j = rows[j] (0 where row_j < 0): the
// scan's U block from W_sel^T (Z_c^T Q)^T.
__global__ void k_scan_u_block(const double* __restrict__ C, int64_t r, const int32_t* __restrict__ rows,
                               const double* __restrict__ s2inv, int64_t M, double* __restrict__ T,
                               int64_t ldt) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < M * r;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = e / r, c = e - j * r;
        const int32_t row = rows[j];
        T[j * ldt + c] = row >= 0 ? C[c + (int64_t)row * r] * s2inv[row] : 0.0;
    }
}


// gamma_q / chisq_prob of src/lmm_engine.cpp:22-64 (series or continued fraction with a
// 1e-7 relative stopping tolerance and at most 100 terms; 0 when neither converges).
__device__ double d_gamma_q(double a, double x) {
    if (x < 0.0 || a <= 0.0) return 1.0;
    if (x < a + 1.0) {
        double ap = a, sum = 1.0 / a, del = sum;
        for (int i = 0; i < 100; ++i) {
            ap += 1.0;
            del *= x / ap;
            sum += del;
            if (fabs(del) < fabs(sum) * 1e-7)
                return 1.0 - sum * exp(-x + a * log(x) - lgamma(a));
        }
    } else {
        double b = x + 1.0 - a, c = 1.0 / 1e-30, d = 1.0 / b, h = d;
        for (int i = 1; i <= 100; ++i) {
            const double an = -i * (i - a);
            b += 2.0;
            d = an * d + b;
            if (fabs(d) < 1e-30) d = 1e-30;
            c = b + an / c;
            if (fabs(c) < 1e-30) c = 1e-30;
            d = 1.0 / d;
            const double del = d * c;
            h *= del;
            if (fabs(del - 1.0) < 1e-7) return exp(-x + a * log(x) - lgamma(a)) * h;
        }
    }
    return 0.0;
}

__device__ double d_chisq_prob(double stat, int df) {
    if (stat <= 0) return 1.0;
    return d_gamma_q(df / 2.0, stat / 2.0);
}

struct ScanParams {
    int64_t n_snps, rank, p, ldt;
    double base;
    const double* T;        // n_snps x ldt: [U^T g | X^T g | py^T g]
    const double* c;        // rank
    const double* UtX;      // rank x p, column-major
    const double* info_inv; // p x p
    const double* gnorm2;   // per SNP ||g_centred||^2
    const uint8_t* pass;    // per SNP MAF filter
    double* beta; double* se; double* pval; double* log10p;
    int32_t* tested;
};

// The variance of lmm_engine.cpp:1309-1313 in the basis,
// var = b ||g||^2 + sum_j c_j t_j^2 - xvg^T I^{-1} xvg, xvg = b X^T g + (U^T X)^T diag(c) t,
// one warp per SNP (a streaming read of T's rows); score and var go to beta / se, which
// k_scan_pvalues then turns into the statistics one thread per SNP (the p-value's series /
// continued fraction on every lane).
__global__ void k_scan_epilogue(ScanParams P) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    constexpr int kMaxP = 16;
    for (int64_t j = warp; j < P.n_snps; j += n_warps) {
        if (!P.pass[j]) continue;
        const double* t = P.T + j * P.ldt;
        double quad = 0.0;
        double xvg[kMaxP];
        for (int a = 0; a < P.p; ++a) xvg[a] = 0.0;
        for (int64_t q = lane; q < P.rank; q += 32) {
            const double tq = t[q], cq = P.c[q];
            quad += cq * tq * tq;
            for (int a = 0; a < P.p; ++a) xvg[a] += P.UtX[q + a * P.rank] * cq * tq;
        }
        for (int off = 16; off; off >>= 1) {
            quad += __shfl_xor_sync(0xffffffffu, quad, off);
            for (int a = 0; a < P.p; ++a) xvg[a] += __shfl_xor_sync(0xffffffffu, xvg[a], off);
        }
        if (lane == 0) {
            for (int a = 0; a < P.p; ++a) xvg[a] += P.base * t[P.rank + a];
            double var = P.base * P.gnorm2[j] + quad;
            for (int a = 0; a < P.p; ++a) {
                double mid = 0.0;
                for (int b = 0; b < P.p; ++b) mid += P.info_inv[a + b * P.p] * xvg[b];
                var -= xvg[a] * mid;
            }
            P.beta[j] = t[P.rank + P.p];  // score
            P.se[j] = var;
        }
    }
}

__global__ void k_scan_pvalues(ScanParams P) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < P.n_snps;
         j += (int64_t)gridDim.x * blockDim.x) {
        if (!P.pass[j]) {
            P.tested[j] = 0;
            continue;
        }
        const double score = P.beta[j], var = P.se[j];
        if (!(var > 1e-12) || !isfinite(var)) {
            P.tested[j] = 0;
            continue;
        }
        const double statistic = score / sqrt(var);
        const double pv = d_chisq_prob(statistic * statistic, 1);
        P.tested[j] = 1;
        P.beta[j] = score / var;
        P.se[j] = 1.0 / sqrt(var);
        P.pval[j] = pv;
        P.log10p[j] = pv > 0.0 ? -log10(pv) : 300.0;
    }
}

// Exact scan (src/lmm_engine.cpp:1428-1474), one chunk of W_proj's columns at a time: per SNP
// (one warp), score += T . Py, var += T^2 . V^-1 and xvg[a] += T . (V^-1 UtX)[:, a], with
// T = W_proj[:, chunk]^T g_c.  acc is M x (2 + p).
__global__ void k_exact_accumulate(const double* __restrict__ T, int64_t ldt, int64_t M,
                                   int64_t kc, const double* __restrict__ py,
                                   const double* __restrict__ vinv, const double* __restrict__ wutx,
                                   int64_t ldw, int p, double* __restrict__ acc) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    constexpr int kMaxP = 16;
    for (int64_t j = warp; j < M; j += n_warps) {
        const double* t = T + j * ldt;
        double sc = 0.0, var = 0.0, x[kMaxP];
        for (int a = 0; a < p; ++a) x[a] = 0.0;
        for (int64_t c = lane; c < kc; c += 32) {
            const double tc = t[c];
            sc += tc * py[c];
            var += tc * tc * vinv[c];
            for (int a = 0; a < p; ++a) x[a] += tc * wutx[c + a * ldw];
        }
        for (int off = 16; off; off >>= 1) {
            sc += __shfl_xor_sync(0xffffffffu, sc, off);
            var += __shfl_xor_sync(0xffffffffu, var, off);
            for (int a = 0; a < p; ++a) x[a] += __shfl_xor_sync(0xffffffffu, x[a], off);
        }
        if (lane == 0) {
            double* o = acc + j * (2 + p);
            o[0] += sc;
            o[1] += var;
            for (int a = 0; a < p; ++a) o[2 + a] += x[a];
        }
    }
}

// Per SNP: var -= xvg^T (X^T V^-1 X)^-1 xvg unless use_residuals, then the Wald statistics
// of src/lmm_engine.cpp:1439-1466 (no row unless var > 1e-12 and finite).
__global__ void k_exact_finish(const double* __restrict__ acc, int p, int64_t M,
                               const uint8_t* __restrict__ pass, const double* __restrict__ inv,
                               int residuals, double* beta, double* se, double* pval,
                               double* log10p, int32_t* tested) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < M;
         j += (int64_t)gridDim.x * blockDim.x) {
        if (!pass[j]) {
            tested[j] = 0;
            continue;
        }
        const double* o = acc + j * (2 + p);
        const double score = o[0];
        double var = o[1];
        if (!residuals && p > 0) {
            double term2 = 0.0;
            for (int a = 0; a < p; ++a) {
                double mid = 0.0;
                for (int b = 0; b < p; ++b) mid += inv[a + b * p] * o[2 + b];
                term2 += o[2 + a] * mid;
            }
            var -= term2;
        }
        if (!(var > 1e-12) || !isfinite(var)) {
            tested[j] = 0;
            continue;
        }
        const double s = sqrt(var);
        const double stat = score / s;
        const double pv = d_chisq_prob(stat * stat, 1);
        tested[j] = 1;
        beta[j] = score / var;
        se[j] = 1.0 / s;
        pval[j] = pv;
        log10p[j] = pv > 0.0 ? -log10(pv) : 300.0;
    }
}

}  // namespace

// Q (host, the tridiagonalising factor) and the QL rotations -> eigenvector matrix in l->d_eig.
static void rotate_eigenvectors(cs_lmm* l, const std::vector<double>& Qh,
                                const std::vector<la::PlaneRotation>& rots, int n, cudaStream_t s) {
    prof::HostScope hs("lowrank_eigvec_rotations");
    const int64_t nr = (int64_t)rots.size();
    std::vector<int32_t> ri(std::max<int64_t>(nr, 1));
    std::vector<double2> rcs(std::max<int64_t>(nr, 1));
    for (int64_t q = 0; q < nr; ++q) {
        ri[q] = rots[q].i;
        rcs[q] = make_double2(rots[q].c, rots[q].s);
    }
    l->d_eig.resize((int64_t)n * n);
    l->d_rot_i.resize(ri.size());
    l->d_rot_cs.resize(2 * rcs.size());
    CS_CUDA(cudaMemcpyAsync(l->d_eig.get(), Qh.data(), 8 * (size_t)n * n, cudaMemcpyHostToDevice, s));
    CS_CUDA(cudaMemcpyAsync(l->d_rot_i.get(), ri.data(), 4 * ri.size(), cudaMemcpyHostToDevice, s));
    CS_CUDA(cudaMemcpyAsync(l->d_rot_cs.get(), rcs.data(), 16 * rcs.size(), cudaMemcpyHostToDevice, s));
    const size_t smem = (size_t)n * 32 * sizeof(double);
    static PerDeviceOnce configured;
    once_per_device(configured, [] {
        return cudaFuncSetAttribute(k_rotate_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    200 * 1024);
    }, "configure eigenvector rotation kernel");
    if (smem > 200 * 1024) fail(CS_ERR_UNSUPPORTED, "sketch too wide for the rotation kernel");
    prof::Scope ps("eigvec_rotations", s, 6.0 * (double)nr * n, 0.0);
    k_rotate_rows<<<(unsigned)((n + 31) / 32), 32, smem, s>>>(
        l->d_eig.get(), n, l->d_rot_i.get(), reinterpret_cast<const double2*>(l->d_rot_cs.get()), nr);
    CS_LAUNCH("eigvec_rotations");
}

// Symmetric eigendecomposition of the k x k matrix at d_B (lower triangle) on the device:
// eigenvectors (columns, ascending eigenvalues) -> l->d_eig, eigenvalues -> w.  cuSOLVER
// syevd (divide and conquer) by default, syevj (Jacobi) with CS_B200_EIGH=syevj; false when
// CS_B200_EIGH=host or the solver reports a failure.
static bool device_eigh(cs_lmm* l, const double* d_B, int64_t k, std::vector<double>& w,
                        cudaStream_t s) {
    static const int mode = [] {
        const char* v = std::getenv("CS_B200_EIGH");
        if (v && std::strcmp(v, "host") == 0) return 0;
        if (v && std::strcmp(v, "syevj") == 0) return 2;
        return 1;
    }();
    if (mode == 0) return false;
    cusolverDnHandle_t sol = shared_solver();
    CS_SOLVER(cusolverDnSetStream(sol, s));
    l->d_eig.resize(k * k);
    l->eig_w.resize(k);
    l->eig_info.resize(1);
    CS_CUDA(cudaMemcpyAsync(l->d_eig.get(), d_B, 8 * k * k, cudaMemcpyDeviceToDevice, s));
    int lwork = 0;
    if (mode == 1) {
        CS_SOLVER(cusolverDnDsyevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                              (int)k, l->d_eig.get(), (int)k, l->eig_w.get(), &lwork));
        l->eig_work.resize(std::max(lwork, 1));
        CS_SOLVER(cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)k,
                                   l->d_eig.get(), (int)k, l->eig_w.get(), l->eig_work.get(), lwork,
                                   l->eig_info.get()));
    } else {
        syevjInfo_t params = nullptr;
        CS_SOLVER(cusolverDnCreateSyevjInfo(&params));
        CS_SOLVER(cusolverDnDsyevj_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                              (int)k, l->d_eig.get(), (int)k, l->eig_w.get(), &lwork,
                                              params));
        l->eig_work.resize(std::max(lwork, 1));
        const cusolverStatus_t st =
            cusolverDnDsyevj(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)k,
                             l->d_eig.get(), (int)k, l->eig_w.get(), l->eig_work.get(), lwork,
                             l->eig_info.get(), params);
        cusolverDnDestroySyevjInfo(params);
        CS_SOLVER(st);
    }
    int info = 0;
    w.resize(k);
    CS_CUDA(cudaMemcpyAsync(w.data(), l->eig_w.get(), 8 * k, cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaMemcpyAsync(&info, l->eig_info.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    return info == 0;
}

cs_lmm* lmm_create() {
    prof::HostScope hs("lmm_create");
    auto* l = new cs_lmm();
    try {
        l->blas = shared_blas();
    } catch (...) {
        delete l;
        throw;
    }
    return l;
}

void lmm_destroy(cs_lmm* l) {
    prof::HostScope hs("lmm_destroy");
    delete l;
}

void lmm_prepare_lowrank(cs_lmm* l, cs_kinship* op, const double* y, const double* X, int64_t p,
                         int rank, int oversample, int64_t seed, double trace_threshold,
                         int min_rank, int precision, cs_lowrank_diagnostics* diag) {
    LowRankTarget t;
    t.rows = op->rows;
    t.trace = op->trace;
    t.apply = [op, precision](const double* X_, int64_t ldx, int64_t k, double* Y_, int64_t ldy,
                              cudaStream_t st) {
        kinship_apply_rowmajor(op, X_, ldx, k, Y_, ldy, precision, st);
    };
    t.fuse_scan_columns = precision == CS_PRECISION_MIXED && op->keep_identity;
    lmm_prepare_lowrank_target(l, t, y, X, p, rank, oversample, seed, trace_threshold, min_rank,
                               diag, 0);
    // keep the final sketch apply's rows pass for the scan (see cs_lmm::d_ztq)
    int64_t R = 0, kq = 0;
    const double* W = precision == CS_PRECISION_MIXED && op->keep_identity
                          ? mixed_rows_output(op, &R, &kq)
                          : nullptr;
    const int64_t sk = l->sketch_diag.sketch_size;
    const bool fused = t.fuse_scan_columns && kq == sk + p + 1;
    if (W && (kq == sk || fused) && R == (int64_t)op->view_snp.size() && R > 0) {
        l->d_ztq.resize(R * kq);
        CS_CUDA(cudaMemcpy(l->d_ztq.get(), W, 8 * R * kq, cudaMemcpyDeviceToDevice));
        std::vector<double> s2inv(R);
        l->snp_row.assign(op->g->n_snps, -1);
        for (int64_t t2 = 0; t2 < R; ++t2) {
            const double sv = op->inv_std[t2];
            s2inv[t2] = sv != 0.0 ? 1.0 / (sv * sv) : 0.0;
            l->snp_row[op->view_snp[t2]] = (int32_t)t2;
        }
        l->d_s2inv.resize(R);
        CS_CUDA(cudaMemcpy(l->d_s2inv.get(), s2inv.data(), 8 * R, cudaMemcpyHostToDevice));
        l->ztq_rows = R;
        l->ztq_cols = kq;
        l->ztq_sk = sk;
        l->fused_p = fused ? p : -1;
        if (fused) {
            l->fused_y.assign(y, y + op->rows);
            l->fused_X.assign(X, X + op->rows * p);
        }
        l->sketch_g_uid = op->g->uid;
    }
}

void lmm_prepare_lowrank_target(cs_lmm* l, const LowRankTarget& target, const double* y,
                                const double* X, int64_t p, int rank, int oversample,
                                int64_t seed, double trace_threshold, int min_rank,
                                cs_lowrank_diagnostics* diag, cudaStream_t s) {
    const auto start = std::chrono::steady_clock::now();
    l->blas = shared_blas();  // the calling thread's handle
    l->sketch_g_uid = 0;  // a new sketch: the kept rows pass (if any) no longer matches
    l->ztq_cols = 0;
    l->fused_p = -1;
    l->dense.reset();     // back to the low-rank mode
    l->utz.clear();
    ++l->basis_gen;
    l->trait_t = 0;
    l->trait_Y.clear();
    l->tcache_valid = false;
    const int64_t n = target.rows;
    if (rank <= 0 || rank >= n || p < 0 || (p > 0 && X == nullptr))
        fail(CS_ERR_INVALID_ARGUMENT,
             "Low-rank LMM requires valid dimensions and 0 < rank < sample count");
    if (p > 16) fail(CS_ERR_UNSUPPORTED, "at most 16 covariate columns are supported");
    const int64_t sk = std::min<int64_t>(n, rank + std::max(0, oversample));
    CS_BLAS(cublasSetStream(l->blas, s));
    DeviceBuffer<double>&omega = l->omega, &sample = l->sample, &q = l->q, &scratch = l->scratch,
                         &gram = l->gram, &small = l->small;
    omega.resize(n * sk);
    sample.resize(n * sk);
    q.resize(n * sk);
    {
        // Omega on the device (the engine's chunks drawn in parallel from jumped windows),
        // then the first apply
        prof::HostScope hs("lowrank_omega_first_apply");
        generate_omega_device((uint64_t)seed, n, sk, omega.get(), sk, l->omega_ws, s);
        target.apply(omega.get(), sk, sk, sample.get(), sk, s);
    }
    {
        prof::HostScope hs("lowrank_subspace_iteration");
        // The iterations only need a well-conditioned basis of the same span (Q = Y R^{-1}
        // spans span(Y) whatever its loss of orthogonality): one Cholesky-QR pass each; the
        // basis that B = Q^T K Q is formed in takes both passes.
        for (int it = 0; it < 2; ++it) {
            cholesky_qr(l->blas, sample.get(), n, sk, q.get(), gram, l->qr_ws, s, 1);
            target.apply(q.get(), sk, sk, sample.get(), sk, s);
        }
        cholesky_qr(l->blas, sample.get(), n, sk, q.get(), gram, l->qr_ws, s);
        if (target.fuse_scan_columns) {
            // [Q | X | y - ybar] in one apply: its rows pass is kept for the scan
            const int64_t kx = sk + p + 1;
            l->qx.resize(n * kx);
            l->sample_x.resize(n * kx);
            double ybar = 0.0;
            for (int64_t i = 0; i < n; ++i) ybar += y[i];
            ybar /= (double)n;
            std::vector<double> h(n * (p + 1));
            for (int64_t i = 0; i < n; ++i) {
                for (int64_t a = 0; a < p; ++a) h[i * (p + 1) + a] = X[i + a * n];
                h[i * (p + 1) + p] = y[i] - ybar;
            }
            CS_CUDA(cudaMemcpy2DAsync(l->qx.get(), 8 * kx, q.get(), 8 * sk, 8 * sk, n,
                                      cudaMemcpyDeviceToDevice, s));
            CS_CUDA(cudaMemcpy2DAsync(l->qx.get() + sk, 8 * kx, h.data(), 8 * (p + 1), 8 * (p + 1),
                                      n, cudaMemcpyHostToDevice, s));
            target.apply(l->qx.get(), kx, kx, l->sample_x.get(), kx, s);
        } else {
            target.apply(q.get(), sk, sk, sample.get(), sk, s);
        }
        CS_CUDA(cudaStreamSynchronize(s));
    }
    std::optional<prof::HostScope> hs_stage;
    hs_stage.emplace("lowrank_eigh");
    // B = Q^T K Q (sk x sk)
    small.resize(sk * sk);
    const double one = 1.0, zero = 0.0;
    {
        const bool fx = target.fuse_scan_columns;
        const double* ks = fx ? l->sample_x.get() : sample.get();
        const int ldk = (int)(fx ? sk + p + 1 : sk);
        CS_BLAS(cublasDgemm(l->blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)sk, (int)sk, (int)n, &one,
                            q.get(), (int)sk, ks, ldk, &zero, small.get(), (int)sk));
    }
    // eigendecomposition of B (its lower triangle): on the device by cuSOLVER, or on the host
    // (tridiagonalisation and QL, the QL rotations applied to the eigenvector matrix on the
    // device) when the device solver reports a failure or CS_B200_EIGH=host asks for it
    std::vector<double> dvals;
    if (!device_eigh(l, small.get(), sk, dvals, s)) {
        std::vector<double> B(sk * sk);
        CS_CUDA(cudaMemcpyAsync(B.data(), small.get(), 8 * sk * sk, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaStreamSynchronize(s));
        std::vector<double> Qh;
        std::vector<la::PlaneRotation> rots;
        if (!la::tridiag_ql(B, (int)sk, dvals, Qh, rots))
            fail(CS_ERR_NUMERIC, "Low-rank GRM eigensolver failed");
        rotate_eigenvectors(l, Qh, rots, (int)sk, s);
    }
    std::vector<int> order(sk);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return dvals[a] < dvals[b]; });
    std::vector<double> evals(sk);
    for (int64_t j = 0; j < sk; ++j) evals[j] = dvals[order[j]];
    std::vector<double> lead(rank);
    for (int j = 0; j < rank; ++j) lead[j] = std::max(0.0, evals[sk - 1 - j]);
    // trace-fraction rank selection (lmm_engine.cpp:958-973)
    const double total_trace = target.trace;
    int selected = rank;
    bool met = trace_threshold <= 0.0;
    if (trace_threshold > 0.0 && total_trace > 0.0) {
        double retained = 0.0;
        const int first_allowed = std::min(rank, std::max(1, min_rank));
        for (int j = 0; j < rank; ++j) {
            retained += lead[j];
            if (j + 1 >= first_allowed && retained / total_trace >= trace_threshold) {
                selected = j + 1;
                met = true;
                break;
            }
        }
    }
    hs_stage.reset();
    hs_stage.emplace("lowrank_basis_reml");
    // U = Q W_top (n x selected, row-major): U^c = W_top^T Q^c, W_top = the eigenvectors of
    // the `selected` largest eigenvalues, largest first
    gram.resize(sk * selected);
    {
        std::vector<int32_t> cols(selected);
        for (int j = 0; j < selected; ++j) cols[j] = order[sk - 1 - j];
        l->d_cols.resize(selected);
        CS_CUDA(cudaMemcpyAsync(l->d_cols.get(), cols.data(), 4 * selected, cudaMemcpyHostToDevice, s));
        k_gather_columns<<<(unsigned)std::max<int64_t>(1, (sk * selected + 255) / 256), 256, 0, s>>>(
            l->d_eig.get(), sk, l->d_cols.get(), selected, gram.get());
        CS_LAUNCH("gather_eigenvectors");
    }
    l->d_U.resize(n * selected);
    CS_BLAS(cublasDgemm(l->blas, CUBLAS_OP_T, CUBLAS_OP_N, selected, (int)n, (int)sk, &one,
                        gram.get(), (int)sk, q.get(), (int)sk, &zero, l->d_U.get(), selected));
    l->d_wsel.resize(sk * selected);  // W_sel (sk x selected, column-major) for the scan
    CS_CUDA(cudaMemcpyAsync(l->d_wsel.get(), gram.get(), 8 * sk * selected, cudaMemcpyDeviceToDevice, s));
    l->n = n;
    l->rank = selected;
    l->lambda.assign(lead.begin(), lead.begin() + selected);
    double lam_sum = 0.0, lam_sq = 0.0;
    for (double v : l->lambda) {
        lam_sum += v;
        lam_sq += v * v;
    }
    l->r0 = std::max(0.0, (total_trace - lam_sum) / static_cast<double>(n - selected));
    const double approx_sq = lam_sq + (double)(n - selected) * l->r0 * l->r0;
    double cross = l->r0 * total_trace;
    for (double v : l->lambda) cross += (v - l->r0) * v;
    const double resid_sq = std::max(0.0, total_trace * total_trace + approx_sq - 2.0 * cross);
    const double rel_err = std::sqrt(resid_sq) / std::max(total_trace, std::numeric_limits<double>::min());
    l->n = n;
    l->sketch_diag = cs_lowrank_diagnostics{};
    l->sketch_diag.requested_rank = rank;
    l->sketch_diag.effective_rank = selected;
    l->sketch_diag.sketch_size = (int32_t)sk;
    l->sketch_diag.trace_threshold_met = met;
    l->sketch_diag.residual_eigenvalue = l->r0;
    l->sketch_diag.relative_frobenius_error = rel_err;
    l->sketch_diag.trace = total_trace;
    l->sketch_diag.trace_fraction = total_trace > 0.0 ? lam_sum / total_trace : 0.0;
    l->sketched = true;
    hs_stage.reset();
    lmm_fit_reml(l, y, X, p, diag, s);
    if (diag)
        diag->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
}

// REML of one trait in the basis of the last sketch (lmm_engine.cpp:1010-1073).
void lmm_fit_reml(cs_lmm* l, const double* y, const double* X, int64_t p,
                  cs_lowrank_diagnostics* diag, cudaStream_t s) {
    const auto start = std::chrono::steady_clock::now();
    prof::HostScope hs("lowrank_reml");
    if (!l->sketched) fail(CS_ERR_INVALID_ARGUMENT, "low-rank basis not computed");
    if (p < 0 || (p > 0 && X == nullptr) || y == nullptr)
        fail(CS_ERR_INVALID_ARGUMENT, "Low-rank LMM requires valid dimensions");
    if (p > 16) fail(CS_ERR_UNSUPPORTED, "at most 16 covariate columns are supported");
    l->blas = shared_blas();
    const int64_t n = l->n;
    const int selected = l->rank;
    l->p = p;
    // REML in the basis
    l->y.assign(y, y + n);
    l->X.assign(X, X + n * p);
    if (n - p <= 0) fail(CS_ERR_INVALID_ARGUMENT, "Low-rank LMM has no residual degrees of freedom");
    std::vector<double> Z(n * (p + 1));
    std::memcpy(Z.data(), X, 8 * n * p);
    std::memcpy(Z.data() + n * p, y, 8 * n);
    std::vector<double> UtZ = project_on_basis(l, Z.data(), p + 1, s);
    l->utz = UtZ;  // U^T [X | y], reused by the scan of this fit
    RemlData d;
    d.n = n; d.p = p; d.rank = selected; d.r0 = l->r0; d.lambda = l->lambda.data();
    d.X = l->X.data(); d.y = l->y.data();
    d.XtX.assign(p * p, 0.0);
    d.Xty.assign(p, 0.0);
    for (int64_t a = 0; a < p; ++a) {
        for (int64_t b = 0; b < p; ++b) {
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) acc += X[i + a * n] * X[i + b * n];
            d.XtX[a + b * p] = acc;
        }
        double acc = 0.0;
        for (int64_t i = 0; i < n; ++i) acc += X[i + a * n] * y[i];
        d.Xty[a] = acc;
    }
    for (int64_t i = 0; i < n; ++i) d.yty += y[i] * y[i];
    d.UtX.assign(UtZ.begin(), UtZ.begin() + selected * p);
    d.Uty.assign(UtZ.begin() + selected * p, UtZ.begin() + selected * (p + 1));
    double ble, bo, quad;
    reml_search(d, &ble, &bo, &quad);
    const double df = (double)(n - p);
    l->delta = std::exp(-ble);
    l->sigma2_e = quad / df;
    l->sigma2_g = std::exp(ble) * l->sigma2_e;
    l->prepared = true;
    if (diag) {
        *diag = l->sketch_diag;
        diag->sigma2_g = l->sigma2_g;
        diag->sigma2_e = l->sigma2_e;
        diag->delta = l->delta;
        diag->log_eta = ble;
        diag->reml_objective = bo;
        diag->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    }
}

int64_t lmm_rank(const cs_lmm* l) { return l->rank; }
const double* lmm_basis_device(const cs_lmm* l) { return l->d_U.get(); }
std::vector<double> lmm_eigenvalues(const cs_lmm* l) { return l->lambda; }
double lmm_residual_eigenvalue(const cs_lmm* l) { return l->r0; }

void lmm_lowrank_basis(const cs_lmm* l, double* U, int64_t ldu, double* lambda) {
    if (!l->prepared) fail(CS_ERR_INVALID_ARGUMENT, "low-rank model not prepared");
    const int64_t n = l->n, r = l->rank;
    if (lambda) std::memcpy(lambda, l->lambda.data(), 8 * r);
    if (U) {
        std::vector<double> h(n * r);
        CS_CUDA(cudaMemcpy(h.data(), l->d_U.get(), 8 * n * r, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < r; ++j) U[i + j * ldu] = h[i * r + j];
    }
}

void lmm_scan(cs_lmm* l, const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
              double min_maf, int precision, double* beta, double* se, double* pvalue,
              double* log10p, double* freq, int32_t* tested) {
    lmm_scan_window(l, g, keep, n_keep, 0, g ? g->n_snps : 0, min_maf, precision, beta, se,
                    pvalue, log10p, freq, tested, 0);
}

// The analysed samples' packed view of SNPs [snp_begin, snp_end) with its code counts, cached
// per (genotypes, window, keep) in l, and the per-SNP encoding of genotype_encoding.h:33-81
// (additive, centred, missing -> the mean): FREQ, the MAF filter, the value table per code,
// the row mean and ||g_c||^2.
struct ScanEncoding {
    std::vector<double> lut, gn2, fr, row_mean;
    std::vector<uint8_t> pass;
    bool cached = false;
    bool reused = false;  // the encoding of the previous scan of this view (and on the device)
};

static ScanEncoding scan_encoding(cs_lmm* l, const cs_genotypes* g, const int32_t* keep,
                                  int64_t n_keep, int64_t snp_begin, int64_t snp_end,
                                  double min_maf, cudaStream_t s) {
    const int64_t M = snp_end - snp_begin;
    ScanEncoding e;
    const bool cached = l->scan_g_uid == g->uid && (int64_t)l->scan_keep.size() == n_keep &&
                        l->scan_begin == snp_begin && l->scan_end == snp_end &&
                        std::memcmp(l->scan_keep.data(), keep, 4 * n_keep) == 0;
    if (cached && l->enc_valid && l->enc_maf == min_maf) {
        e.cached = true;
        e.reused = true;
        e.lut = l->enc_lut;
        e.gn2 = l->enc_gn2;
        e.fr = l->enc_fr;
        e.row_mean = l->enc_row_mean;
        e.pass = l->enc_pass;
        return e;
    }
    l->enc_valid = false;
    l->enc_on_device = false;
    if (!cached) {
        mixed_scan_destroy(l->scan_mixed);
        l->scan_mixed = nullptr;
        bool identity = n_keep == g->n_samples;
        for (int64_t i = 0; identity && i < n_keep; ++i) identity = keep[i] == i;
        const uint8_t* first_row = g->packed.get() + snp_begin * g->stride;
        l->scan_view = cs_packed_view{first_row, M, g->n_samples, g->stride};
        if (!identity) {
            const int64_t n = n_keep;
            const int64_t stride = round_up((n + 3) / 4, kRowAlign);
            l->scan_own.resize(std::max<int64_t>(1, M * stride));
            DeviceBuffer<int32_t> d_keep;
            d_keep.resize(n);
            CS_CUDA(cudaMemcpyAsync(d_keep.get(), keep, 4 * n, cudaMemcpyHostToDevice, s));
            repack(first_row, g->stride, nullptr, M, d_keep.get(), n, l->scan_own.get(),
                   stride, s);
            CS_CUDA(cudaStreamSynchronize(s));
            l->scan_view = cs_packed_view{l->scan_own.get(), M, n, stride};
        }
        l->scan_counts.assign(4 * M, 0);
        if (identity && (int64_t)g->code_counts.size() == 4 * g->n_snps) {
            // every sample in .fam order: the counts of the statistics pass
            std::copy_n(g->code_counts.begin() + 4 * snp_begin, 4 * M, l->scan_counts.begin());
        } else if (M) {
            l->d_counts.resize(std::max<int64_t>(1, 4 * M));
            row_code_counts(l->scan_view, l->d_counts.get(), s);
            CS_CUDA(cudaMemcpyAsync(l->scan_counts.data(), l->d_counts.get(), 16 * M,
                                    cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaStreamSynchronize(s));
        }
        l->scan_g_uid = g->uid;
        l->scan_begin = snp_begin;
        l->scan_end = snp_end;
        l->scan_keep.assign(keep, keep + n_keep);
    }
    e.cached = cached;
    const std::vector<int32_t>& counts = l->scan_counts;
    // ---- per-SNP encoding over the analysed samples (genotype_encoding.h:33-81)
    e.lut.assign(4 * M, 0.0);
    e.gn2.assign(M, 0.0);
    e.fr.assign(M, 0.0);
    e.row_mean.assign(M, 0.0);
    e.pass.assign(M, 0);
    std::vector<double>&lut = e.lut, &gn2 = e.gn2, &fr = e.fr, &row_mean = e.row_mean;
    std::vector<uint8_t>& pass = e.pass;
    for (int64_t j = 0; j < M; ++j) {
        const int64_t c00 = counts[4 * j], c10 = counts[4 * j + 2], c11 = counts[4 * j + 3];
        const int64_t obs = c00 + c10 + c11;
        if (obs == 0) continue;
        const int64_t isum = 2 * c00 + c10;
        const double dosage_sum = (double)isum;
        const double af = dosage_sum / (2.0 * (double)obs);
        fr[j] = af;
        pass[j] = obs >= 3 && std::min(af, 1.0 - af) >= min_maf;
        // the encoded mean (additive model); rows that fail the filter are never reported
        const double mean = dosage_sum / (double)obs;
        row_mean[j] = mean;
        lut[4 * j + 0] = 2.0 - mean;
        lut[4 * j + 1] = 0.0;  // missing -> mean -> centred 0
        lut[4 * j + 2] = 1.0 - mean;
        lut[4 * j + 3] = 0.0 - mean;
        const int64_t sq = 4 * c00 + c10;  // sum of squared dosages
        gn2[j] = (double)(obs * sq - isum * isum) / (double)obs;
    }
    return e;
}

// Results to the caller's host arrays; untested SNPs get NaN statistics.
static void scan_finish(cs_lmm* l, int64_t M, const std::vector<double>& fr, double* beta,
                        double* se, double* pvalue, double* log10p, double* freq,
                        int32_t* tested, cudaStream_t s) {
    std::vector<int32_t> t(M);
    CS_CUDA(cudaMemcpyAsync(t.data(), l->d_tested.get(), 4 * M, cudaMemcpyDeviceToHost, s));
    if (beta) CS_CUDA(cudaMemcpyAsync(beta, l->d_beta.get(), 8 * M, cudaMemcpyDeviceToHost, s));
    if (se) CS_CUDA(cudaMemcpyAsync(se, l->d_se.get(), 8 * M, cudaMemcpyDeviceToHost, s));
    if (pvalue) CS_CUDA(cudaMemcpyAsync(pvalue, l->d_p.get(), 8 * M, cudaMemcpyDeviceToHost, s));
    if (log10p) CS_CUDA(cudaMemcpyAsync(log10p, l->d_l10.get(), 8 * M, cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    for (int64_t j = 0; j < M; ++j) {
        if (tested) tested[j] = t[j];
        if (freq) freq[j] = fr[j];
        if (!t[j]) {
            const double nan = std::numeric_limits<double>::quiet_NaN();
            if (beta) beta[j] = nan;
            if (se) se[j] = nan;
            if (pvalue) pvalue[j] = nan;
            if (log10p) log10p[j] = nan;
        }
    }
}

// LmmEngine::scan's exact branch (src/lmm_engine.cpp:1363-1474) over SNPs [snp_begin,
// snp_end): the null quantities in the eigenbasis on the host (O(n p^2)), then per chunk of
// W_proj's columns the projection T = W_proj[:, chunk]^T G_c of every SNP (tensor cores in the
// mixed form, the FP64 decode-GEMM otherwise) folded into per-SNP sums.
static void lmm_scan_exact(cs_lmm* l, const cs_genotypes* g, const int32_t* keep,
                           int64_t n_keep, int64_t snp_begin, int64_t snp_end, double min_maf,
                           int precision, double* beta, double* se, double* pvalue,
                           double* log10p, double* freq, int32_t* tested, cudaStream_t s) {
    const DenseNull& d = *l->dense;
    const int64_t n = d.n, ne = d.n_eig, p = d.p, M = snp_end - snp_begin;
    if (keep == nullptr || n_keep != n) fail(CS_ERR_INVALID_ARGUMENT, "Sample size mismatch in scan");
    for (int64_t i = 0; i < n_keep; ++i)
        if (keep[i] < 0 || keep[i] >= g->n_samples)
            fail(CS_ERR_INVALID_ARGUMENT, "scan: sample index out of range");
    CS_BLAS(cublasSetStream(l->blas, s));
    std::vector<double> vinv(ne), wutx(ne * p), py(ne);
    for (int64_t i = 0; i < ne; ++i) vinv[i] = 1.0 / (d.sigma2_g * d.D[i] + d.sigma2_e);
    for (int64_t a = 0; a < p; ++a)
        for (int64_t i = 0; i < ne; ++i) wutx[i + a * ne] = d.UtX[i + a * ne] * vinv[i];
    std::vector<double> xvx_inv;
    if (p > 0) {
        std::vector<double> xvx(p * p, 0.0), L, Dl;
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b) {
                double acc = 0.0;
                for (int64_t i = 0; i < ne; ++i) acc += d.UtX[i + a * ne] * wutx[i + b * ne];
                xvx[a + b * p] = acc;
            }
        if (!la::ldlt(xvx, (int)p, L, Dl))
            fail(CS_ERR_NUMERIC, "LMM scan: X^T V^-1 X is singular");
        xvx_inv = la::ldlt_inverse(L, Dl, (int)p);
    }
    std::vector<double> xvy(p, 0.0), bx(p, 0.0);
    for (int64_t i = 0; i < ne; ++i)
        for (int64_t a = 0; a < p; ++a) xvy[a] += vinv[i] * (d.UtX[i + a * ne] * d.Uty[i]);
    for (int64_t a = 0; a < p; ++a)
        for (int64_t b = 0; b < p; ++b) bx[a] += xvx_inv[a + b * p] * xvy[b];
    for (int64_t i = 0; i < ne; ++i) {
        double r = d.Uty[i];
        for (int64_t a = 0; a < p; ++a) r -= d.UtX[i + a * ne] * bx[a];
        py[i] = r * vinv[i];
    }
    prof::HostScope hs_scan("scan_host_setup");
    ScanEncoding enc = scan_encoding(l, g, keep, n_keep, snp_begin, snp_end, min_maf, s);
    for (auto* b : {&l->d_beta, &l->d_se, &l->d_p, &l->d_l10}) b->resize(std::max<int64_t>(1, M));
    l->d_tested.resize(std::max<int64_t>(1, M));
    if (M == 0) return;
    l->d_lut.resize(4 * M);
    l->d_pass.resize(M);
    l->d_py.resize(std::max<int64_t>(1, ne));
    l->d_vinv.resize(std::max<int64_t>(1, ne));
    l->d_wutx.resize(std::max<int64_t>(1, ne * p));
    l->d_inv.resize(std::max<int64_t>(1, p * p));
    l->d_acc.resize(M * (2 + p));
    l->enc_on_device = false;  // d_lut / d_pass now hold this scan's upload (not the cache's)
    CS_CUDA(cudaMemcpyAsync(l->d_lut.get(), enc.lut.data(), 32 * M, cudaMemcpyHostToDevice, s));
    CS_CUDA(cudaMemcpyAsync(l->d_pass.get(), enc.pass.data(), M, cudaMemcpyHostToDevice, s));
    CS_CUDA(cudaMemcpyAsync(l->d_py.get(), py.data(), 8 * ne, cudaMemcpyHostToDevice, s));
    CS_CUDA(cudaMemcpyAsync(l->d_vinv.get(), vinv.data(), 8 * ne, cudaMemcpyHostToDevice, s));
    if (p) {
        CS_CUDA(cudaMemcpyAsync(l->d_wutx.get(), wutx.data(), 8 * ne * p, cudaMemcpyHostToDevice, s));
        CS_CUDA(cudaMemcpyAsync(l->d_inv.get(), xvx_inv.data(), 8 * p * p, cudaMemcpyHostToDevice, s));
    }
    CS_CUDA(cudaMemsetAsync(l->d_acc.get(), 0, 8 * M * (2 + p), s));
    if (precision == CS_PRECISION_MIXED && (!enc.cached || !l->scan_mixed)) {
        mixed_scan_destroy(l->scan_mixed);
        l->scan_mixed = nullptr;
        l->scan_mixed = mixed_scan_create(l->scan_view, enc.row_mean.data(), l->scan_counts.data());
    }
    // chunk width: 1024 columns, fewer when the window is long (T stays within 4 GiB)
    int64_t kc = std::min<int64_t>(1024, std::max<int64_t>(64, ((int64_t)1 << 29) / M));
    kc = std::max<int64_t>(16, kc / 16 * 16);
    kc = std::min<int64_t>(kc, round_up(ne, 16));
    l->d_chunk.resize(n * kc);
    l->d_T.resize(M * kc);
    Workspace ws;
    for (int64_t c0 = 0; c0 < ne; c0 += kc) {
        const int64_t k = std::min<int64_t>(kc, ne - c0);
        colmajor_to_rowmajor(d.W.get() + c0 * n, n, n, k, l->d_chunk.get(), kc, s);
        if (precision == CS_PRECISION_MIXED)
            mixed_scan_project(l->scan_mixed, l->d_chunk.get(), kc, k, l->d_T.get(), kc, s);
        else
            decode_gemm_rows_fp64(l->scan_view, l->d_lut.get(), l->d_chunk.get(), kc, k,
                                  l->d_T.get(), kc, ws, s);
        prof::Scope ps("exact_scan_accumulate", s, (4.0 + 2.0 * p) * M * k, 8.0 * M * k);
        const int blocks = (int)std::min<int64_t>((M * 32 + 255) / 256, 64LL * num_sms());
        k_exact_accumulate<<<std::max(blocks, 1), 256, 0, s>>>(
            l->d_T.get(), kc, M, k, l->d_py.get() + c0, l->d_vinv.get() + c0,
            l->d_wutx.get() + c0, ne, (int)p, l->d_acc.get());
        CS_LAUNCH("exact_scan_accumulate");
    }
    {
        prof::Scope ps("exact_scan_finish", s, 0.0, 8.0 * M * (2 + p));
        k_exact_finish<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((M + 255) / 256, 16LL * num_sms())),
                         256, 0, s>>>(l->d_acc.get(), (int)p, M, l->d_pass.get(), l->d_inv.get(),
                                      l->dense_residuals ? 1 : 0, l->d_beta.get(), l->d_se.get(),
                                      l->d_p.get(), l->d_l10.get(), l->d_tested.get());
        CS_LAUNCH("exact_scan_finish");
    }
    scan_finish(l, M, enc.fr, beta, se, pvalue, log10p, freq, tested, s);
}

void lmm_prepare_from_vce(cs_lmm* l, const cs_eigen_vce* v, bool use_residuals) {
    if (!l || !v || !v->d) fail(CS_ERR_INVALID_ARGUMENT, "prepareFromVce: null argument");
    if (!v->d->solved)
        fail(CS_ERR_INVALID_ARGUMENT, "prepareFromVce: the null model has not been run");
    l->dense = v->d;
    l->dense_residuals = use_residuals;
    l->sigma2_g = v->d->sigma2_g;
    l->sigma2_e = v->d->sigma2_e;
    l->delta = v->d->delta;
    l->n = v->d->n;
    l->sketched = false;
    l->prepared = false;
    l->sketch_g_uid = 0;
    l->ztq_cols = 0;
}

// The y columns of every trait of one request (n x t, column-major) that the following scans
// of this sketch will fit one after the other; the first scan then projects them all.
void lmm_set_scan_traits(cs_lmm* l, const double* Y, int64_t t) {
    l->trait_t = Y && t > 1 ? t : 0;
    l->trait_Y.assign(Y, Y + (l->trait_t ? l->n * t : 0));
    l->tcache_valid = false;
}

void lmm_scan_window(cs_lmm* l, const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                     int64_t snp_begin, int64_t snp_end, double min_maf, int precision,
                     double* beta, double* se, double* pvalue, double* log10p, double* freq,
                     int32_t* tested, cudaStream_t s) {
    l->blas = shared_blas();  // the calling thread's handle
    if (precision != CS_PRECISION_FP64 && precision != CS_PRECISION_MIXED)
        fail(CS_ERR_INVALID_ARGUMENT, "unknown precision mode");
    if (snp_begin < 0 || snp_end > g->n_snps || snp_begin > snp_end)
        fail(CS_ERR_INVALID_ARGUMENT, "scan: SNP window out of range");
    if (l->dense) {
        lmm_scan_exact(l, g, keep, n_keep, snp_begin, snp_end, min_maf, precision, beta, se,
                       pvalue, log10p, freq, tested, s);
        return;
    }
    if (!l->prepared) fail(CS_ERR_INVALID_ARGUMENT, "low-rank model not prepared");
    const int64_t n = l->n, p = l->p, r = l->rank, M = snp_end - snp_begin;
    if (keep == nullptr || n_keep != n)
        fail(CS_ERR_INVALID_ARGUMENT, "Sample size mismatch in scan");
    for (int64_t i = 0; i < n_keep; ++i)
        if (keep[i] < 0 || keep[i] >= g->n_samples)
            fail(CS_ERR_INVALID_ARGUMENT, "scan: sample index out of range");
    CS_BLAS(cublasSetStream(l->blas, s));
    // ---- null quantities (lmm_engine.cpp:1273-1287) in the basis
    const double base = 1.0 / std::max(1e-12, l->sigma2_g * l->r0 + l->sigma2_e);
    std::vector<double> c(r);
    for (int64_t j = 0; j < r; ++j) c[j] = 1.0 / (l->sigma2_g * l->lambda[j] + l->sigma2_e) - base;
    std::vector<double> Z(n * (p + 1));
    std::memcpy(Z.data(), l->X.data(), 8 * n * p);
    std::memcpy(Z.data() + n * p, l->y.data(), 8 * n);
    // U^T [X | y]: kept by the fit for this y and X
    const std::vector<double> UtZ = l->utz.size() == (size_t)(r * (p + 1))
                                        ? l->utz
                                        : project_on_basis(l, Z.data(), p + 1, s);
    const double* UtX = UtZ.data();
    const double* Uty = UtZ.data() + r * p;
    const double* X = l->X.data();
    const double* y = l->y.data();
    std::vector<double> info(p * p), xvy(p);
    for (int64_t a = 0; a < p; ++a) {
        for (int64_t b = 0; b < p; ++b) {
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) acc += X[i + a * n] * X[i + b * n];
            acc *= base;
            for (int64_t j = 0; j < r; ++j) acc += UtX[j + a * r] * c[j] * UtX[j + b * r];
            info[a + b * p] = acc;
        }
        double acc = 0.0;
        for (int64_t i = 0; i < n; ++i) acc += X[i + a * n] * y[i];
        acc *= base;
        for (int64_t j = 0; j < r; ++j) acc += UtX[j + a * r] * c[j] * Uty[j];
        xvy[a] = acc;
    }
    std::vector<double> L, D, info_inv;
    if (p > 0) {
        if (!la::ldlt(info, (int)p, L, D))
            fail(CS_ERR_NUMERIC, "Low-rank LMM fixed-effect information matrix is singular");
        info_inv = la::ldlt_inverse(L, D, (int)p);
    }
    std::vector<double> betaX(p, 0.0);
    for (int64_t a = 0; a < p; ++a)
        for (int64_t b = 0; b < p; ++b) betaX[a] += info_inv[a + b * p] * xvy[b];
    std::vector<double> resid(n);
    for (int64_t i = 0; i < n; ++i) {
        double fit = 0.0;
        for (int64_t a = 0; a < p; ++a) fit += X[i + a * n] * betaX[a];
        resid[i] = y[i] - fit;
    }
    std::vector<double> Utr = project_on_basis(l, resid.data(), 1, s);
    for (int64_t j = 0; j < r; ++j) Utr[j] *= c[j];
    // basis matrix [U | X | py] (n x b, row-major) on the device; py = b r + U (c o U^T r)
    const int64_t bw = r + p + 1;
    l->d_c.resize(n * bw);
    l->d_d.resize(r);
    double* Bm = l->d_c.get();
    {
        std::vector<double> hx(n * (p + 1));
        for (int64_t i = 0; i < n; ++i) {
            for (int64_t a = 0; a < p; ++a) hx[i * (p + 1) + a] = X[i + a * n];
            hx[i * (p + 1) + p] = base * resid[i];
        }
        l->d_a.resize(n * (p + 1));
        CS_CUDA(cudaMemcpyAsync(l->d_a.get(), hx.data(), 8 * n * (p + 1), cudaMemcpyHostToDevice, s));
        CS_CUDA(cudaMemcpyAsync(l->d_d.get(), Utr.data(), 8 * r, cudaMemcpyHostToDevice, s));
        // columns 0..r-1 = U
        CS_CUDA(cudaMemcpy2DAsync(Bm, 8 * bw, l->d_U.get(), 8 * r, 8 * r, n, cudaMemcpyDeviceToDevice, s));
        CS_CUDA(cudaMemcpy2DAsync(Bm + r, 8 * bw, l->d_a.get(), 8 * (p + 1), 8 * (p + 1), n,
                                  cudaMemcpyDeviceToDevice, s));
        // py column += U (c o U^T r):  (Bm^c)[r+p, :] += (U^c)^T t  -> DGEMV on U^c (r x n)
        const double one = 1.0;
        CS_BLAS(cublasDgemv(l->blas, CUBLAS_OP_T, (int)r, (int)n, &one, l->d_U.get(), (int)r,
                            l->d_d.get(), 1, &one, Bm + r + p, (int)bw));
    }
    prof::HostScope hs_scan("scan_host_setup");
    ScanEncoding enc = scan_encoding(l, g, keep, n_keep, snp_begin, snp_end, min_maf, s);
    const bool cached = enc.cached;
    const cs_packed_view& v = l->scan_view;
    const std::vector<int32_t>& counts = l->scan_counts;
    std::vector<double>&lut = enc.lut, &gn2 = enc.gn2, &fr = enc.fr, &row_mean = enc.row_mean;
    std::vector<uint8_t>& pass = enc.pass;
    l->d_lut.resize(std::max<int64_t>(1, 4 * M));
    l->d_T.resize(std::max<int64_t>(1, M * bw));
    l->d_gn2.resize(std::max<int64_t>(1, M));
    l->d_pass.resize(std::max<int64_t>(1, M));
    l->d_cv.resize(std::max<int64_t>(1, r));
    l->d_utx.resize(std::max<int64_t>(1, r * p));
    l->d_inv.resize(std::max<int64_t>(1, p * p));
    for (auto* b : {&l->d_beta, &l->d_se, &l->d_p, &l->d_l10}) b->resize(std::max<int64_t>(1, M));
    l->d_tested.resize(std::max<int64_t>(1, M));
    if (M == 0) return;
    if (!(enc.reused && l->enc_on_device)) {
        CS_CUDA(cudaMemcpyAsync(l->d_lut.get(), lut.data(), 32 * M, cudaMemcpyHostToDevice, s));
        CS_CUDA(cudaMemcpyAsync(l->d_gn2.get(), gn2.data(), 8 * M, cudaMemcpyHostToDevice, s));
        CS_CUDA(cudaMemcpyAsync(l->d_pass.get(), pass.data(), M, cudaMemcpyHostToDevice, s));
        // cached so that later traits over the same window reuse this encoding (the copies
        // above are staged from pageable memory before they return, so nothing here keeps
        // their sources alive; pinned sources would have to be kept until the copy ends)
        l->enc_lut = lut;
        l->enc_gn2 = gn2;
        l->enc_fr = fr;
        l->enc_row_mean = row_mean;
        l->enc_pass = pass;
        l->enc_maf = min_maf;
        l->enc_valid = true;
        l->enc_on_device = true;
    }
    CS_CUDA(cudaMemcpyAsync(l->d_cv.get(), c.data(), 8 * r, cudaMemcpyHostToDevice, s));
    if (p) {
        CS_CUDA(cudaMemcpyAsync(l->d_utx.get(), UtX, 8 * r * p, cudaMemcpyHostToDevice, s));
        CS_CUDA(cudaMemcpyAsync(l->d_inv.get(), info_inv.data(), 8 * p * p, cudaMemcpyHostToDevice, s));
    }
    // ---- T = G_c^T [U | X | py]: the per-SNP projections (the scan's GEMM)
    // Several traits of one request over the same basis, covariates and window: the first
    // scan projects [U | X | py | y_1 - ybar_1 .. y_t - ybar_t] once; every later trait's py
    // column follows from its y column (py = b (y - X bX) + U (c o U^T r), G_c^T 1 = 0)
    // without a genotype pass.
    int64_t trait = -1;
    if (l->trait_t > 0 && (int64_t)l->trait_Y.size() == n * l->trait_t)
        for (int64_t j = 0; j < l->trait_t && trait < 0; ++j)
            if (std::memcmp(l->trait_Y.data() + j * n, y, 8 * n) == 0) trait = j;
    const double* Tptr = l->d_T.get();
    int64_t ldt = bw;
    if (trait >= 0) {
        const int64_t tc = l->trait_t, ldc = bw + tc;
        const double one = 1.0;
        const bool valid = cached && l->tcache_valid && l->tcache_gen == l->basis_gen &&
                           l->tcache_prec == precision && l->tcache_X == l->X &&
                           (precision != CS_PRECISION_MIXED || l->scan_mixed);
        l->d_tc.resize(M * ldc);
        if (!valid) {
            l->d_bt.resize(n * ldc);
            std::vector<double> hy(n * tc);
            for (int64_t j = 0; j < tc; ++j) {
                const double* yj = l->trait_Y.data() + j * n;
                double mean = 0.0;
                for (int64_t i = 0; i < n; ++i) mean += yj[i];
                mean /= (double)n;
                for (int64_t i = 0; i < n; ++i) hy[i * tc + j] = yj[i] - mean;
            }
            CS_CUDA(cudaMemcpy2DAsync(l->d_bt.get(), 8 * ldc, Bm, 8 * bw, 8 * bw, n,
                                      cudaMemcpyDeviceToDevice, s));
            CS_CUDA(cudaMemcpy2DAsync(l->d_bt.get() + bw, 8 * ldc, hy.data(), 8 * tc, 8 * tc, n,
                                      cudaMemcpyHostToDevice, s));
            if (precision == CS_PRECISION_MIXED) {
                if (!cached || !l->scan_mixed) {
                    mixed_scan_destroy(l->scan_mixed);
                    l->scan_mixed = nullptr;
                    l->scan_mixed = mixed_scan_create(v, row_mean.data(), counts.data());
                }
                mixed_scan_project(l->scan_mixed, l->d_bt.get(), ldc, ldc, l->d_tc.get(), ldc, s);
            } else {
                Workspace ws;
                decode_gemm_rows_fp64(v, l->d_lut.get(), l->d_bt.get(), ldc, ldc, l->d_tc.get(),
                                      ldc, ws, s);
            }
            CS_CUDA(cudaStreamSynchronize(s));  // hy is a host temporary
            l->tcache_valid = true;
            l->tcache_gen = l->basis_gen;
            l->tcache_prec = precision;
            l->tcache_X = l->X;
        } else {
            l->d_betax.resize(std::max<int64_t>(1, p));
            if (p)
                CS_CUDA(cudaMemcpyAsync(l->d_betax.get(), betaX.data(), 8 * p,
                                        cudaMemcpyHostToDevice, s));
            {
                prof::Scope ps("scan_py_from_y", s, 0.0, 8.0 * (double)M * (p + 2));
                k_scan_py_from_y<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(
                                       (M + 255) / 256, 32LL * num_sms())),
                                   256, 0, s>>>(l->d_tc.get(), ldc, r, (int)p, bw + trait,
                                                l->d_betax.get(), base, M);
                CS_LAUNCH("scan_py_from_y");
            }
            // py column += U block (c o U^T resid)
            CS_BLAS(cublasDgemv(l->blas, CUBLAS_OP_T, (int)r, (int)M, &one, l->d_tc.get(), (int)ldc,
                                l->d_d.get(), 1, &one, l->d_tc.get() + r + p, (int)ldc));
        }
        Tptr = l->d_tc.get();
        ldt = ldc;
    } else if (precision == CS_PRECISION_MIXED) {
        if (!cached || !l->scan_mixed) {
            mixed_scan_destroy(l->scan_mixed);
            l->scan_mixed = nullptr;
            l->scan_mixed = mixed_scan_create(v, row_mean.data(), counts.data());
        }
        // The U block from the kept sketch apply when every analysed sample is in the
        // operator (then the scan's centring means are the operator's) and every SNP that can
        // be tested has an operator row.  X and py come from the same apply when it carried
        // [X | y - ybar] for this y and X (py = b resid + U (c o U^T resid), resid = y - X bX,
        // and G_c^T 1 = 0), else from one narrow genotype pass.
        // (CS_B200_SCAN_REUSE=0 always takes the full projection)
        const char* env = std::getenv("CS_B200_SCAN_REUSE");
        bool reuse = !(env && env[0] == '0') && l->sketch_g_uid == g->uid && l->ztq_cols > 0 &&
                     n_keep == g->n_samples && l->ztq_sk == l->sketch_diag.sketch_size;
        const bool fused_cols = reuse && l->fused_p == p && l->ztq_cols == l->ztq_sk + p + 1 &&
                                l->fused_y == l->y && l->fused_X == l->X;
        for (int64_t i = 0; reuse && i < n_keep; ++i) reuse = keep[i] == i;
        std::vector<int32_t> win_rows;
        if (reuse) {
            win_rows.resize(M);
            for (int64_t j = 0; j < M; ++j) {
                win_rows[j] = l->snp_row[snp_begin + j];
                if (pass[j] && win_rows[j] < 0) reuse = false;
            }
        }
        if (reuse) {
            const int64_t R = l->ztq_rows, kq = l->ztq_sk;
            const double one = 1.0, zero = 0.0;
            l->d_ztq_u.resize(r * R);
            // C (r x R) = W_sel^T (Z_c^T Q s^2)^T
            CS_BLAS(cublasDgemm(l->blas, CUBLAS_OP_T, CUBLAS_OP_T, (int)r, (int)R, (int)kq, &one,
                                l->d_wsel.get(), (int)kq, l->d_ztq.get(), (int)R, &zero,
                                l->d_ztq_u.get(), (int)r));
            l->d_win_rows.resize(M);
            CS_CUDA(cudaMemcpyAsync(l->d_win_rows.get(), win_rows.data(), 4 * M,
                                    cudaMemcpyHostToDevice, s));
            {
                prof::Scope ps("scan_u_block", s, 0.0, 16.0 * (double)M * r);
                k_scan_u_block<<<(unsigned)std::min<int64_t>((M * r + 255) / 256, 32LL * num_sms()), 256,
                                 0, s>>>(l->d_ztq_u.get(), r, l->d_win_rows.get(), l->d_s2inv.get(), M,
                                         l->d_T.get(), bw);
                CS_LAUNCH("scan_u_block");
            }
            if (fused_cols) {
                l->d_betax.resize(std::max<int64_t>(1, p));
                if (p)
                    CS_CUDA(cudaMemcpyAsync(l->d_betax.get(), betaX.data(), 8 * p,
                                            cudaMemcpyHostToDevice, s));
                {
                    prof::Scope ps("scan_fused_columns", s, 0.0, 8.0 * (double)M * (p + 2));
                    k_scan_fused_cols<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(
                                            (M + 255) / 256, 32LL * num_sms())),
                                        256, 0, s>>>(l->d_ztq.get() + kq * R, R, (int)p,
                                                     l->d_win_rows.get(), l->d_s2inv.get(),
                                                     l->d_betax.get(), base, M, l->d_T.get() + r,
                                                     bw);
                    CS_LAUNCH("scan_fused_columns");
                }
                // py column += U block (c o U^T resid)
                CS_BLAS(cublasDgemv(l->blas, CUBLAS_OP_T, (int)r, (int)M, &one, l->d_T.get(), (int)bw,
                                    l->d_d.get(), 1, &one, l->d_T.get() + r + p, (int)bw));
            } else {
                mixed_scan_project(l->scan_mixed, Bm + r, bw, bw - r, l->d_T.get() + r, bw, s);
            }
        } else {
            mixed_scan_project(l->scan_mixed, Bm, bw, bw, l->d_T.get(), bw, s);
        }
    } else {
        Workspace ws;
        decode_gemm_rows_fp64(v, l->d_lut.get(), Bm, bw, bw, l->d_T.get(), bw, ws, s);
    }
    ScanParams P;
    P.n_snps = M; P.rank = r; P.p = p; P.ldt = ldt; P.base = base;
    P.T = Tptr; P.c = l->d_cv.get(); P.UtX = l->d_utx.get(); P.info_inv = l->d_inv.get();
    P.gnorm2 = l->d_gn2.get(); P.pass = l->d_pass.get();
    P.beta = l->d_beta.get(); P.se = l->d_se.get(); P.pval = l->d_p.get();
    P.log10p = l->d_l10.get();
    P.tested = l->d_tested.get();
    {
        const int blocks = (int)std::min<int64_t>((M * 32 + 255) / 256, 64LL * num_sms());
        prof::Scope ps("scan_epilogue", s, 0.0, 8.0 * (double)M * bw);
        k_scan_epilogue<<<std::max(blocks, 1), 256, 0, s>>>(P);
        CS_LAUNCH("scan_epilogue");
    }
    {
        prof::Scope ps("scan_pvalues", s, 0.0, 37.0 * (double)M);
        k_scan_pvalues<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((M + 127) / 128,
                                                                            16LL * num_sms())),
                         128, 0, s>>>(P);
        CS_LAUNCH("scan_pvalues");
    }
    scan_finish(l, M, fr, beta, se, pvalue, log10p, freq, tested, s);
}

}  // namespace cs
