// Dense exact tier of the LMM: the genomic relationship matrix, its eigenbasis and the Brent
// null model, all resident on the device.
//
//   grm_create      GrmBuilder::compute (libCosmicCore/src/grm_builder.cpp:87-394), one
//                   population, unit SNP weights, no HWE filter
//   eigen_prepare   EigenVce::prepare (libCosmicCore/src/eigen_vce.cpp:19-63)
//   eigen_run_null  EigenVce::runNullModel, Brent branch (eigen_vce.cpp:83-112) =
//                   VCESolver::solveDiagonal (libCosmicCore/src/vce.cpp:3073-3175), then
//                   updateRemlDiagnostics (eigen_vce.cpp:114-153)
//
// Device work: decoding 2048-SNP blocks of centred genotypes (the reference's block size) and
// accumulating G += Z Z^T with cuBLAS DSYRK (a plain library GEMM on the decoded block);
// symmetrising and normalising G in shared-memory tiles; gathering G[keep, keep]; the
// covariate projection as one rank-2p update; the eigendecomposition (cuSOLVER syevd, 64-bit
// interface, so n^2 may exceed 2^31).  Host work: per-SNP statistics from the code counts
// (float roundings as the reference stores them), the Gram-Schmidt basis of X (n x p,
// p <= 16), and the golden-section search, which costs O(n p^2) per evaluation.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "cs_internal.h"
#include "dense_internal.h"
#include "linalg_host.h"
#include "vce_internal.h"

namespace cs {

namespace {

constexpr int64_t kGrmBlock = 2048;  // GrmBuilder::Options::block_size

// Z (n x b, column-major) of the block: Z[i, c] = lut[4 c + code(rows[c], i)].
__global__ void k_grm_decode(const uint8_t* __restrict__ packed, int64_t stride,
                             const int32_t* __restrict__ rows, const double* __restrict__ lut,
                             int64_t n, double* __restrict__ Z) {
    const int64_t c = blockIdx.y;
    const int64_t bytes = (n + 3) / 4;
    const uint8_t* src = packed + (int64_t)rows[c] * stride;
    const double v0 = lut[4 * c], v1 = lut[4 * c + 1], v2 = lut[4 * c + 2], v3 = lut[4 * c + 3];
    double* dst = Z + c * n;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < bytes;
         q += (int64_t)gridDim.x * blockDim.x) {
        const unsigned byte = src[q];
        const int64_t i = 4 * q;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (i + k < n) {
                const unsigned code = (byte >> (2 * k)) & 3u;
                dst[i + k] = code == 0 ? v0 : code == 1 ? v1 : code == 2 ? v2 : v3;
            }
        }
    }
}

// The lower triangle (DSYRK's output) divided by div, mirrored into the upper one through a
// shared-memory tile so both the read and the transposed write are coalesced.
__global__ void k_grm_finish(double* __restrict__ G, int64_t n, double div) {
    __shared__ double tile[32][33];
    const int64_t ti = blockIdx.x, tj = blockIdx.y;
    if (ti < tj) return;
    const int64_t i0 = ti * 32, j0 = tj * 32;
    const int tx = threadIdx.x;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int64_t i = i0 + tx, j = j0 + k;
        double v = 0.0;
        if (i < n && j < n && i >= j) {
            v = G[i + j * n] / div;
            G[i + j * n] = v;
        }
        tile[tx][k] = v;
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int64_t j = j0 + tx, i = i0 + k;
        if (i < n && j < n && i > j) G[j + i * n] = tile[k][tx];
    }
}

// out = a * G - (b * R) / c, elementwise (the LOCO GRM of src/gwas_scanner.cpp:489).
__global__ void k_loco_combine(const double* __restrict__ G, const double* __restrict__ R,
                               int64_t total, double a, double b, double c,
                               double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = G[i] * a - (R[i] * b) / c;
}

// out[i + j ld] = G[keep[i] + keep[j] N] (DataFilter::subsetSquare).
__global__ void k_gather_square(const double* __restrict__ G, int64_t N,
                                const int32_t* __restrict__ keep, int64_t nk,
                                double* __restrict__ out, int64_t ld) {
    for (int64_t j = blockIdx.y; j < nk; j += gridDim.y) {
        const double* col = G + (int64_t)keep[j] * N;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nk;
             i += (int64_t)gridDim.x * blockDim.x)
            out[i + j * ld] = col[keep[i]];
    }
}

// Column sums of |A| (n x n, ld n): a Gershgorin bound of the spectrum is their maximum.
__global__ void k_abs_col_sums(const double* __restrict__ A, int64_t n, double* __restrict__ out) {
    __shared__ double red[8];
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x) {
        double acc = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += fabs(A[i + j * n]);
        for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
            out[j] = t;
        }
        __syncthreads();
    }
}

// Per-SNP statistics and value map of GrmBuilder::compute (grm_builder.cpp:187-312) from the
// code counts c00 (hom A1, x = 2), c01 (missing), c10 (het), c11 (hom A2, x = 0).
struct GrmSnp {
    bool valid = false;
    double lut[4] = {0, 0, 0, 0};
    float two_pq = 0.0f;
};

GrmSnp grm_snp(const int32_t* cnt, int algorithm, float min_maf) {
    GrmSnp out;
    const long long n_hom1 = cnt[0], n_het = cnt[2], n_hom2 = cnt[3];
    const long long n_obs = n_hom1 + n_het + n_hom2;
    if (n_obs == 0) return out;
    const long long sum_x = 2 * n_hom1 + n_het;
    const double freq = (double)sum_x / (2.0 * n_obs);
    const double maf = std::min(freq, 1.0 - freq);
    if (maf < min_maf || std::abs(maf) < 1e-8) return out;
    // float-rounded 2pq (or its algorithm variant) as the reference stores it: the GRM's
    // block sums of these floats must group identically for parity
    if (algorithm == 4) {
        out.two_pq = (float)(4.0 * freq * freq * (1.0 - freq) * (1.0 - freq));
    } else if (algorithm == 5) {
        const double p1 = (double)n_het / n_obs, p2 = (double)n_hom1 / n_obs;
        const double mu = p1 + 2.0 * p2;
        out.two_pq = (float)(p1 + 4.0 * p2 - mu * mu);
    } else {
        out.two_pq = (float)(2.0 * freq * (1.0 - freq));
    }
    const float mean_f = (float)(freq * 2.0);
    float scale_f = 1.0f;
    if (algorithm == 0 || algorithm == 3) {
        const double pq2 = 2.0 * freq * (1.0 - freq);
        scale_f = (float)((pq2 > 1e-9) ? (1.0 / std::sqrt(pq2)) : 0.0);
    } else if (algorithm == 5) {
        const double p1 = (double)n_het / n_obs, p2 = (double)n_hom1 / n_obs;
        const double mu = p1 + 2.0 * p2;
        const double var = p1 + 4.0 * p2 - mu * mu;
        scale_f = (float)((var > 1e-9) ? (1.0 / std::sqrt(var)) : 0.0);
    }
    const double mean = mean_f;
    const double scale = scale_f;
    if (algorithm == 4) {
        const double fp = mean / 2.0, fq = 1.0 - fp;
        out.lut[0] = (-2.0 * fq * fq) * scale;
        out.lut[2] = (2.0 * fp * fq) * scale;
        out.lut[3] = (-2.0 * fp * fp) * scale;
    } else if (algorithm == 2) {
        const double fp = mean / 2.0;
        out.lut[0] = (1.0 - fp) * scale;
        out.lut[2] = (1.0 - 2.0 * fp) * scale;
        out.lut[3] = (-fp) * scale;
    } else {
        out.lut[0] = (2.0 - mean) * scale;
        out.lut[2] = (1.0 - mean) * scale;
        out.lut[3] = (0.0 - mean) * scale;
    }
    out.lut[1] = 0.0;
    out.valid = true;
    return out;
}

void symmetric_eigh(double* A, int64_t n, double* d_w, cudaStream_t s) {
    cusolverDnHandle_t sol = shared_solver();
    CS_SOLVER(cusolverDnSetStream(sol, s));
    cusolverDnParams_t params = nullptr;
    CS_SOLVER(cusolverDnCreateParams(&params));
    size_t dev_bytes = 0, host_bytes = 0;
    cusolverStatus_t st = cusolverDnXsyevd_bufferSize(
        sol, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, A, n,
        CUDA_R_64F, d_w, CUDA_R_64F, &dev_bytes, &host_bytes);
    if (st != CUSOLVER_STATUS_SUCCESS) {
        cusolverDnDestroyParams(params);
        CS_SOLVER(st);
    }
    DeviceBuffer<char> dwork;
    dwork.resize(std::max<size_t>(dev_bytes, 1));
    std::vector<char> hwork(std::max<size_t>(host_bytes, 1));
    DeviceBuffer<int> info;
    info.resize(1);
    st = cusolverDnXsyevd(sol, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n,
                          CUDA_R_64F, A, n, CUDA_R_64F, d_w, CUDA_R_64F, dwork.get(), dev_bytes,
                          hwork.data(), host_bytes, info.get());
    cusolverDnDestroyParams(params);
    CS_SOLVER(st);
    int h_info = 0;
    CS_CUDA(cudaMemcpyAsync(&h_info, info.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    if (h_info != 0)
        fail(CS_ERR_NUMERIC, "EigenVce: eigendecomposition failed (syevd info " +
                                 std::to_string(h_info) + ")");
}

}  // namespace

cs_grm* grm_create(const cs_genotypes* g, const int32_t* variants, int64_t n_variants,
                   const cs_grm_options* opt) {
    if (!g) fail(CS_ERR_INVALID_ARGUMENT, "GrmBuilder: null genotypes");
    cs_grm_options o;
    cs_grm_default_options(&o);
    if (opt) o = *opt;
    if (o.algorithm < 0 || o.algorithm > 5)
        fail(CS_ERR_INVALID_ARGUMENT, "GrmBuilder: unknown algorithm " + std::to_string(o.algorithm));
    const int64_t N = g->n_samples, M = g->n_snps;
    if (N == 0 || M == 0) fail(CS_ERR_INVALID_ARGUMENT, "Empty dataset provided to GrmBuilder");
    std::vector<int32_t> sel;
    if (variants) {
        if (n_variants < 0) fail(CS_ERR_INVALID_ARGUMENT, "GrmBuilder: negative variant count");
        sel.assign(variants, variants + n_variants);
        for (size_t t = 0; t < sel.size(); ++t)
            if (sel[t] < 0 || sel[t] >= M || (t && sel[t] <= sel[t - 1]))
                fail(CS_ERR_INVALID_ARGUMENT,
                     "GrmBuilder: variants must be increasing SNP indices of the .bed");
    } else {
        sel.resize(M);
        for (int64_t t = 0; t < M; ++t) sel[t] = (int32_t)t;
    }
    cudaStream_t s = 0;
    cublasHandle_t blas = shared_blas();
    CS_BLAS(cublasSetStream(blas, s));
    auto* grm = new cs_grm();
    try {
        grm->n = N;
        grm->algorithm = o.algorithm;
        grm->G.resize(N * N);
        CS_CUDA(cudaMemsetAsync(grm->G.get(), 0, 8 * N * N, s));
        // code counts of every SNP over every sample
        std::vector<int32_t> counts(4 * M);
        {
            DeviceBuffer<int32_t> d_counts;
            d_counts.resize(4 * M);
            row_code_counts(cs_packed_view{g->packed.get(), M, N, g->stride}, d_counts.get(), s);
            CS_CUDA(cudaMemcpyAsync(counts.data(), d_counts.get(), 16 * M, cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaStreamSynchronize(s));
        }
        // the reference's blocks are ranges of the .bed; 2pq sums per block, then over blocks
        const float min_maf = (float)o.min_maf;
        double total_2pq = 0.0;
        int64_t total_valid = 0;
        std::vector<int32_t> rows;
        std::vector<double> lut;
        rows.reserve(kGrmBlock);
        lut.reserve(4 * kGrmBlock);
        DeviceBuffer<int32_t> d_rows;
        DeviceBuffer<double> d_lut, Z;
        d_rows.resize(kGrmBlock);
        d_lut.resize(4 * kGrmBlock);
        Z.resize(N * kGrmBlock);
        bool first = true;
        auto flush = [&]() {
            const int64_t b = (int64_t)rows.size();
            if (b == 0) return;
            CS_CUDA(cudaMemcpyAsync(d_rows.get(), rows.data(), 4 * b, cudaMemcpyHostToDevice, s));
            CS_CUDA(cudaMemcpyAsync(d_lut.get(), lut.data(), 32 * b, cudaMemcpyHostToDevice, s));
            {
                prof::Scope ps("grm_decode", s, 0.0, (double)b * ((N + 3) / 4) + 8.0 * N * b);
                const int64_t bytes = (N + 3) / 4;
                dim3 grid((unsigned)std::min<int64_t>((bytes + 255) / 256, 64), (unsigned)b);
                k_grm_decode<<<grid, 256, 0, s>>>(g->packed.get(), g->stride, d_rows.get(),
                                                  d_lut.get(), N, Z.get());
                CS_LAUNCH("grm_decode");
            }
            const double one = 1.0;
            const double beta = first ? 0.0 : 1.0;
            CS_BLAS(cublasDsyrk(blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, (int)N, (int)b, &one,
                                Z.get(), (int)N, &beta, grm->G.get(), (int)N));
            first = false;
            // the next block's host arrays are refilled only after this one's copies ran
            CS_CUDA(cudaStreamSynchronize(s));
            rows.clear();
            lut.clear();
        };
        size_t t = 0;
        while (t < sel.size()) {
            const int64_t block = sel[t] / kGrmBlock;
            double block_2pq = 0.0;
            int64_t block_valid = 0;
            for (; t < sel.size() && sel[t] / kGrmBlock == block; ++t) {
                const GrmSnp st = grm_snp(&counts[4 * (int64_t)sel[t]], o.algorithm, min_maf);
                if (!st.valid) continue;
                block_2pq += st.two_pq;
                ++block_valid;
                rows.push_back(sel[t]);
                lut.insert(lut.end(), st.lut, st.lut + 4);
                if ((int64_t)rows.size() == kGrmBlock) flush();
            }
            total_2pq += block_2pq;
            total_valid += block_valid;
        }
        flush();
        grm->n_valid = total_valid;
        grm->sum_2pq = total_2pq;
        // normalisation (grm_builder.cpp:383-391): no valid SNP leaves G = 0
        double div = 1.0;
        if (o.algorithm == 0 || o.algorithm == 3) {
            if (total_valid > 0) div = (double)total_valid;
        } else if (o.algorithm == 2) {
            std::vector<double> diag(N);
            CS_CUDA(cudaMemcpy2DAsync(diag.data(), 8, grm->G.get(), 8 * (N + 1), 8, N,
                                      cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaStreamSynchronize(s));
            double tr = 0.0;
            for (double v : diag) tr += v;
            if (tr > 0) div = tr / (double)N;
        } else {
            if (total_2pq > 0) div = total_2pq;
        }
        grm->div = div;
        {
            prof::Scope ps("grm_finish", s, 0.0, 16.0 * N * N);
            const unsigned tiles = (unsigned)((N + 31) / 32);
            k_grm_finish<<<dim3(tiles, tiles), dim3(32, 8), 0, s>>>(grm->G.get(), N, div);
            CS_LAUNCH("grm_finish");
        }
        CS_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        delete grm;
        throw;
    }
    return grm;
}

cs_grm* grm_loco(const cs_grm* global, const cs_grm* chrom) {
    if (!global || !chrom) fail(CS_ERR_INVALID_ARGUMENT, "grm_loco: null argument");
    if (global->n != chrom->n || global->algorithm != chrom->algorithm)
        fail(CS_ERR_INVALID_ARGUMENT, "grm_loco: the matrices differ in samples or algorithm");
    const int64_t n = global->n;
    // S = the valid-SNP count (algorithms 0, 3) or the 2pq sum (src/gwas_scanner.cpp:484-486)
    const bool by_count = global->algorithm == 0 || global->algorithm == 3;
    const double s_global = by_count ? (double)global->n_valid : global->sum_2pq;
    const double s_chr = by_count ? (double)chrom->n_valid : chrom->sum_2pq;
    const double s_loco = s_global - s_chr;
    auto* out = new cs_grm();
    try {
        out->n = n;
        out->algorithm = global->algorithm;
        out->n_valid = global->n_valid - chrom->n_valid;
        out->sum_2pq = global->sum_2pq - chrom->sum_2pq;
        out->G.resize(n * n);
        if (s_chr > 0.0 && s_loco > 1e-6) {
            // G_loco = G_global (S_global / S_loco) - raw_chr / S_loco, raw_chr = G_chr div_chr
            out->div = s_loco;
            prof::Scope ps("grm_loco", 0, 0.0, 24.0 * n * n);
            const int64_t total = n * n;
            k_loco_combine<<<(unsigned)std::min<int64_t>((total + 255) / 256, 64LL * num_sms()), 256>>>(
                global->G.get(), chrom->G.get(), total, s_global / s_loco, chrom->div, s_loco,
                out->G.get());
            CS_LAUNCH("grm_loco");
        } else {
            out->div = global->div;
            CS_CUDA(cudaMemcpy(out->G.get(), global->G.get(), 8 * n * n, cudaMemcpyDeviceToDevice));
        }
        CS_CUDA(cudaDeviceSynchronize());
    } catch (...) {
        delete out;
        throw;
    }
    return out;
}

cs_grm* grm_from_host(int64_t n, const double* G, int64_t ldg) {
    if (n <= 0 || !G || ldg < n) fail(CS_ERR_INVALID_ARGUMENT, "grm_from_host: bad dimensions");
    auto* grm = new cs_grm();
    try {
        grm->n = n;
        grm->G.resize(n * n);
        CS_CUDA(cudaMemcpy2D(grm->G.get(), 8 * n, G, 8 * ldg, 8 * n, n, cudaMemcpyHostToDevice));
    } catch (...) {
        delete grm;
        throw;
    }
    return grm;
}

void grm_copy(const cs_grm* grm, const int32_t* keep, int64_t n_keep, double* out, int64_t ld) {
    if (!grm || !out) fail(CS_ERR_INVALID_ARGUMENT, "grm_copy: null argument");
    const int64_t N = grm->n;
    if (!keep) {
        if (ld < N) fail(CS_ERR_INVALID_ARGUMENT, "grm_copy: ld < n");
        CS_CUDA(cudaMemcpy2D(out, 8 * ld, grm->G.get(), 8 * N, 8 * N, N, cudaMemcpyDeviceToHost));
        return;
    }
    if (n_keep <= 0 || ld < n_keep) fail(CS_ERR_INVALID_ARGUMENT, "grm_copy: bad keep size");
    for (int64_t i = 0; i < n_keep; ++i)
        if (keep[i] < 0 || keep[i] >= N) fail(CS_ERR_INVALID_ARGUMENT, "grm_copy: keep index out of range");
    DeviceBuffer<int32_t> d_keep;
    DeviceBuffer<double> sub;
    d_keep.resize(n_keep);
    sub.resize(n_keep * n_keep);
    CS_CUDA(cudaMemcpy(d_keep.get(), keep, 4 * n_keep, cudaMemcpyHostToDevice));
    k_gather_square<<<dim3((unsigned)((n_keep + 255) / 256), (unsigned)std::min<int64_t>(n_keep, 65535)),
                      256>>>(grm->G.get(), N, d_keep.get(), n_keep, sub.get(), n_keep);
    CS_LAUNCH("gather_square");
    CS_CUDA(cudaMemcpy2D(out, 8 * ld, sub.get(), 8 * n_keep, 8 * n_keep, n_keep, cudaMemcpyDeviceToHost));
}

std::shared_ptr<DenseNull> eigen_basis(const cs_grm* grm, const int32_t* keep, int64_t n_keep,
                                       const double* y, int64_t nt, const double* X, int64_t p,
                                       bool projection) {
    if (!grm || !y || nt < 1 || p < 0 || (p > 0 && !X))
        fail(CS_ERR_INVALID_ARGUMENT, "EigenVce::prepare: null argument");
    if (p > 16) fail(CS_ERR_UNSUPPORTED, "at most 16 covariate columns are supported");
    const int64_t N = grm->n;
    const int64_t n = keep ? n_keep : N;
    if (keep) {
        if (n_keep <= 0) fail(CS_ERR_INVALID_ARGUMENT, "EigenVce::prepare: Dimension mismatch");
        for (int64_t i = 0; i < n_keep; ++i)
            if (keep[i] < 0 || keep[i] >= N)
                fail(CS_ERR_INVALID_ARGUMENT, "EigenVce::prepare: keep index out of range");
    }
    if (projection && p >= n) fail(CS_ERR_INVALID_ARGUMENT, "EigenVce::prepare: no residual dimension");
    cudaStream_t s = 0;
    cublasHandle_t blas = shared_blas();
    CS_BLAS(cublasSetStream(blas, s));
    {
        auto d = std::make_shared<DenseNull>();
        d->n = n;
        d->traits = nt;
        DeviceBuffer<double>& A = d->W;  // G[keep, keep], then its eigenvectors
        A.resize(n * n);
        if (keep) {
            DeviceBuffer<int32_t> d_keep;
            d_keep.resize(n);
            CS_CUDA(cudaMemcpyAsync(d_keep.get(), keep, 4 * n, cudaMemcpyHostToDevice, s));
            prof::Scope ps("gather_square", s, 0.0, 16.0 * n * n);
            k_gather_square<<<dim3((unsigned)((n + 255) / 256), (unsigned)std::min<int64_t>(n, 65535)),
                              256, 0, s>>>(grm->G.get(), N, d_keep.get(), n, A.get(), n);
            CS_LAUNCH("gather_square");
            CS_CUDA(cudaStreamSynchronize(s));
        } else {
            CS_CUDA(cudaMemcpyAsync(A.get(), grm->G.get(), 8 * n * n, cudaMemcpyDeviceToDevice, s));
        }
        const bool project = projection && p > 0;
        double alpha = 0.0, bound = 0.0;
        if (project) {
            // Q_x: orthonormal basis of span(X) by Gram-Schmidt applied twice
            std::vector<double> Q(X, X + n * p);
            for (int64_t a = 0; a < p; ++a) {
                double* qa = &Q[a * n];
                double norm0 = 0.0;
                for (int64_t i = 0; i < n; ++i) norm0 += qa[i] * qa[i];
                norm0 = std::sqrt(norm0);
                for (int pass = 0; pass < 2; ++pass)
                    for (int64_t b = 0; b < a; ++b) {
                        const double* qb = &Q[b * n];
                        double dot = 0.0;
                        for (int64_t i = 0; i < n; ++i) dot += qb[i] * qa[i];
                        for (int64_t i = 0; i < n; ++i) qa[i] -= dot * qb[i];
                    }
                double norm = 0.0;
                for (int64_t i = 0; i < n; ++i) norm += qa[i] * qa[i];
                norm = std::sqrt(norm);
                if (!(norm > 1e-10 * std::max(norm0, 1e-300)))
                    fail(CS_ERR_NUMERIC, "EigenVce::prepare: covariate matrix is rank deficient");
                for (int64_t i = 0; i < n; ++i) qa[i] /= norm;
            }
            // alpha above the spectrum of P G P: 1.5 x the Gershgorin bound of G + 1
            {
                DeviceBuffer<double> sums;
                sums.resize(n);
                prof::Scope ps("abs_col_sums", s, 0.0, 8.0 * n * n);
                k_abs_col_sums<<<(unsigned)std::min<int64_t>(n, 8LL * num_sms()), 256, 0, s>>>(
                    A.get(), n, sums.get());
                CS_LAUNCH("abs_col_sums");
                std::vector<double> h(n);
                CS_CUDA(cudaMemcpyAsync(h.data(), sums.get(), 8 * n, cudaMemcpyDeviceToHost, s));
                CS_CUDA(cudaStreamSynchronize(s));
                for (double x : h) bound = std::max(bound, x);
            }
            alpha = 1.5 * bound + 1.0;
            DeviceBuffer<double> dQ, B, C;
            dQ.resize(n * p);
            B.resize(n * p);
            C.resize(p * p);
            CS_CUDA(cudaMemcpyAsync(dQ.get(), Q.data(), 8 * n * p, cudaMemcpyHostToDevice, s));
            const double one = 1.0, zero = 0.0, minus_one = -1.0;
            // B = G Q, C = Q^T B
            CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)p, (int)n, &one, A.get(),
                                (int)n, dQ.get(), (int)n, &zero, B.get(), (int)n));
            CS_BLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)p, (int)p, (int)n, &one, dQ.get(),
                                (int)n, B.get(), (int)n, &zero, C.get(), (int)p));
            std::vector<double> hC(p * p);
            CS_CUDA(cudaMemcpyAsync(hC.data(), C.get(), 8 * p * p, cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaStreamSynchronize(s));
            // F = B - Q (C + alpha I) / 2, so G - Q F^T - F Q^T = P G P + alpha Q Q^T
            std::vector<double> Ca(p * p);
            for (int64_t a = 0; a < p; ++a)
                for (int64_t b = 0; b < p; ++b)
                    Ca[a + b * p] = 0.5 * (hC[a + b * p] + hC[b + a * p]) + (a == b ? alpha : 0.0);
            CS_CUDA(cudaMemcpyAsync(C.get(), Ca.data(), 8 * p * p, cudaMemcpyHostToDevice, s));
            const double minus_half = -0.5;
            CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)p, (int)p, &minus_half,
                                dQ.get(), (int)n, C.get(), (int)p, &one, B.get(), (int)n));
            CS_BLAS(cublasDsyr2k(blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, (int)n, (int)p,
                                 &minus_one, dQ.get(), (int)n, B.get(), (int)n, &one, A.get(),
                                 (int)n));
            CS_CUDA(cudaStreamSynchronize(s));
        }
        DeviceBuffer<double> w;
        w.resize(n);
        {
            prof::HostScope hs("eigen_vce_eigh");
            symmetric_eigh(A.get(), n, w.get(), s);
        }
        std::vector<double> evals(n);
        CS_CUDA(cudaMemcpy(evals.data(), w.get(), 8 * n, cudaMemcpyDeviceToHost));
        d->projected = project;
        d->n_eig = project ? n - p : n;
        d->p = project ? 0 : p;
        if (project) {
            // the p covariate directions carry alpha; everything else lies below the bound
            for (int64_t j = d->n_eig; j < n; ++j)
                if (!(evals[j] > 1.25 * bound + 0.5))
                    fail(CS_ERR_NUMERIC, "EigenVce::prepare: covariate directions did not separate");
            if (d->n_eig > 0 && !(evals[d->n_eig - 1] < 1.25 * bound + 0.5))
                fail(CS_ERR_NUMERIC, "EigenVce::prepare: covariate directions did not separate");
        }
        d->D.assign(evals.begin(), evals.begin() + d->n_eig);
        for (double& x : d->D)
            if (x < 0) x = 0;
        // Uty = W^T Y (n_eig x nt); UtX = W^T X (no projection)
        {
            DeviceBuffer<double> dy, out;
            dy.resize(n * (nt + d->p));
            out.resize(d->n_eig * (nt + d->p));
            CS_CUDA(cudaMemcpyAsync(dy.get(), y, 8 * n * nt, cudaMemcpyHostToDevice, s));
            if (d->p)
                CS_CUDA(cudaMemcpyAsync(dy.get() + n * nt, X, 8 * n * d->p, cudaMemcpyHostToDevice, s));
            const double one = 1.0, zero = 0.0;
            CS_BLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)d->n_eig, (int)(nt + d->p), (int)n,
                                &one, A.get(), (int)n, dy.get(), (int)n, &zero, out.get(),
                                (int)d->n_eig));
            std::vector<double> h(d->n_eig * (nt + d->p));
            CS_CUDA(cudaMemcpyAsync(h.data(), out.get(), 8 * h.size(), cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaStreamSynchronize(s));
            d->Uty.assign(h.begin(), h.begin() + d->n_eig * nt);
            d->UtX.assign(h.begin() + d->n_eig * nt, h.end());
        }
        return d;
    }
}

cs_eigen_vce* eigen_prepare(const cs_grm* grm, const int32_t* keep, int64_t n_keep,
                            const double* y, const double* X, int64_t p, bool projection) {
    auto d = eigen_basis(grm, keep, n_keep, y, 1, X, p, projection);
    auto* v = new cs_eigen_vce();
    v->d = std::move(d);
    v->result.n_eig = v->d->n_eig;
    return v;
}

namespace {

// (X^T V^-1 X, X^T V^-1 y) at V = D + delta, its LDLT, the GLS fit and the REML objective of
// VCESolver::solveDiagonal's calc_neg_logL (vce.cpp:3090-3116).
struct DiagFit {
    std::vector<double> L, Dl, beta;
    double quad = 0.0, log_det_v = 0.0, log_det_xvx = 0.0;
    bool ok = true;
};

DiagFit diag_fit(const DenseNull& d, double delta) {
    const int64_t n = d.n_eig, p = d.p;
    DiagFit f;
    std::vector<double> xvx(p * p, 0.0), xvy(p, 0.0), vinv(n);
    for (int64_t i = 0; i < n; ++i) {
        const double vd = d.D[i] + delta;
        vinv[i] = 1.0 / vd;
        f.log_det_v += std::log(vd);
    }
    for (int64_t a = 0; a < p; ++a) {
        for (int64_t b = 0; b <= a; ++b) {
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) acc += d.UtX[i + a * n] * vinv[i] * d.UtX[i + b * n];
            xvx[a + b * p] = xvx[b + a * p] = acc;
        }
        double acc = 0.0;
        for (int64_t i = 0; i < n; ++i) acc += d.UtX[i + a * n] * vinv[i] * d.Uty[i];
        xvy[a] = acc;
    }
    f.beta = xvy;
    if (p > 0) {
        f.ok = la::ldlt(xvx, (int)p, f.L, f.Dl);
        if (f.ok) la::ldlt_solve(f.L, f.Dl, (int)p, f.beta.data());
        for (double x : f.Dl) f.log_det_xvx += std::log(x);
    }
    for (int64_t i = 0; i < n; ++i) {
        double r = d.Uty[i];
        for (int64_t a = 0; a < p; ++a) r -= d.UtX[i + a * n] * f.beta[a];
        f.quad += r * r * vinv[i];
    }
    return f;
}

double neg_reml(const DenseNull& d, double delta) {
    const DiagFit f = diag_fit(d, delta);
    const double n_eff = (double)(d.n_eig - d.p);
    const double sigma_g2 = f.quad / n_eff;
    const double logl =
        -0.5 * (f.log_det_v + f.log_det_xvx + n_eff * std::log(sigma_g2) + n_eff);
    return -logl;
}

}  // namespace

void eigen_run_null(cs_eigen_vce* v, cs_eigen_vce_result* out) {
    if (!v || !v->d) fail(CS_ERR_INVALID_ARGUMENT, "EigenVce::runNullModel: not prepared");
    const auto start = std::chrono::steady_clock::now();
    DenseNull& d = *v->d;
    const int64_t n = d.n_eig, p = d.p;
    if (n - p <= 0) fail(CS_ERR_INVALID_ARGUMENT, "EigenVce: no residual degrees of freedom");
    const double n_eff = (double)(n - p);
    // golden-section search over log10 delta (vce.cpp:3118-3146)
    double lo = -5.0, hi = 5.0;
    const double gr = (std::sqrt(5.0) + 1.0) / 2.0;
    double c = hi - (hi - lo) / gr, dd = lo + (hi - lo) / gr;
    double fc = neg_reml(d, std::pow(10.0, c)), fd = neg_reml(d, std::pow(10.0, dd));
    const double tol = 1e-5;
    while (std::abs(c - dd) > tol) {
        if (fc < fd) {
            hi = dd;
            dd = c;
            fd = fc;
            c = hi - (hi - lo) / gr;
            fc = neg_reml(d, std::pow(10.0, c));
        } else {
            lo = c;
            c = dd;
            fc = fd;
            dd = lo + (hi - lo) / gr;
            fd = neg_reml(d, std::pow(10.0, dd));
        }
    }
    const double best_delta = std::pow(10.0, (lo + hi) / 2.0);
    const DiagFit f = diag_fit(d, best_delta);
    const double var_g = f.quad / n_eff;
    const double var_e = var_g * best_delta;
    cs_eigen_vce_result& r = v->result;
    r.sigma2_g = var_g;
    r.sigma2_e = var_e;
    r.sigma2_g_se = var_g * std::sqrt(2.0 / n_eff);
    r.sigma2_e_se = var_e * std::sqrt(2.0 / n_eff);
    r.delta = var_e / var_g;
    r.converged = 1;
    r.n_eig = n;
    d.sigma2_g = var_g;
    d.sigma2_e = var_e;
    d.delta = r.delta;
    d.solved = true;
    // updateRemlDiagnostics (eigen_vce.cpp:114-153) with P = V^-1 - V^-1 X I^-1 X^T V^-1
    // applied through its rank-p form
    std::vector<double> inv(n);
    double log_det_cov = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double cv = std::max(var_g * d.D[i] + var_e, 1e-12);
        inv[i] = 1.0 / cv;
        log_det_cov += std::log(cv);
    }
    std::vector<double> info_inv;
    double log_det_fixed = 0.0;
    bool ok = true;
    if (p > 0) {
        std::vector<double> info(p * p, 0.0), L, Dl;
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b) {
                double acc = 0.0;
                for (int64_t i = 0; i < n; ++i) acc += d.UtX[i + a * n] * inv[i] * d.UtX[i + b * n];
                info[a + b * p] = acc;
            }
        ok = la::ldlt(info, (int)p, L, Dl);
        if (ok) {
            info_inv = la::ldlt_inverse(L, Dl, (int)p);
            for (double x : Dl) log_det_fixed += std::log(std::max(std::abs(x), 1e-300));
        }
    }
    if (ok) {
        // P v = inv o v - inv o (UtX (I^-1 (UtX^T (inv o v))))
        auto apply_p = [&](const std::vector<double>& x) {
            std::vector<double> out(n);
            for (int64_t i = 0; i < n; ++i) out[i] = inv[i] * x[i];
            if (p > 0) {
                std::vector<double> t(p, 0.0), u(p, 0.0);
                for (int64_t a = 0; a < p; ++a)
                    for (int64_t i = 0; i < n; ++i) t[a] += d.UtX[i + a * n] * out[i];
                for (int64_t a = 0; a < p; ++a)
                    for (int64_t b = 0; b < p; ++b) u[a] += info_inv[a + b * p] * t[b];
                for (int64_t i = 0; i < n; ++i) {
                    double acc = 0.0;
                    for (int64_t a = 0; a < p; ++a) acc += d.UtX[i + a * n] * u[a];
                    out[i] -= inv[i] * acc;
                }
            }
            return out;
        };
        std::vector<double> pdiag(n);
        for (int64_t i = 0; i < n; ++i) {
            double corr = 0.0;
            for (int64_t a = 0; a < p; ++a)
                for (int64_t b = 0; b < p; ++b)
                    corr += d.UtX[i + a * n] * info_inv[a + b * p] * d.UtX[i + b * n];
            pdiag[i] = inv[i] - inv[i] * inv[i] * corr;
        }
        const std::vector<double> py = apply_p(d.Uty);
        std::vector<double> kpy(n);
        for (int64_t i = 0; i < n; ++i) kpy[i] = d.D[i] * py[i];
        const std::vector<double> pk = apply_p(kpy);
        const std::vector<double> ppy = apply_p(py);
        double s_g = 0.0, tr_pk = 0.0, pp = 0.0, tr_p = 0.0, uy_py = 0.0;
        double a_gg = 0.0, a_ge = 0.0, a_ee = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            s_g += py[i] * kpy[i];
            tr_pk += pdiag[i] * d.D[i];
            pp += py[i] * py[i];
            tr_p += pdiag[i];
            uy_py += d.Uty[i] * py[i];
            a_gg += kpy[i] * pk[i];   // (KPy)^T P (KPy)
            a_ge += kpy[i] * ppy[i];  // (KPy)^T P (Py)
            a_ee += py[i] * ppy[i];   // (Py)^T P (Py)
        }
        const double score_g = 0.5 * (s_g - tr_pk), score_e = 0.5 * (pp - tr_p);
        const double ai_gg = 0.5 * a_gg, ai_ge = 0.5 * a_ge, ai_ee = 0.5 * a_ee;
        const double det = ai_gg * ai_ee - ai_ge * ai_ge;
        if (det > 0.0 && ai_gg > 0.0 && std::isfinite(det)) {
            r.sigma2_g_se = std::sqrt(std::max(0.0, ai_ee / det));
            r.sigma2_e_se = std::sqrt(std::max(0.0, ai_gg / det));
        }
        r.max_score = std::max(std::abs(score_g), std::abs(score_e));
        r.log_likelihood = -0.5 * (log_det_cov + log_det_fixed + uy_py +
                                   (double)(n - p) * std::log(2.0 * 3.14159265358979323846));
    }
    r.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    if (out) *out = r;
}

void eigen_get(const cs_eigen_vce* v, double* D, double* Uty, double* UtX, double* W, int64_t ldw) {
    if (!v || !v->d) fail(CS_ERR_INVALID_ARGUMENT, "EigenVce: not prepared");
    const DenseNull& d = *v->d;
    if (D) std::copy(d.D.begin(), d.D.end(), D);
    if (Uty) std::copy(d.Uty.begin(), d.Uty.end(), Uty);
    if (UtX) std::copy(d.UtX.begin(), d.UtX.end(), UtX);
    if (W) {
        if (ldw < d.n) fail(CS_ERR_INVALID_ARGUMENT, "EigenVce: ldw < n");
        CS_CUDA(cudaMemcpy2D(W, 8 * ldw, d.W.get(), 8 * d.n, 8 * d.n, d.n_eig, cudaMemcpyDeviceToHost));
    }
}

}  // namespace cs
