// FP64 decode-GEMV passes for one to four right-hand sides.
//
// A kinship apply with a single vector is what the reference's MatrixFreePCG issues on every
// CG step (STCG_VCE::apply_G through GenotypeMatrix::multiply_Zt_v / multiply_Z_v,
// libCosmicCore/src/plink_reader.cpp:241-438).  With so few columns the tile GEMMs idle: the
// work is one fused multiply-add per genotype and column, and the packed matrix is read once
// per pass.  Here every thread owns a short run of samples (32 / K of them) and keeps their
// right-hand-side values in registers; a CTA covers 8192 / K consecutive samples and a range
// of SNP rows, and streams the rows' packed bytes (each warp reads 256 contiguous bytes per
// row):
//   rows pass    out[t, c] = sum_i lut_t[code(t,i)] V[i, c]: per row, the thread's partial
//                sum is reduced over the warp (shuffles) and the CTA's warps (shared memory)
//                into one partial per (sample chunk, row);
//   samples pass out[i, c] = sum_t lut_t[code(t,i)] W[t, c]: each thread accumulates its own
//                samples over the CTA's rows; one partial per (row range, sample).
// The partials are summed in a fixed order by a second kernel, so results are bitwise
// repeatable.  Samples past the analysed ones read the rows' missing-code padding (value 0).
#include <cuda_runtime.h>

#include <algorithm>

#include "cs_internal.h"

namespace cs {

namespace {

constexpr int kNThreads = 256, kNWarps = kNThreads / 32;
constexpr int kRowBatch = 32;  // rows pass: rows reduced per shared-memory round

template <int K>
struct Narrow {
    static constexpr int SPL = 32 / K;                 // samples per thread
    static constexpr int CH = kNThreads * SPL;         // samples per CTA
    static constexpr int BYTES = SPL / 4;              // packed bytes per thread per row
};

template <int K>
__device__ __forceinline__ uint64_t load_bits(const uint8_t* p) {
    if constexpr (K == 1) {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
        return (uint64_t)v.x | ((uint64_t)v.y << 32);
    } else if constexpr (K == 2) {
        return (uint64_t)__ldg(reinterpret_cast<const uint32_t*>(p));
    } else {
        return (uint64_t)__ldg(reinterpret_cast<const uint16_t*>(p));
    }
}

__device__ __forceinline__ double pick(uint32_t code, double l0, double l1, double l2, double l3) {
    const double lo = (code & 1u) ? l1 : l0;
    const double hi = (code & 1u) ? l3 : l2;
    return (code & 2u) ? hi : lo;
}

template <int K>
__global__ void __launch_bounds__(kNThreads)
k_narrow_rows(const uint8_t* __restrict__ packed, int64_t n_rows, int64_t n_samples,
              int64_t stride, const double* __restrict__ lut, const double* __restrict__ V,
              int64_t ldv, int64_t k, int64_t rows_per_cta, double* __restrict__ part) {
    using NW = Narrow<K>;
    __shared__ double red[kNWarps][kRowBatch][K];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t chunk = blockIdx.x;
    const int64_t i0 = chunk * NW::CH + (int64_t)tid * NW::SPL;
    const bool in_row = i0 < stride * 4;  // inside the padded packed row
    double v[NW::SPL][K];
#pragma unroll
    for (int j = 0; j < NW::SPL; ++j)
#pragma unroll
        for (int c = 0; c < K; ++c) v[j][c] = (i0 + j < n_samples && c < k) ? __ldg(V + (i0 + j) * ldv + c) : 0.0;
    const int64_t t_begin = (int64_t)blockIdx.y * rows_per_cta;
    const int64_t t_end = min(n_rows, t_begin + rows_per_cta);
    const int64_t n_chunks = gridDim.x;
    for (int64_t tb = t_begin; tb < t_end; tb += kRowBatch) {
        const int nb = (int)min((int64_t)kRowBatch, t_end - tb);
        for (int r = 0; r < nb; ++r) {
            const int64_t t = tb + r;
            const double* L = lut + 4 * t;
            const double l0 = __ldg(L), l1 = __ldg(L + 1), l2 = __ldg(L + 2), l3 = __ldg(L + 3);
            const uint64_t bits = in_row ? load_bits<K>(packed + t * stride + (i0 >> 2)) : ~0ull;
            double acc[K];
#pragma unroll
            for (int c = 0; c < K; ++c) acc[c] = 0.0;
            if (in_row) {
#pragma unroll
                for (int j = 0; j < NW::SPL; ++j) {
                    const double val = pick((uint32_t)(bits >> (2 * j)) & 3u, l0, l1, l2, l3);
#pragma unroll
                    for (int c = 0; c < K; ++c) acc[c] = fma(val, v[j][c], acc[c]);
                }
            }
#pragma unroll
            for (int c = 0; c < K; ++c)
#pragma unroll
                for (int off = 16; off; off >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], off);
            if (lane == 0)
#pragma unroll
                for (int c = 0; c < K; ++c) red[warp][r][c] = acc[c];
        }
        __syncthreads();
        if (tid < nb * K) {
            const int r = tid / K, c = tid - r * K;
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < kNWarps; ++w) s += red[w][r][c];
            part[((tb + r) * n_chunks + chunk) * K + c] = s;
        }
        __syncthreads();
    }
}

template <int K>
__global__ void __launch_bounds__(kNThreads)
k_narrow_samples(const uint8_t* __restrict__ packed, int64_t n_rows, int64_t n_samples,
                 int64_t stride, const double* __restrict__ lut, const double* __restrict__ W,
                 int64_t ldw, int64_t k, int64_t rows_per_cta, double* __restrict__ part) {
    using NW = Narrow<K>;
    const int tid = threadIdx.x;
    const int64_t i0 = (int64_t)blockIdx.x * NW::CH + (int64_t)tid * NW::SPL;
    const bool in_row = i0 < stride * 4;
    double acc[NW::SPL][K];
#pragma unroll
    for (int j = 0; j < NW::SPL; ++j)
#pragma unroll
        for (int c = 0; c < K; ++c) acc[j][c] = 0.0;
    const int64_t t_begin = (int64_t)blockIdx.y * rows_per_cta;
    const int64_t t_end = min(n_rows, t_begin + rows_per_cta);
    if (in_row) {
        for (int64_t t = t_begin; t < t_end; ++t) {
            const double* L = lut + 4 * t;
            const double l0 = __ldg(L), l1 = __ldg(L + 1), l2 = __ldg(L + 2), l3 = __ldg(L + 3);
            double w[K];
#pragma unroll
            for (int c = 0; c < K; ++c) w[c] = c < k ? __ldg(W + t * ldw + c) : 0.0;
            const uint64_t bits = load_bits<K>(packed + t * stride + (i0 >> 2));
#pragma unroll
            for (int j = 0; j < NW::SPL; ++j) {
                const double val = pick((uint32_t)(bits >> (2 * j)) & 3u, l0, l1, l2, l3);
#pragma unroll
                for (int c = 0; c < K; ++c) acc[j][c] = fma(val, w[c], acc[j][c]);
            }
        }
    }
    // part[split][i][c] for the thread's samples that are analysed
    double* dst = part + ((int64_t)blockIdx.y * n_samples) * K;
#pragma unroll
    for (int j = 0; j < NW::SPL; ++j)
        if (i0 + j < n_samples)
#pragma unroll
            for (int c = 0; c < K; ++c) dst[(i0 + j) * K + c] = acc[j][c];
}

// out[r * ldo + c] = scale * sum_q part[...] in q order (rows pass: part[r][q][c]; samples
// pass: part[q][r][c]), c < k.
__global__ void k_narrow_reduce(const double* __restrict__ part, int64_t R, int64_t nq, int K,
                                int64_t k, bool row_major_q, double scale, double* __restrict__ out,
                                int64_t ldo) {
    const int64_t total = R * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        double s = 0.0;
        if (row_major_q)
            for (int64_t q = 0; q < nq; ++q) s += part[(r * nq + q) * K + c];
        else
            for (int64_t q = 0; q < nq; ++q) s += part[(q * R + r) * K + c];
        out[r * ldo + c] = s * scale;
    }
}

template <int K>
void launch_narrow(bool rows_pass, const cs_packed_view& v, const double* lut, const double* in,
                   int64_t ldi, int64_t k, double* out, int64_t ldo, double scale, Workspace& ws,
                   cudaStream_t s) {
    using NW = Narrow<K>;
    const int64_t n = v.n_samples, M = v.n_rows;
    const int64_t chunks = (n + NW::CH - 1) / NW::CH;
    // row ranges so that about four CTAs per SM are in flight, at least 64 rows each
    const int64_t want = std::max<int64_t>(1, (4LL * num_sms() + chunks - 1) / chunks);
    const int64_t rows_per = std::max<int64_t>(64, (M + want - 1) / want);
    const int64_t splits = (M + rows_per - 1) / rows_per;
    const dim3 grid((unsigned)chunks, (unsigned)splits);
    const int64_t R = rows_pass ? M : n;
    const int64_t nq = rows_pass ? chunks : splits;
    ws.partial.resize((size_t)std::max<int64_t>(1, R * nq * K));
    {
        prof::Scope ps(rows_pass ? "decode_gemv_rows_fp64" : "decode_gemv_samples_fp64", s,
                       2.0 * (double)n * (double)M * (double)k, (double)M * (double)((n + 3) / 4));
        if (rows_pass)
            k_narrow_rows<K><<<grid, kNThreads, 0, s>>>(v.rows, M, n, v.stride, lut, in, ldi, k,
                                                        rows_per, ws.partial.get());
        else
            k_narrow_samples<K><<<grid, kNThreads, 0, s>>>(v.rows, M, n, v.stride, lut, in, ldi, k,
                                                           rows_per, ws.partial.get());
        CS_LAUNCH(rows_pass ? "decode_gemv_rows_fp64" : "decode_gemv_samples_fp64");
    }
    {
        prof::Scope ps("gemv_reduce", s, 0.0, 8.0 * (double)(nq + 1) * R * k);
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((R * k + 255) / 256, 32LL * num_sms()));
        k_narrow_reduce<<<blocks, 256, 0, s>>>(ws.partial.get(), R, nq, K, k, rows_pass, scale,
                                               out, ldo);
        CS_LAUNCH("gemv_reduce");
    }
}

}  // namespace

// The narrow form for k <= 4 right-hand sides.
void decode_narrow_fp64(bool rows_pass, const cs_packed_view& v, const double* lut,
                        const double* in, int64_t ldi, int64_t k, double* out, int64_t ldo,
                        double scale, Workspace& ws, cudaStream_t s) {
    if (k <= 0 || v.n_rows == 0) return;
    if (k == 1) launch_narrow<1>(rows_pass, v, lut, in, ldi, k, out, ldo, scale, ws, s);
    else if (k == 2) launch_narrow<2>(rows_pass, v, lut, in, ldi, k, out, ldo, scale, ws, s);
    else if (k <= 4) launch_narrow<4>(rows_pass, v, lut, in, ldi, k, out, ldo, scale, ws, s);
    else fail(CS_ERR_INVALID_ARGUMENT, "narrow decode pass: at most 4 columns");
}

}  // namespace cs
