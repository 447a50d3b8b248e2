// FP64 decode-GEMM passes on the FP64 tensor datapath (DMMA, mma.sync m8n8k4 f64).
//
// The plain (all-FP64) form of the kinship operator computes the same two products as the
// SIMT kernels of kinship_fp64.cu,
//   rows pass    out[t, c] = sum_i lut_t[code(t,i)] B[i, c]   (Z^T V: SNP-major output)
//   samples pass out[i, c] = sum_t lut_t[code(t,i)] B[t, c]   (Z W: sample-major output)
// with the decoded genotype tile in shared memory as the A operand and B staged by cp.async,
// but every warp issues m8n8k4 FP64 MMAs on a 32 x (BN / 4) register tile: 256 FMAs per
// instruction, and one fragment load feeds four MMAs, so shared-memory bandwidth no longer
// bounds the FP64 pipe as it does the register-tiled SIMT form.
//
// Tiles: 64 output rows x BN columns per CTA (8 warps as 2 x 4), 32 contraction steps per
// stage, two stages (B by cp.async with zero fill, the packed bytes of the next stage held in
// registers while the current one computes).  Shared layouts are padded so that fragment
// loads and decode stores are free of bank conflicts:
//   rows pass    A[m][k]  stride 36 doubles (m = SNP row, k = sample)
//   samples pass A[k][m]  stride 72 doubles (k = SNP row, m = sample)
//   B[k][n]               stride BN + 8 doubles
// The contraction may be split over blockIdx.z (fixed-order reduction of the partials by the
// caller), so results are bitwise repeatable.
#include <cuda_runtime.h>

#include <algorithm>

#include "cs_internal.h"

namespace cs {

namespace {

constexpr int kBM = 64, kBK = 32, kThreadsD = 256;
constexpr int kAStrideRows = kBK + 4;     // rows pass: A[m][k]
constexpr int kAStrideSamples = kBM + 8;  // samples pass: A[k][m]
constexpr int kATile = kBM * kAStrideRows > kBK * kAStrideSamples ? kBM * kAStrideRows
                                                                  : kBK * kAStrideSamples;

template <int BN>
struct DmmaSmem {
    static constexpr int kBStride = BN + 8;
    static constexpr int kBTile = kBK * kBStride;
    // two stages of A and B, the rows pass's 64-row lookup table or the samples pass's two
    // stages of 32-row tables
    static constexpr size_t bytes = sizeof(double) * (2 * kATile + 2 * kBTile + 4 * kBM);
};

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    const int size = valid ? 8 : 0;  // zero-fill when out of range
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(src), "r"(size));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// B[kk][n] <- src[(r0 + kk) * ld + c0 + n] (zero outside [r0, r_end) x [c0, k)).
template <int BN>
__device__ __forceinline__ void stage_b(double* __restrict__ Bs, const double* __restrict__ src,
                                        int64_t ld, int64_t r0, int64_t r_end, int64_t c0,
                                        int64_t k, int tid) {
    constexpr int S = DmmaSmem<BN>::kBStride;
#pragma unroll 4
    for (int idx = tid; idx < kBK * BN; idx += kThreadsD) {
        const int kk = idx / BN, n = idx - kk * BN;
        const int64_t r = r0 + kk, c = c0 + n;
        const bool ok = r < r_end && c < k;
        cp_async8(Bs + kk * S + n, ok ? src + r * ld + c : src, ok);
    }
    cp_async_commit();
}

template <bool ROWS, int BN>
__global__ void __launch_bounds__(kThreadsD, 2)
k_dmma_pass(const uint8_t* __restrict__ packed, int64_t n_rows, int64_t n_samples,
            int64_t stride, const double* __restrict__ lut, const double* __restrict__ Bsrc,
            int64_t ldb, int64_t k, double* __restrict__ out, int64_t ldo, int64_t chunk,
            double scale) {
    using S = DmmaSmem<BN>;
    constexpr int NT = BN / 32;  // n8 tiles per warp
    extern __shared__ __align__(16) double smem_d[];
    double* As = smem_d;                     // [2][kATile]
    double* Bs = As + 2 * kATile;            // [2][kBTile]
    double* Ls = Bs + 2 * S::kBTile;         // rows: [64][4]; samples: [2][32][4]

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int64_t R = ROWS ? n_rows : n_samples;  // output rows
    const int64_t K = ROWS ? n_samples : n_rows;  // contraction length
    const int64_t m0 = (int64_t)blockIdx.x * kBM;
    const int64_t c0 = (int64_t)blockIdx.y * BN;
    const int64_t k_begin = (int64_t)blockIdx.z * chunk;
    const int64_t k_end = min(K, k_begin + chunk);

    if (ROWS) {
        for (int idx = tid; idx < 4 * kBM; idx += kThreadsD) {
            const int r = idx >> 2;
            Ls[idx] = (m0 + r < n_rows) ? __ldg(lut + 4 * (m0 + r) + (idx & 3)) : 0.0;
        }
    }

    // decode role: ROWS - SNP row tid / 4, samples 8 (tid % 4) .. + 7 of the stage;
    //              SAMPLES - SNP row tid / 8, samples 8 (tid % 8) .. + 7 of the CTA's 64
    const int d_row = ROWS ? tid >> 2 : tid >> 3;
    const int d_col = ROWS ? 8 * (tid & 3) : 8 * (tid & 7);
    auto fetch = [&](int64_t kk0) -> uint32_t {
        // two packed bytes (8 samples); missing codes outside the matrix
        if (ROWS) {
            const int64_t t = m0 + d_row, i = kk0 + d_col;
            if (t >= n_rows || i >= k_end) return 0x5555u;
            const uint8_t* p = packed + t * stride + (i >> 2);
            return (uint32_t)__ldg(p) | ((uint32_t)__ldg(p + 1) << 8);
        } else {
            const int64_t t = kk0 + d_row, i = m0 + d_col;
            if (t >= k_end || i >= n_samples) return 0x5555u;
            const uint8_t* p = packed + t * stride + (i >> 2);
            return (uint32_t)__ldg(p) | ((uint32_t)__ldg(p + 1) << 8);
        }
    };
    auto decode = [&](uint32_t bytes, double* A, const double* L) {
        double v[8];
        if (ROWS) {
            const double* l = L + 4 * d_row;
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = l[(bytes >> (2 * q)) & 3u];
            double2* dst = reinterpret_cast<double2*>(A + d_row * kAStrideRows + d_col);
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[q] = make_double2(v[2 * q], v[2 * q + 1]);
        } else {
            const double* l = L + 4 * d_row;
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = l[(bytes >> (2 * q)) & 3u];
            double2* dst = reinterpret_cast<double2*>(A + d_row * kAStrideSamples + d_col);
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[q] = make_double2(v[2 * q], v[2 * q + 1]);
        }
    };
    // samples pass: the lookup table of the stage's 32 SNP rows
    auto stage_lut = [&](int64_t kk0, double* L) {
        if (!ROWS && tid < 4 * kBK) {
            const int64_t t = kk0 + (tid >> 2);
            L[tid] = t < k_end ? __ldg(lut + 4 * t + (tid & 3)) : 0.0;
        }
    };

    double acc[4][NT][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    const int n_steps = (int)((k_end - k_begin + kBK - 1) / kBK);
    // prologue: stage 0
    uint32_t bytes = n_steps > 0 ? fetch(k_begin) : 0x5555u;
    if (n_steps > 0) {
        stage_b<BN>(Bs, Bsrc, ldb, k_begin, k_end, c0, k, tid);
        stage_lut(k_begin, Ls);
    }
    __syncthreads();  // Ls (rows pass) and the stage-0 table ready
    if (n_steps > 0) decode(bytes, As, ROWS ? Ls : Ls);

    const int gid = lane >> 2, tig = lane & 3;
    for (int st = 0; st < n_steps; ++st) {
        const int cur = st & 1, nxt = cur ^ 1;
        const int64_t kk0 = k_begin + (int64_t)st * kBK;
        const bool more = st + 1 < n_steps;
        if (more) {
            bytes = fetch(kk0 + kBK);
            stage_lut(kk0 + kBK, Ls + (ROWS ? 0 : nxt * 4 * kBK));
        }
        cp_async_wait_all();
        __syncthreads();  // stage cur: A decoded, B landed; the other stage's buffers free
        if (more) stage_b<BN>(Bs + nxt * S::kBTile, Bsrc, ldb, kk0 + kBK, k_end, c0, k, tid);
        const double* A = As + cur * kATile;
        const double* B = Bs + cur * S::kBTile;
#pragma unroll
        for (int ks = 0; ks < kBK / 4; ++ks) {
            double a[4], b[NT];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int m = wm * 32 + i * 8 + gid, kk = ks * 4 + tig;
                a[i] = ROWS ? A[m * kAStrideRows + kk] : A[kk * kAStrideSamples + m];
            }
#pragma unroll
            for (int j = 0; j < NT; ++j)
                b[j] = B[(ks * 4 + tig) * S::kBStride + wn * (BN / 4) + j * 8 + gid];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < NT; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        if (more) {
            __syncthreads();  // the table of the next stage written before its decode reads it
            decode(bytes, As + nxt * kATile, ROWS ? Ls : Ls + nxt * 4 * kBK);
        }
    }

    double* dst = out + (int64_t)blockIdx.z * R * ldo;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t r = m0 + wm * 32 + i * 8 + gid;
        if (r >= R) continue;
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const int64_t c = c0 + wn * (BN / 4) + j * 8 + 2 * tig;
            if (c < k) dst[r * ldo + c] = acc[i][j][0] * scale;
            if (c + 1 < k) dst[r * ldo + c + 1] = acc[i][j][1] * scale;
        }
    }
}

__global__ void k_reduce_splits_d(const double* __restrict__ part, int splits, int64_t R,
                                  int64_t k, double* __restrict__ dst, int64_t ldo, double scale) {
    const int64_t total = R * k;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = idx / k, c = idx - r * k;
        double acc = 0.0;
        for (int z = 0; z < splits; ++z) acc += part[((int64_t)z * R + r) * k + c];
        dst[r * ldo + c] = acc * scale;
    }
}

template <bool ROWS, int BN>
void launch_dmma(const cs_packed_view& v, const double* lut, const double* in, int64_t ldi,
                 int64_t k, double* out, int64_t ldo, double scale, Workspace& ws, cudaStream_t s,
                 int64_t max_splits) {
    using S = DmmaSmem<BN>;
    auto kern = k_dmma_pass<ROWS, BN>;
    static PerDeviceOnce configured;
    once_per_device(configured, [&] {
        return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
    }, "configure FP64 tensor decode-GEMM kernel");
    const int64_t R = ROWS ? v.n_rows : v.n_samples;
    const int64_t K = ROWS ? v.n_samples : v.n_rows;
    const int64_t gx = (R + kBM - 1) / kBM, gy = (k + BN - 1) / BN;
    // split the contraction only while the grid covers the GPU less than about twice
    const int64_t target = 4LL * num_sms();
    int64_t splits = std::max<int64_t>(1, std::min<int64_t>((target + gx * gy - 1) / (gx * gy),
                                                            (K + 511) / 512));
    splits = std::min<int64_t>(splits, max_splits);
    int64_t chunk = round_up((K + splits - 1) / splits, ROWS ? 8 * kBK : kBK);
    chunk = std::max<int64_t>(chunk, kBK);
    splits = std::max<int64_t>(1, (K + chunk - 1) / chunk);
    double* dst = out;
    int64_t ldd = ldo;
    double kscale = scale;
    if (splits > 1) {
        ws.partial.resize((size_t)splits * R * k);
        dst = ws.partial.get();
        ldd = k;
        kscale = 1.0;
    }
    {
        prof::Scope ps(ROWS ? "decode_dmma_rows_fp64" : "decode_dmma_samples_fp64", s,
                       2.0 * (double)R * (double)K * (double)k,
                       (double)v.n_rows * (double)((v.n_samples + 3) / 4));
        kern<<<dim3((unsigned)gx, (unsigned)gy, (unsigned)splits), kThreadsD, S::bytes, s>>>(
            v.rows, v.n_rows, v.n_samples, v.stride, lut, in, ldi, k, dst, ldd, chunk, kscale);
        CS_LAUNCH(ROWS ? "decode_dmma_rows_fp64" : "decode_dmma_samples_fp64");
    }
    if (splits > 1) {
        const int64_t total = R * k;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 32LL * num_sms());
        prof::Scope ps("reduce_splits", s, 0.0, 8.0 * (double)(splits + 1) * total);
        k_reduce_splits_d<<<std::max(blocks, 1), 256, 0, s>>>(ws.partial.get(), (int)splits, R, k,
                                                              out, ldo, scale);
        CS_LAUNCH("reduce_splits");
    }
}

}  // namespace

// The FP64 tensor form for k right-hand sides (column tiles of 32, 64 or 128).
void decode_dmma_fp64(bool rows_pass, const cs_packed_view& v, const double* lut, const double* in,
                      int64_t ldi, int64_t k, double* out, int64_t ldo, double scale,
                      Workspace& ws, cudaStream_t s, int64_t max_splits) {
    if (k <= 0) return;
    if (k > 128 && k % 128 != 0) {
        // whole 128-column tiles, then the remainder in a narrower tile (k = 266: 2 x 128 + 32
        // instead of 3 x 128, a third less padding)
        const int64_t full = k / 128 * 128;
        decode_dmma_fp64(rows_pass, v, lut, in, ldi, full, out, ldo, scale, ws, s, max_splits);
        decode_dmma_fp64(rows_pass, v, lut, in + full, ldi, k - full, out + full, ldo, scale, ws,
                         s, max_splits);
        return;
    }
    if (rows_pass) {
        if (k <= 32) launch_dmma<true, 32>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
        else if (k <= 64) launch_dmma<true, 64>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
        else launch_dmma<true, 128>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
    } else {
        if (k <= 32) launch_dmma<false, 32>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
        else if (k <= 64) launch_dmma<false, 64>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
        else launch_dmma<false, 128>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
    }
}

}  // namespace cs
