// FP64 decode-GEMM kernels: the plain (all-FP64) form of the kinship operator and of the
// scan's basis projection.
//
// The packed 2-bit genotypes are expanded inside the kernel through a per-row lookup
// table lut_t[code] (e.g. {(2-mu)s, 0, (1-mu)s, -mu s} for Z, exactly the values
// src/kinship_operator.cpp:276-283 decodes), so a decoded matrix never touches HBM:
//
//   rows pass    out[t, c] = sum_i lut_t[code(t,i)] V[i, c]   (Z^T V: SNP-major output)
//   samples pass out[i, c] = sum_t lut_t[code(t,i)] W[t, c]   (Z W: sample-major output)
//
// Each CTA owns a BM x BN output tile and a slice of the contraction; slices write
// partial tiles that a second kernel sums in a fixed order, so results are bitwise
// repeatable (src/kinship_operator.cpp:196-208 keeps the same guarantee with per-worker
// buffers reduced in worker order).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "cs_internal.h"

namespace cs {

void decode_dmma_fp64(bool rows_pass, const cs_packed_view& v, const double* lut, const double* in,
                      int64_t ldi, int64_t k, double* out, int64_t ldo, double scale,
                      Workspace& ws, cudaStream_t s, int64_t max_splits);
void decode_narrow_fp64(bool rows_pass, const cs_packed_view& v, const double* lut,
                        const double* in, int64_t ldi, int64_t k, double* out, int64_t ldo,
                        double scale, Workspace& ws, cudaStream_t s);

namespace {

constexpr int kThreads = 256;
constexpr int kTileElems = 2048;  // SUBK * BM: decoded tile of 16 KB

template <int BM, int BN, int TM, int TN>
struct Cfg {
    static constexpr int SUBK = kTileElems / BM;
    static_assert((BM / TM) * (BN / TN) == kThreads, "thread layout");
    static constexpr size_t smem_a = sizeof(double) * SUBK * BM;
    static constexpr size_t smem_b = sizeof(double) * SUBK * BN;
    static constexpr size_t smem_p = (size_t)BM * 32 + sizeof(double) * 4 * BM;  // rows pass:
                                       // 128-sample packed window + per-row lookup table
};


// Column owned by thread tx for its j-th output: pairs of adjacent columns, strided by
// 2*TX between pairs, so that a warp's 16-byte shared-memory reads of a B row are
// contiguous (conflict-free) and the A row reads are broadcasts.
template <int BN, int TN>
__device__ __forceinline__ int tile_col(int tx, int j) {
    constexpr int TX = BN / TN;
    if constexpr (TN == 1) return tx;
    else return 2 * tx + 2 * TX * (j >> 1) + (j & 1);
}

// SUBK-step rank-1 updates of the TM x TN register tile from As[SUBK][BM], Bs[SUBK][BN].
template <int BM, int BN, int TM, int TN, int SUBK>
__device__ __forceinline__ void tile_fma(const double* __restrict__ As,
                                         const double* __restrict__ Bs, int tx, int ty,
                                         double (&acc)[TM][TN]) {
    constexpr int TX = BN / TN;
#pragma unroll 4
    for (int kk = 0; kk < SUBK; ++kk) {
        double a[TM], b[TN];
        const double* ap = As + kk * BM + ty * TM;
        if constexpr (TM % 2 == 0) {
#pragma unroll
            for (int i = 0; i < TM / 2; ++i) {
                const double2 v = reinterpret_cast<const double2*>(ap)[i];
                a[2 * i] = v.x;
                a[2 * i + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = ap[i];
        }
        const double* bp = Bs + kk * BN;
        if constexpr (TN % 2 == 0) {
#pragma unroll
            for (int q = 0; q < TN / 2; ++q) {
                const double2 v = *reinterpret_cast<const double2*>(bp + 2 * tx + 2 * TX * q);
                b[2 * q] = v.x;
                b[2 * q + 1] = v.y;
            }
        } else {
            b[0] = bp[tx];
        }
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
}

// Bs[kk][n] = src[(r0 + kk) * ld + c0 + n] for rows r0 + kk < r_end and columns < k, else 0.
template <int BN, int SUBK>
__device__ __forceinline__ void load_b_tile(double* __restrict__ Bs, const double* __restrict__ src,
                                            int64_t ld, int64_t r0, int64_t r_end, int64_t c0,
                                            int64_t k, int tid) {
    if (BN >= 2 && (ld & 1) == 0 && ((reinterpret_cast<uintptr_t>(src) & 15) == 0)) {
        for (int idx = tid; idx < SUBK * BN / 2; idx += kThreads) {
            const int kk = idx / (BN / 2), n = 2 * (idx % (BN / 2));
            const int64_t r = r0 + kk, c = c0 + n;
            double2 v = make_double2(0.0, 0.0);
            if (r < r_end) {
                if (c + 1 < k) v = __ldg(reinterpret_cast<const double2*>(src + r * ld + c));
                else if (c < k) v.x = __ldg(src + r * ld + c);
            }
            *reinterpret_cast<double2*>(Bs + kk * BN + n) = v;
        }
    } else {
        for (int idx = tid; idx < SUBK * BN; idx += kThreads) {
            const int kk = idx / BN, n = idx % BN;
            const int64_t r = r0 + kk, c = c0 + n;
            Bs[idx] = (r < r_end && c < k) ? __ldg(src + r * ld + c) : 0.0;
        }
    }
}

// ---------------------------------------------------------------- rows pass (Z^T V)
template <int BM, int BN, int TM, int TN>
__global__ void __launch_bounds__(kThreads, 2)
k_rows_fp64(const uint8_t* __restrict__ packed, int64_t n_rows, int64_t n_samples, int64_t stride,
            const double* __restrict__ lut, const double* __restrict__ V, int64_t ldv, int64_t k,
            double* __restrict__ out, int64_t ldo, int64_t chunk, double scale) {
    using C = Cfg<BM, BN, TM, TN>;
    constexpr int SUBK = C::SUBK;
    extern __shared__ __align__(16) unsigned char smem[];
    double* As = reinterpret_cast<double*>(smem);                 // [SUBK][BM]
    double* Bs = As + SUBK * BM;                                   // [SUBK][BN]
    double* Ls = Bs + SUBK * BN;                                   // [4][BM] lookup table
    uint8_t* Ps = reinterpret_cast<uint8_t*>(Ls + 4 * BM);         // [BM][32]

    const int tid = threadIdx.x;
    const int tx = tid % (BN / TN), ty = tid / (BN / TN);
    const int64_t row0 = (int64_t)blockIdx.x * BM;
    const int64_t col0 = (int64_t)blockIdx.y * BN;
    const int64_t s_begin = (int64_t)blockIdx.z * chunk;
    const int64_t s_end = std::min<int64_t>(n_samples, s_begin + chunk);

    // decode role: row dm, two bytes starting at byte db of each SUBK-sample step
    const int dm = tid % BM;
    const int db = (tid / BM) * 2;
    for (int idx = tid; idx < 4 * BM; idx += kThreads) {
        const int r = idx >> 2, code = idx & 3;
        Ls[code * BM + r] = (row0 + r < n_rows) ? __ldg(lut + 4 * (row0 + r) + code) : 0.0;
    }

    double acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = 0.0;

    for (int64_t w0 = s_begin; w0 < s_end; w0 += 128) {
        __syncthreads();
        for (int idx = tid; idx < BM * 2; idx += kThreads) {
            const int r = idx >> 1, half = idx & 1;
            uint4 v = make_uint4(0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u);
            if (row0 + r < n_rows)
                v = __ldg(reinterpret_cast<const uint4*>(packed + (row0 + r) * stride + (w0 >> 2)) + half);
            *reinterpret_cast<uint4*>(Ps + r * 32 + half * 16) = v;
        }
        __syncthreads();
        for (int sub = 0; sub < 128 / SUBK; ++sub) {
            const int64_t s0 = w0 + (int64_t)sub * SUBK;
            if (s0 >= s_end) break;
            // decode 8 samples of row dm
            {
                const int byte_base = sub * (SUBK / 4) + db;
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const uint32_t b = Ps[dm * 32 + byte_base + j];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const uint32_t code = (b >> (2 * q)) & 3u;
                        As[(4 * (db + j) + q) * BM + dm] = Ls[code * BM + dm];
                    }
                }
            }
            load_b_tile<BN, SUBK>(Bs, V, ldv, s0, s_end, col0, k, tid);
            __syncthreads();
            tile_fma<BM, BN, TM, TN, SUBK>(As, Bs, tx, ty, acc);
            __syncthreads();
        }
    }
    double* dst = out + (int64_t)blockIdx.z * n_rows * ldo;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int64_t t = row0 + ty * TM + i;
        if (t >= n_rows) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int64_t c = col0 + tile_col<BN, TN>(tx, j);
            if (c < k) dst[t * ldo + c] = acc[i][j] * scale;
        }
    }
}

// ---------------------------------------------------------------- samples pass (Z W)
template <int BM, int BN, int TM, int TN>
__global__ void __launch_bounds__(kThreads, 2)
k_samples_fp64(const uint8_t* __restrict__ packed, int64_t n_rows, int64_t n_samples,
               int64_t stride, const double* __restrict__ lut, const double* __restrict__ W,
               int64_t ldw, int64_t k, double* __restrict__ out, int64_t ldo, int64_t chunk,
               double scale) {
    using C = Cfg<BM, BN, TM, TN>;
    constexpr int SUBK = C::SUBK;  // rows per step
    constexpr int BYTES = BM / 4;  // packed bytes of one row inside the tile
    extern __shared__ __align__(16) unsigned char smem[];
    double* As = reinterpret_cast<double*>(smem);  // [SUBK][BM]
    double* Bs = As + SUBK * BM;                   // [SUBK][BN]

    const int tid = threadIdx.x;
    const int tx = tid % (BN / TN), ty = tid / (BN / TN);
    const int64_t smp0 = (int64_t)blockIdx.x * BM;
    const int64_t col0 = (int64_t)blockIdx.y * BN;
    const int64_t t_begin = (int64_t)blockIdx.z * chunk;
    const int64_t t_end = std::min<int64_t>(n_rows, t_begin + chunk);

    // decode role: 2 bytes per thread; SUBK * BYTES == 2 * kThreads
    const int bidx = tid * 2;
    const int dk = bidx / BYTES;       // row within the step
    const int dbyte = bidx % BYTES;    // byte within the tile row

    double acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = 0.0;

    for (int64_t t0 = t_begin; t0 < t_end; t0 += SUBK) {
        {
            const int64_t t = t0 + dk;
            double l0 = 0.0, l1 = 0.0, l2 = 0.0, l3 = 0.0;
            uint32_t bytes = 0x5555u;
            if (t < t_end) {
                const double* L = lut + 4 * t;
                l0 = __ldg(L); l1 = __ldg(L + 1); l2 = __ldg(L + 2); l3 = __ldg(L + 3);
                const uint8_t* p = packed + t * stride + (smp0 >> 2) + dbyte;
                bytes = (uint32_t)__ldg(p) | ((uint32_t)__ldg(p + 1) << 8);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t code = (bytes >> (2 * q)) & 3u;
                As[dk * BM + 4 * dbyte + q] =
                    code == 0 ? l0 : code == 1 ? l1 : code == 2 ? l2 : l3;
            }
        }
        load_b_tile<BN, SUBK>(Bs, W, ldw, t0, t_end, col0, k, tid);
        __syncthreads();
        tile_fma<BM, BN, TM, TN, SUBK>(As, Bs, tx, ty, acc);
        __syncthreads();
    }
    double* dst = out + (int64_t)blockIdx.z * n_samples * ldo;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int64_t s = smp0 + ty * TM + i;
        if (s >= n_samples) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int64_t c = col0 + tile_col<BN, TN>(tx, j);
            if (c < k) dst[s * ldo + c] = acc[i][j] * scale;
        }
    }
}

// Fixed-order sum of split partials: dst[r, c] = scale * sum_z part[z][r][c].
__global__ void k_reduce_splits(const double* __restrict__ part, int splits, int64_t R,
                                int64_t ldp, int64_t k, double* __restrict__ dst, int64_t ldo,
                                double scale) {
    const int64_t total = R * k;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = idx / k, c = idx - r * k;
        double acc = 0.0;
        for (int z = 0; z < splits; ++z) acc += part[((int64_t)z * R + r) * ldp + c];
        dst[r * ldo + c] = acc * scale;
    }
}

template <int BM, int BN, int TM, int TN, bool ROWS>
void launch_cfg(const cs_packed_view& v, const double* lut, const double* in, int64_t ldi,
                int64_t k, double* out, int64_t ldo, double scale, Workspace& ws, cudaStream_t s,
                int64_t max_splits) {
    using C = Cfg<BM, BN, TM, TN>;
    const size_t smem = C::smem_a + C::smem_b + (ROWS ? C::smem_p : 0);
    auto kern = ROWS ? k_rows_fp64<BM, BN, TM, TN> : k_samples_fp64<BM, BN, TM, TN>;
    static PerDeviceOnce configured;
    once_per_device(configured, [&] {
        return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }, "configure FP64 decode-GEMM kernel");
    const int64_t R = ROWS ? v.n_rows : v.n_samples;   // output rows
    const int64_t K = ROWS ? v.n_samples : v.n_rows;   // contraction length
    const int64_t gx = (R + BM - 1) / BM, gy = (k + BN - 1) / BN;
    // split the contraction so that the grid covers the GPU about twice
    const int64_t unit = ROWS ? 1024 : 256;            // minimum slice (multiple of 128 / SUBK)
    const int64_t target = 4LL * num_sms();
    int64_t splits = std::max<int64_t>(1, std::min<int64_t>((target + gx * gy - 1) / (gx * gy),
                                                            (K + unit - 1) / unit));
    splits = std::min<int64_t>(splits, max_splits);
    int64_t chunk = (K + splits - 1) / splits;
    chunk = round_up(std::max<int64_t>(chunk, 1), ROWS ? 128 : C::SUBK);
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
    dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)splits);
    {
        // algorithmic work: 2 R K k flops, one pass over the packed rows
        prof::Scope ps(ROWS ? "decode_gemm_rows_fp64" : "decode_gemm_samples_fp64", s,
                       2.0 * (double)R * (double)K * (double)k,
                       (double)v.n_rows * (double)((v.n_samples + 3) / 4));
        kern<<<grid, kThreads, smem, s>>>(v.rows, v.n_rows, v.n_samples, v.stride, lut, in, ldi,
                                          k, dst, ldd, chunk, kscale);
        CS_LAUNCH(ROWS ? "decode_gemm_rows_fp64" : "decode_gemm_samples_fp64");
    }
    if (splits > 1) {
        const int64_t total = R * k;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 32LL * num_sms());
        prof::Scope ps("reduce_splits", s, 0.0, 8.0 * (double)(splits + 1) * total);
        k_reduce_splits<<<std::max(blocks, 1), 256, 0, s>>>(ws.partial.get(), (int)splits, R, k,
                                                            k, out, ldo, scale);
        CS_LAUNCH("reduce_splits");
    }
}

// The FP64 tensor (DMMA) form for 8 or more right-hand sides (CS_B200_FP64_DMMA=0 keeps the
// SIMT form everywhere, =1 uses DMMA from one column on).
int64_t dmma_min_columns() {
    static const int64_t v = [] {
        const char* e = std::getenv("CS_B200_FP64_DMMA");
        if (e && e[0] == '0') return (int64_t)1 << 40;
        if (e && e[0] == '1') return (int64_t)1;
        return (int64_t)8;
    }();
    return v;
}

// The decode-GEMV form for up to 4 right-hand sides (CS_B200_FP64_NARROW=0 keeps the tile
// kernels).  It needs a partials workspace, so the single-slice (workspace-free) callers keep
// the tile kernels.
bool narrow_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("CS_B200_FP64_NARROW");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <bool ROWS>
void dispatch(const cs_packed_view& v, const double* lut, const double* in, int64_t ldi,
              int64_t k, double* out, int64_t ldo, double scale, Workspace& ws, cudaStream_t s,
              int64_t max_splits = 64) {
    if (k <= 0) return;
    if (k <= 4 && max_splits > 1 && narrow_enabled()) {
        decode_narrow_fp64(ROWS, v, lut, in, ldi, k, out, ldo, scale, ws, s);
        return;
    }
    if (k >= dmma_min_columns()) {
        decode_dmma_fp64(ROWS, v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
        return;
    }
    if (k == 1)
        launch_cfg<256, 1, 1, 1, ROWS>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
    else if (k <= 8)
        launch_cfg<128, 8, 4, 1, ROWS>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
    else if (k <= 32)
        launch_cfg<64, 32, 4, 2, ROWS>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
    else if (k <= 64)
        launch_cfg<64, 64, 4, 4, ROWS>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
    else
        launch_cfg<64, 128, 4, 8, ROWS>(v, lut, in, ldi, k, out, ldo, scale, ws, s, max_splits);
}

}  // namespace

void decode_gemm_rows_fp64(const cs_packed_view& v, const double* d_lut, const double* V,
                           int64_t ldv, int64_t k, double* out, int64_t ldo, Workspace& ws,
                           cudaStream_t s) {
    dispatch<true>(v, d_lut, V, ldv, k, out, ldo, 1.0, ws, s);
}

void decode_gemm_samples_fp64(const cs_packed_view& v, const double* d_lut, const double* W,
                              int64_t ldw, int64_t k, double* out, int64_t ldo, double scale,
                              Workspace& ws, cudaStream_t s) {
    dispatch<false>(v, d_lut, W, ldw, k, out, ldo, scale, ws, s);
}

// Single-slice forms: each CTA covers the whole contraction, so no partial tiles and no
// workspace are needed (used where the caller cannot allocate).
void decode_gemm_rows_fp64_unsplit(const cs_packed_view& v, const double* d_lut, const double* V,
                                   int64_t ldv, int64_t k, double* out, int64_t ldo,
                                   cudaStream_t s) {
    Workspace unused;
    dispatch<true>(v, d_lut, V, ldv, k, out, ldo, 1.0, unused, s, 1);
}

void decode_gemm_samples_fp64_unsplit(const cs_packed_view& v, const double* d_lut,
                                      const double* W, int64_t ldw, int64_t k, double* out,
                                      int64_t ldo, double scale, cudaStream_t s) {
    Workspace unused;
    dispatch<false>(v, d_lut, W, ldw, k, out, ldo, scale, unused, s, 1);
}

}  // namespace cs
