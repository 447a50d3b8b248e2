// The reference's Gaussian test matrix on the device.
//
// src/lmm_engine.cpp:917-922 draws Omega column by column from
// std::normal_distribution<double> over std::mt19937_64(seed).  This file reproduces that
// stream on the GPU:
//  1. The 64-bit Mersenne Twister (the engine the C++ standard specifies as mt19937_64:
//     n = 312, m = 156, r = 31, a = 0xB5026F5AA96619E9, tempering (29, d), (17, b), (37, c),
//     43, seeding multiplier 6364136223846793005) is the linear recurrence
//     x[k] = x[k - 156] ^ twist(x[k - 312], x[k - 311]), so 156 consecutive words depend only
//     on earlier words: one CTA advances the stream 156 words per step.
//  2. Marsaglia's polar method as libstdc++ implements it: uniforms u = double(raw) / 2^64
//     (clamped below 1), x = 2u - 1, y = 2u' - 1 from consecutive draws, an attempt is
//     accepted when r2 = x^2 + y^2 is in (0, 1]; accepted attempts are compacted in order.
//  3. mult = sqrt(-2 log(r2) / r2); the pair yields y * mult, then x * mult.
// Uniforms and acceptance are bit-exact; the normals can differ from the host library's in
// the last bit where the device log differs from the host's by an ulp.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "cs_internal.h"

namespace cs {

namespace {

constexpr int kMtN = 312, kMtM = 156, kRing = 468;
constexpr uint64_t kMatA = 0xB5026F5AA96619E9ull;
constexpr uint64_t kUpper = 0xFFFFFFFF80000000ull, kLower = 0x7FFFFFFFull;

__device__ __forceinline__ uint64_t temper(uint64_t y) {
    y ^= (y >> 29) & 0x5555555555555555ull;
    y ^= (y << 17) & 0x71D67FFFEDA60000ull;
    y ^= (y << 37) & 0xFFF7EEE000000000ull;
    y ^= y >> 43;
    return y;
}

// One CTA of 156 threads: continues the sequence from the 312 words in `state`
// (x[K-312 .. K-1]), writes n_out tempered outputs x[K ..], then the new last 312 words.
__global__ void __launch_bounds__(kMtM, 1)
k_mt64(uint64_t* __restrict__ state, int64_t n_out, uint64_t* __restrict__ out) {
    __shared__ uint64_t ring[kRing];
    const int tid = threadIdx.x;
    for (int i = tid; i < kMtN; i += kMtM) ring[i] = state[i];
    __syncthreads();
    // local index L = global index - (K - 312); ring slot = L mod 468
    int a = 0, b = 1, c = kMtM, w = kMtN;  // slots of L-312, L-311, L-156, L for L = 312 + tid
    a += tid; b += tid; c += tid; w += tid;
    a %= kRing; b %= kRing; c %= kRing; w %= kRing;
    for (int64_t base = 0; base < n_out; base += kMtM) {
        const uint64_t y = (ring[a] & kUpper) | (ring[b] & kLower);
        const uint64_t v = ring[c] ^ (y >> 1) ^ ((y & 1ull) ? kMatA : 0ull);
        ring[w] = v;  // slot of L - 468: no thread reads it in this step
        if (base + tid < n_out) out[base + tid] = temper(v);
        __syncthreads();
        a += kMtM; b += kMtM; c += kMtM; w += kMtM;
        if (a >= kRing) a -= kRing;
        if (b >= kRing) b -= kRing;
        if (c >= kRing) c -= kRing;
        if (w >= kRing) w -= kRing;
    }
    // last 312 words in order: local indices steps*156 .. steps*156 + 311
    const int64_t steps = (n_out + kMtM - 1) / kMtM;
    const int start = (int)((steps * kMtM) % kRing);
    for (int i = tid; i < kMtN; i += kMtM) state[i] = ring[(start + i) % kRing];
}

__device__ __forceinline__ double canonical(uint64_t r) {
    double u = __dmul_rn(__ull2double_rn(r), 5.421010862427522170037264e-20);  // 2^-64
    if (u >= 1.0) u = 0.99999999999999988898;  // nextafter(1, 0)
    return u;
}

// attempt a uses draws 2a, 2a+1
__device__ __forceinline__ bool attempt(const uint64_t* raw, int64_t a, double& x, double& y) {
    x = __dsub_rn(__dmul_rn(2.0, canonical(raw[2 * a])), 1.0);
    y = __dsub_rn(__dmul_rn(2.0, canonical(raw[2 * a + 1])), 1.0);
    const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    return !(r2 > 1.0 || r2 == 0.0);
}

constexpr int kAttemptsPerBlock = 1024;

__global__ void k_accept_count(const uint64_t* __restrict__ raw, int64_t attempts,
                               int32_t* __restrict__ counts) {
    __shared__ int warp_sums[8];
    int c = 0;
    const int64_t a0 = (int64_t)blockIdx.x * kAttemptsPerBlock;
    for (int q = 0; q < kAttemptsPerBlock / 256; ++q) {
        const int64_t a = a0 + q * 256 + threadIdx.x;
        double x, y;
        if (a < attempts && attempt(raw, a, x, y)) ++c;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int i = 0; i < 8; ++i) s += warp_sums[i];
        counts[blockIdx.x] = s;
    }
}

// Writes accepted attempts in order: pairs[2 * idx] = x, pairs[2 * idx + 1] = y.
__global__ void k_accept_write(const uint64_t* __restrict__ raw, int64_t attempts,
                               const int64_t* __restrict__ offsets, int64_t max_pairs,
                               double* __restrict__ pairs) {
    __shared__ int warp_sums[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t running = offsets[blockIdx.x];
    const int64_t a0 = (int64_t)blockIdx.x * kAttemptsPerBlock;
    for (int q = 0; q < kAttemptsPerBlock / 256; ++q) {
        const int64_t a = a0 + q * 256 + threadIdx.x;
        double x = 0, y = 0;
        const bool ok = a < attempts && attempt(raw, a, x, y);
        const uint32_t ballot = __ballot_sync(0xffffffffu, ok);
        if (lane == 0) warp_sums[warp] = __popc(ballot);
        __syncthreads();
        int before = 0, total = 0;
        for (int i = 0; i < 8; ++i) {
            if (i < warp) before += warp_sums[i];
            total += warp_sums[i];
        }
        const int64_t idx = running + before + __popc(ballot & ((1u << lane) - 1u));
        if (ok && idx < max_pairs) {
            pairs[2 * idx] = x;
            pairs[2 * idx + 1] = y;
        }
        running += total;
        __syncthreads();
    }
}

// draw idx of the column-by-column stream -> out[row * ld + col], row = idx % n, col = idx / n
__global__ void k_polar(const double* __restrict__ pairs, int64_t count, int64_t n, int64_t ld,
                        double* __restrict__ out) {
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = idx >> 1;
        const double x = pairs[2 * p], y = pairs[2 * p + 1];
        const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
        const double mult = sqrt(__ddiv_rn(__dmul_rn(-2.0, log(r2)), r2));
        const double v = (idx & 1) ? __dmul_rn(x, mult) : __dmul_rn(y, mult);
        const int64_t col = idx / n, row = idx - col * n;
        out[row * ld + col] = v;
    }
}

}  // namespace

// Omega (n x cols, written row-major with leading dimension ld) on the device.
void generate_omega_device(uint64_t seed, int64_t n, int64_t cols, double* d_out, int64_t ld,
                           OmegaWorkspace& ws, cudaStream_t s) {
    const int64_t count = n * cols;
    if (count == 0) return;
    const int64_t pairs = (count + 1) / 2;
    // seeded state (mt19937_64 seeding recurrence)
    std::vector<uint64_t> st(kMtN);
    st[0] = seed;
    for (int i = 1; i < kMtN; ++i)
        st[i] = 6364136223846793005ull * (st[i - 1] ^ (st[i - 1] >> 62)) + (uint64_t)i;
    ws.state.resize(kMtN);
    CS_CUDA(cudaMemcpyAsync(ws.state.get(), st.data(), 8 * kMtN, cudaMemcpyHostToDevice, s));
    ws.pairs.resize(2 * pairs);
    int64_t have = 0;
    // acceptance is pi/4 per attempt: draw for 1.3x the needed attempts, then top up
    int64_t want_attempts = (int64_t)(pairs * 1.3) + 8192;
    while (have < pairs) {
        // an even number of draws that is a multiple of 156 keeps the stream contiguous
        // across top-ups (each call advances the engine by exactly its outputs)
        const int64_t attempts = round_up(want_attempts, kMtM / 2);
        const int64_t blocks = (attempts + kAttemptsPerBlock - 1) / kAttemptsPerBlock;
        ws.raw.resize(2 * attempts);
        ws.counts.resize(blocks);
        ws.offsets.resize(blocks);
        {
            prof::Scope ps("mt19937_64_stream", s, 0.0, 16.0 * attempts);
            k_mt64<<<1, kMtM, 0, s>>>(ws.state.get(), 2 * attempts, ws.raw.get());
            CS_LAUNCH("mt19937_64_stream");
        }
        {
            prof::Scope ps("polar_accept_count", s, 0.0, 16.0 * attempts);
            k_accept_count<<<(unsigned)blocks, 256, 0, s>>>(ws.raw.get(), attempts, ws.counts.get());
            CS_LAUNCH("polar_accept_count");
        }
        std::vector<int32_t> c(blocks);
        CS_CUDA(cudaMemcpyAsync(c.data(), ws.counts.get(), 4 * blocks, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaStreamSynchronize(s));
        std::vector<int64_t> off(blocks);
        int64_t run = have;
        for (int64_t b = 0; b < blocks; ++b) {
            off[b] = run;
            run += c[b];
        }
        CS_CUDA(cudaMemcpyAsync(ws.offsets.get(), off.data(), 8 * blocks, cudaMemcpyHostToDevice, s));
        {
            prof::Scope ps("polar_accept_write", s, 0.0, 16.0 * attempts);
            k_accept_write<<<(unsigned)blocks, 256, 0, s>>>(ws.raw.get(), attempts,
                                                            ws.offsets.get(), pairs, ws.pairs.get());
            CS_LAUNCH("polar_accept_write");
        }
        have = run;
        want_attempts = (int64_t)((pairs - std::min(have, pairs)) * 1.3) + 8192;
    }
    {
        prof::Scope ps("polar_pairs", s, 0.0, 16.0 * count);
        const int blocks = (int)std::min<int64_t>((count + 255) / 256, 32LL * num_sms());
        k_polar<<<std::max(blocks, 1), 256, 0, s>>>(ws.pairs.get(), count, n, ld, d_out);
        CS_LAUNCH("polar_pairs");
    }
}

}  // namespace cs
