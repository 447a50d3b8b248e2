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
#include "vce_internal.h"

namespace cs {
namespace {
// X^(c J) mod p(X) for the stream's characteristic polynomial p, generated at build time by
// gen_mt64_jump.cpp (which checks a jump against direct generation)
#include "mt64_jump_table.inc"
}  // namespace
}  // namespace cs

namespace cs {

namespace {

constexpr int kMtN = 312, kMtM = 156;
constexpr uint64_t kMatA = 0xB5026F5AA96619E9ull;
constexpr uint64_t kUpper = 0xFFFFFFFF80000000ull, kLower = 0x7FFFFFFFull;

__device__ __forceinline__ uint64_t temper(uint64_t y) {
    y ^= (y >> 29) & 0x5555555555555555ull;
    y ^= (y << 17) & 0x71D67FFFEDA60000ull;
    y ^= (y << 37) & 0xFFF7EEE000000000ull;
    y ^= y >> 43;
    return y;
}

// One CTA of 156 threads per chunk: CTA c continues the sequence from the 312-word window
// windows[c] (x[K-312 .. K-1]) and writes its n_out words (n_out = chunk, the last CTA:
// total - c chunk) to out[c chunk ..], tempered or not; the last CTA stores its final window
// in final_window when given (the engine advances by n_out rounded up to a multiple of 156).
// Step s produces x[K + 156 s + t], t = 0..155, from x[. - 312] and x[. - 156] (thread t's own
// words of steps s - 2 and s - 1, kept in registers) and x[. - 311] (slot t + 1 of step s - 2,
// or slot 0 of step s - 1 for t = 155), exchanged through a 3-step shared ring: one barrier
// per step.
template <bool TEMPER>
__global__ void __launch_bounds__(kMtM, 1)
k_mt64(const uint64_t* windows, int64_t chunk, int64_t total, uint64_t* __restrict__ out,
       uint64_t* final_window) {
    __shared__ uint64_t ring[3][kMtM];
    const int t = threadIdx.x;
    const int64_t begin = (int64_t)blockIdx.x * chunk;
    const bool last = blockIdx.x + 1 == gridDim.x;
    const int64_t n_out = last ? total - begin : chunk;
    const uint64_t* state = windows + (int64_t)blockIdx.x * kMtN;
    uint64_t p2 = state[t], p1 = state[kMtM + t];
    out += begin;
    ring[1][t] = p2;  // step -2
    ring[2][t] = p1;  // step -1
    __syncthreads();
    const int64_t steps = (n_out + kMtM - 1) / kMtM;
    int cur = 0, older = 1, prev = 2;  // ring slots of steps s, s - 2, s - 1
    for (int64_t st = 0; st < steps; ++st) {
        const uint64_t nb = t + 1 < kMtM ? ring[older][t + 1] : ring[prev][0];
        const uint64_t y = (p2 & kUpper) | (nb & kLower);
        const uint64_t v = p1 ^ (y >> 1) ^ ((y & 1ull) ? kMatA : 0ull);
        ring[cur][t] = v;
        if (st * kMtM + t < n_out) out[st * kMtM + t] = TEMPER ? temper(v) : v;
        p2 = p1;
        p1 = v;
        __syncthreads();
        const int next = older;  // the slot of step s - 2 is free for step s + 1
        older = prev;
        prev = cur;
        cur = next;
    }
    if (last && final_window) {
        final_window[t] = p2;
        final_window[kMtM + t] = p1;
    }
}

// Windows of the chunks c = 1 .. gridDim.x (J words apart) from the untempered stream x
// (x[0..311] = the seeded window, then 19936 further words): word k of window c is the XOR of
// x[i + k] over the set bits i of X^(c J) mod p(X).  CTA (c, part) takes 1 / gridDim.y of the
// polynomial's words, one thread per window word, and XORs its partial into the zeroed
// window; the polynomial's words are read by every thread at once (broadcast), x coalesced.
constexpr int kJumpParts = 8;
__global__ void __launch_bounds__(kMtN)
k_mt64_jump(const uint64_t* __restrict__ x, unsigned long long* __restrict__ windows) {
    const int c = blockIdx.x + 1, k = threadIdx.x;
    const unsigned long long* g = kMt64Jump[c];
    const int w0 = blockIdx.y * kMtN / gridDim.y, w1 = (blockIdx.y + 1) * kMtN / gridDim.y;
    uint64_t acc = 0;
    for (int wi = w0; wi < w1; ++wi) {
        unsigned long long word = g[wi];
        const uint64_t* xb = x + wi * 64 + k;
        while (word) {
            const int b = __ffsll((long long)word) - 1;
            word &= word - 1;
            acc ^= xb[b];
        }
    }
    atomicXor(windows + (int64_t)c * kMtN + k, (unsigned long long)acc);
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

// draws idx (first <= idx < first + count) of the column-by-column stream ->
// out[row * ld + col], row = idx % n, col = idx / n.  One thread per accepted pair: its
// multiplier serves both draws (2 p and 2 p + 1).
__global__ void k_polar(const double* __restrict__ pairs, int64_t first, int64_t count, int64_t n,
                        int64_t ld, double* __restrict__ out) {
    const int64_t p0 = first >> 1, p1 = (first + count - 1) >> 1;
    for (int64_t p = p0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p <= p1;
         p += (int64_t)gridDim.x * blockDim.x) {
        const double x = pairs[2 * p], y = pairs[2 * p + 1];
        const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
        const double mult = sqrt(__ddiv_rn(__dmul_rn(-2.0, log(r2)), r2));
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t idx = 2 * p + h;
            if (idx < first || idx >= first + count) continue;
            const double v = h ? __dmul_rn(x, mult) : __dmul_rn(y, mult);
            const int64_t col = idx / n, row = idx - col * n;
            out[row * ld + col] = v;
        }
    }
}

// out[i * ld + t] = +1 / -1 from the top bit of draw t * n + i
// (std::uniform_int_distribution<int>(0, 1) over mt19937_64 returns the draw's top bit).
__global__ void k_rademacher(const uint64_t* __restrict__ raw, int64_t n, int64_t cols,
                             double* __restrict__ out, int64_t ld) {
    const int64_t total = n * cols;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = e / n, i = e - t * n;
        out[i * ld + t] = (raw[e] >> 63) ? 1.0 : -1.0;
    }
}

std::vector<uint64_t> seeded_state(uint64_t seed) {
    std::vector<uint64_t> st(kMtN);
    st[0] = seed;
    for (int i = 1; i < kMtN; ++i)
        st[i] = 6364136223846793005ull * (st[i - 1] ^ (st[i - 1] >> 62)) + (uint64_t)i;
    return st;
}

}  // namespace

// Incremental generation: the stream is seeded once, pairs are accepted in order as the
// caller asks for them, and column ranges are transformed as soon as their pairs exist, so a
// caller can start using the first columns while later ones are still being drawn.
void omega_begin(uint64_t seed, int64_t total_count, OmegaWorkspace& ws, cudaStream_t s) {
    const std::vector<uint64_t> st = seeded_state(seed);
    // earlier work on s may still read the buffers that grow here
    if ((int64_t)ws.pairs.count < 2 * ((total_count + 1) / 2)) CS_CUDA(cudaStreamSynchronize(s));
    ws.state.resize(kMtN);
    CS_CUDA(cudaMemcpyAsync(ws.state.get(), st.data(), 8 * kMtN, cudaMemcpyHostToDevice, s));
    ws.total_pairs = (total_count + 1) / 2;
    ws.pairs.resize(std::max<int64_t>(2, 2 * ws.total_pairs));
    ws.have = 0;
    ws.position = 0;
}

OmegaWorkspace::~OmegaWorkspace() {
    if (counted) cudaEventSynchronize(counted);
    if (h_counts) cudaFreeHost(h_counts);
    if (counted) cudaEventDestroy(counted);
}

void omega_draw(OmegaWorkspace& ws, int64_t pairs_needed, cudaStream_t s) {
    pairs_needed = std::min(pairs_needed, ws.total_pairs);
    ws.pending_blocks = 0;
    if (ws.have >= pairs_needed) return;
    // acceptance is pi/4 per attempt: draw for 1.3x the missing pairs (a top-up follows in the
    // rare case that is short).  An even number of draws that is a multiple of 156 keeps the
    // stream contiguous across calls: each call advances the engine by exactly its outputs.
    const int64_t want = (int64_t)((pairs_needed - ws.have) * 1.3) + 8192;
    const int64_t attempts = round_up(want, kMtM / 2);
    const int64_t blocks = (attempts + kAttemptsPerBlock - 1) / kAttemptsPerBlock;
    if ((int64_t)ws.raw.count < 2 * attempts || (int64_t)ws.counts.count < blocks ||
        ws.h_counts_cap < blocks) {
        CS_CUDA(cudaStreamSynchronize(s));  // earlier draws' kernels may still read them
        ws.raw.resize(2 * attempts);
        ws.counts.resize(blocks);
        ws.offsets.resize(blocks);
        if (ws.h_counts_cap < blocks) {
            if (ws.h_counts) CS_CUDA(cudaFreeHost(ws.h_counts));
            ws.h_counts = nullptr;
            ws.h_counts_cap = 0;
            CS_CUDA(cudaMallocHost(&ws.h_counts, 4 * blocks));
            ws.h_counts_cap = blocks;
        }
    }
    if (!ws.counted) CS_CUDA(cudaEventCreateWithFlags(&ws.counted, cudaEventDisableTiming));
    const int64_t draws = 2 * attempts;
    if (ws.position == 0 && draws > kMt64JumpWords) {
        // from the seeded window: chunks of J draws in parallel from jumped windows
        constexpr int64_t kPrefix = kMt64JumpWords > 0 ? 19936 : 0;  // x[312 .. 20247]
        const int chunks = (int)std::min<int64_t>(kMt64JumpChunks, (draws + kMt64JumpWords - 1) / kMt64JumpWords);
        ws.prefix.resize(kMtN + kPrefix);
        ws.windows.resize((int64_t)chunks * kMtN);
        CS_CUDA(cudaMemcpyAsync(ws.prefix.get(), ws.state.get(), 8 * kMtN, cudaMemcpyDeviceToDevice, s));
        CS_CUDA(cudaMemcpyAsync(ws.windows.get(), ws.state.get(), 8 * kMtN, cudaMemcpyDeviceToDevice, s));
        {
            prof::Scope ps("mt19937_64_prefix", s, 0.0, 8.0 * kPrefix);
            k_mt64<false><<<1, kMtM, 0, s>>>(ws.state.get(), kPrefix, kPrefix, ws.prefix.get() + kMtN,
                                             nullptr);
            CS_LAUNCH("mt19937_64_prefix");
        }
        {
            prof::Scope ps("mt19937_64_jump", s, 0.0, 8.0 * kMtN * (chunks - 1));
            if (chunks > 1) {
                CS_CUDA(cudaMemsetAsync(ws.windows.get() + kMtN, 0, 8 * (int64_t)(chunks - 1) * kMtN, s));
                k_mt64_jump<<<dim3(chunks - 1, kJumpParts), kMtN, 0, s>>>(
                    ws.prefix.get(), reinterpret_cast<unsigned long long*>(ws.windows.get()));
            }
            CS_LAUNCH("mt19937_64_jump");
        }
        {
            prof::Scope ps("mt19937_64_stream", s, 0.0, 8.0 * draws);
            k_mt64<true><<<chunks, kMtM, 0, s>>>(ws.windows.get(), kMt64JumpWords, draws, ws.raw.get(),
                                                 ws.state.get());
            CS_LAUNCH("mt19937_64_stream");
        }
    } else {
        prof::Scope ps("mt19937_64_stream", s, 0.0, 8.0 * draws);
        k_mt64<true><<<1, kMtM, 0, s>>>(ws.state.get(), draws, draws, ws.raw.get(), ws.state.get());
        CS_LAUNCH("mt19937_64_stream");
    }
    ws.position += draws;
    {
        prof::Scope ps("polar_accept_count", s, 0.0, 16.0 * attempts);
        k_accept_count<<<(unsigned)blocks, 256, 0, s>>>(ws.raw.get(), attempts, ws.counts.get());
        CS_LAUNCH("polar_accept_count");
    }
    CS_CUDA(cudaMemcpyAsync(ws.h_counts, ws.counts.get(), 4 * blocks, cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaEventRecord(ws.counted, s));
    ws.pending_attempts = attempts;
    ws.pending_blocks = blocks;
    ws.pending_target = pairs_needed;
}

void omega_accept(OmegaWorkspace& ws, cudaStream_t s) {
    while (ws.pending_blocks > 0) {
        const int64_t blocks = ws.pending_blocks, attempts = ws.pending_attempts;
        CS_CUDA(cudaEventSynchronize(ws.counted));
        std::vector<int64_t> off(blocks);
        int64_t run = ws.have;
        for (int64_t b = 0; b < blocks; ++b) {
            off[b] = run;
            run += ws.h_counts[b];
        }
        CS_CUDA(cudaMemcpyAsync(ws.offsets.get(), off.data(), 8 * blocks, cudaMemcpyHostToDevice, s));
        {
            prof::Scope ps("polar_accept_write", s, 0.0, 16.0 * attempts);
            k_accept_write<<<(unsigned)blocks, 256, 0, s>>>(ws.raw.get(), attempts, ws.offsets.get(),
                                                            ws.total_pairs, ws.pairs.get());
            CS_LAUNCH("polar_accept_write");
        }
        ws.have = run;
        omega_draw(ws, ws.pending_target, s);  // a top-up when this draw fell short
    }
}

void omega_ensure(OmegaWorkspace& ws, int64_t pairs_needed, cudaStream_t s) {
    omega_draw(ws, pairs_needed, s);
    omega_accept(ws, s);
}

// Normals [c0 n, c1 n) of the column-by-column stream -> columns c0 .. c1 - 1 of d_out.
void omega_emit(OmegaWorkspace& ws, int64_t n, int64_t c0, int64_t c1, double* d_out, int64_t ld,
                cudaStream_t s) {
    const int64_t first = c0 * n, count = (c1 - c0) * n;
    if (count <= 0) return;
    prof::Scope ps("polar_pairs", s, 0.0, 16.0 * count);
    const int blocks = (int)std::min<int64_t>((count / 2 + 256) / 256, 32LL * num_sms());
    k_polar<<<std::max(blocks, 1), 256, 0, s>>>(ws.pairs.get(), first, count, n, ld, d_out);
    CS_LAUNCH("polar_pairs");
}

// Omega (n x cols, written row-major with leading dimension ld) on the device.
void generate_omega_device(uint64_t seed, int64_t n, int64_t cols, double* d_out, int64_t ld,
                           OmegaWorkspace& ws, cudaStream_t s) {
    const int64_t count = n * cols;
    if (count == 0) return;
    omega_begin(seed, count, ws, s);
    omega_ensure(ws, ws.total_pairs, s);
    omega_emit(ws, n, 0, cols, d_out, ld, s);
}

void mt64_seed_device(uint64_t seed, uint64_t* d_state, cudaStream_t s) {
    const std::vector<uint64_t> st = seeded_state(seed);
    CS_CUDA(cudaMemcpyAsync(d_state, st.data(), 8 * kMtN, cudaMemcpyHostToDevice, s));
    CS_CUDA(cudaStreamSynchronize(s));
}

void mt64_generate(uint64_t* d_state, int64_t n_out, uint64_t* d_out, cudaStream_t s) {
    if (n_out <= 0) return;
    prof::Scope ps("mt19937_64_stream", s, 0.0, 8.0 * n_out);
    k_mt64<true><<<1, kMtM, 0, s>>>(d_state, n_out, n_out, d_out, d_state);
    CS_LAUNCH("mt19937_64_stream");
}

void RademacherStream::seed(uint64_t sd, cudaStream_t s) {
    state.resize(kMtN);
    carry.resize(kMtM);
    n_carry = 0;
    mt64_seed_device(sd, state.get(), s);
}

// Draws n * cols words in order; the engine runs in whole 156-word steps, and the words of
// the last step that this call does not use are kept for the next call.
void RademacherStream::draw(int64_t n, int64_t cols, double* out, int64_t ld, cudaStream_t s) {
    const int64_t need = n * cols;
    if (need <= 0) return;
    const int64_t fresh = std::max<int64_t>(0, need - n_carry);
    const int64_t gen = round_up(fresh, kMtM);
    raw.resize(n_carry + gen);
    if (n_carry)
        CS_CUDA(cudaMemcpyAsync(raw.get(), carry.get(), 8 * n_carry, cudaMemcpyDeviceToDevice, s));
    mt64_generate(state.get(), gen, raw.get() + n_carry, s);
    {
        prof::Scope ps("rademacher_signs", s, 0.0, 16.0 * need);
        const int blocks = (int)std::min<int64_t>((need + 255) / 256, 32LL * num_sms());
        k_rademacher<<<std::max(blocks, 1), 256, 0, s>>>(raw.get(), n, cols, out, ld);
        CS_LAUNCH("rademacher_signs");
    }
    const int64_t left = n_carry + gen - need;
    if (left > 0)
        CS_CUDA(cudaMemcpyAsync(carry.get(), raw.get() + need, 8 * left, cudaMemcpyDeviceToDevice, s));
    n_carry = left;
}

}  // namespace cs
