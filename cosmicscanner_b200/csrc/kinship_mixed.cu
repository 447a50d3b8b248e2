// Tensor-core (mixed-precision) form of the kinship operator Y = Z Z^T X / M.
//
// Arithmetic.  Both passes run on tcgen05.mma kind::i8 with exact int32 accumulation:
//  * the genotype tile enters as int8 imputed codes e = Q G in {0, Q, 2Q} (Q = 63) for
//    observed calls and e = q_t = rint(Q mu_t) for missing ones, so that e / Q is the
//    mean-imputed dosage up to the row's residual r_t = mu_t - q_t / Q (|r_t| <= 1 / 2Q),
//    together with an int8 missing-indicator tile, both decoded from the packed 2-bit rows in
//    shared memory (a 128-SNP x 128-sample tile, 128-byte swizzled) through a per-row
//    byte-permute table;
//  * right-hand sides are quantised per column into three int8 pieces (base 254) after
//    centring: x' = (x - mean) * 127 / max|x - mean| ~ q1 + q2/254 + q3/254^2, i.e. about
//    23 significant bits, so the only rounding is this quantisation (~6e-8 of the column
//    maximum per element); products and sums are exact while a K slice holds at most
//    kMaxKbPerAccum K-blocks (|e q| <= 126 * 127 per element, plus 127 for the residual).
// With G_ti + mu_t miss_ti = e_ti / Q + r_t miss_ti, the residual term carries the factor
// |r_t| <= 1/126, so two pieces of its operand match the precision of the main term's three:
// per missing call the residual's rounding is at most 1.6e-5 (rows pass) / 3.1e-5 (samples
// pass) of a first-piece step, against up to 1.55e-5 per element for the main term's own.
// Five operand sets per K-block instead of the six of a separate dosage and missing-call
// product.
// Rows pass (U = Z^T X): with S_t, n_t the exact allele sum and observed count of row t,
//   u_t / s_t = mean * (S_t - mu_t n_t) + ( sum_i e_ti x'_i / Q + r_t sum_{i missing} x'_i
//               - mu_t sum_i x'_i ) / scale
// (the centring identity of src/kinship_operator.cpp:135 with the missing-call terms split
// out).  Samples pass (Y = Z W / M, W = s o U):
//   y_i = ( sum_t e_ti w_t / Q + sum_t miss_ti r_t w_t - sum_t mu_t w_t ) / M
// with W f and (Q r o W) f quantised with one factor f = 127 / max|w| (|Q r_t| <= 1/2 keeps
// the second operand's first piece within 64), three pieces of the first and two of the
// second accumulating into the same TMEM columns.  Each pass is one MMA of the imputed-code
// tile against three pieces (N = 3 kc) plus one of the missing-indicator tile against two
// (N = 2 kc): the first two pieces of the same operand in the rows pass (own accumulator,
// scaled by r_t in the epilogue), the residual pieces in the samples pass.
//
// Kernel structure (one CTA per SM, 15 warps): warp 14 issues TMA loads of the packed
// tiles (from HBM) into a deep ring of their own, warp 0 those of the quantised pieces (L2
// resident) into a ring of stages; warps 2-9 decode (with A in TMEM as two groups of four
// that take alternate K-blocks); warp 1 issues the MMAs from one thread
// into a TMEM accumulator; warps 10-13 drain it (tcgen05.ld) and write FP64 slice partials.
// The decoded tile (SNP rows x samples) serves as a K-major A operand in the rows pass and
// as an MN-major A operand in the samples pass.  The TMEMA layouts decode into tensor memory
// instead (tcgen05.st) and the MMAs read A from there; the samples pass then reads a
// sample-major copy of the packed matrix, where A is K-major too, either with the fixed
// dosage table and W / mu o W in six operand sets, or (TMEMA = 5) with each SNP's imputed
// code put in along K under a per-byte missing-call mask (the five sets, and the int32 sums,
// of the shared-memory form).  Wide blocks run on CTA pairs
// (cta_group::2): the partner CTA's MMA warp forwards each of its landed B stages to the
// leader.  Every wait is bounded; a timeout leaves a status code that the host reports as an
// error.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "cs_internal.h"
#include "sm100.cuh"

namespace cs {

namespace {

using namespace sm100;

constexpr int kTile = 128;        // MMA M, and SNP rows / samples per decoded tile
constexpr int kKBlock = 128;      // K elements (int8) per stage: one 128-byte swizzle row
constexpr int kMaxKc = 80;        // column-tile width cap (MMA N = 3 kc <= 256)
constexpr int kWarps = 15;
constexpr int kThreads = kWarps * 32;
constexpr int kDecodeWarp0 = 2, kDecodeWarps = 8;
constexpr int kEpiWarp0 = 10;
constexpr int kPackedWarp = 14;
constexpr uint32_t kTmemCols = 512;
constexpr double kBase = 254.0;
constexpr int kImputeQ = 63;          // dosage scale of the imputed-code tile
constexpr int kMaxKbPerAccum = 1024;  // K-blocks one int32 accumulation may hold:
                                      // 1024 * 128 * (126 * 127 + 127) < 2^31

constexpr int kATileBytes = kTile * kKBlock;     // 16 KB
constexpr int kPackedBytes = kTile * 32;         // 128 rows x 32 B

// Shared memory: a ring of decoded tiles {imputed codes, missing indicators}, a deep ring of
// packed tiles (HBM latency is the longest, so they are requested furthest ahead) and a ring
// of B stages (the quantised pieces, re-read by every CTA from L2).  The rows pass has 3 B
// pieces and accumulators of 3 kc + 2 kc TMEM columns (main and missing-call sums kept
// apart); the samples pass has 5 B pieces (W and Q r o W with one scale) and one accumulator
// of 3 kc columns, double-buffered.
//
// CTA pairs (cta_group::2): a cluster of two CTAs shares each MMA, M = 256 rows (128 from
// each CTA's decoded tile) by N = 3 kc, and each CTA holds only half of the B pieces (rows
// [1.5 kc r, 1.5 kc (r + 1)) of the 3 kc-row set, r = CTA rank).  The tensor core then
// reads half the B bytes per MAC from each SM's shared memory, which is what bounds the
// single-CTA MMAs (about 68 bytes of operands per clock per SM); the smaller B stages leave
// room for wider column tiles and a deeper decode ring, which covers the extra hop of the
// cross-CTA handshakes.
// Narrow single-CTA layouts (column tiles of at most 32): the small B stages leave room for
// a decode ring twice as deep and, in the rows pass, a second accumulator, for widths where the
// MMAs are short and the per-K-block handshakes set the pace.
// Pipeline depths {column-tile width cap, B stages, packed stages, decode stages}:
constexpr int kRowsW = 80, kRowsST = 4, kRowsSP = 8, kRowsSD = 2;
constexpr int kSamplesW = 48, kSamplesST = 3, kSamplesSP = 12, kSamplesSD = 2;
constexpr int kPairRowsW = 80, kPairRowsST = 4, kPairRowsSP = 8, kPairRowsSD = 4;
constexpr int kPairSamplesW = 80, kPairSamplesST = 3, kPairSamplesSP = 6, kPairSamplesSD = 3;
constexpr int kNarrowRowsW = 32, kNarrowRowsST = 4, kNarrowRowsSP = 8, kNarrowRowsSD = 4;
static_assert(kNarrowRowsW == 32, "the plans use one narrow width for both passes");
constexpr int kNarrowSamplesW = 32, kNarrowSamplesST = 3, kNarrowSamplesSP = 8, kNarrowSamplesSD = 4;
// Narrow passes with their A operand in tensor memory (TMEMA): the decoders store the two
// genotype tiles into TMEM (tcgen05.st) and the MMAs read them there, so shared memory
// carries only the packed tiles and the B pieces.  A TMEM operand must be K-major, so the
// samples pass then reads a sample-major copy of the packed matrix (rows = samples, four
// SNPs per byte).  Along its K the SNPs change every two bits, so one byte-permute table
// cannot carry the per-SNP imputed codes: these passes decode with the fixed dosage table and
// carry the missing calls with W and mu o W, three pieces each (the six-set form), except
// TMEMA = 5 below.  TMEMA = 1: column tiles of at most 32, two
// accumulators (5 x 32 columns rows, 3 x 32 samples); TMEMA = 2: tiles of at most 64, one
// accumulator (5 x 64 / 3 x 64), for 33 to 64 right-hand sides.  Then A stages of 64 TMEM
// columns (32 per tile: 128 int8 K elements per lane).
constexpr int kTmemARowsST = 8, kTmemARowsSP = 16, kTmemARowsSD = 3;
constexpr int kTmemASamplesST = 4, kTmemASamplesSP = 16, kTmemASamplesSD = 4;
constexpr int kTmemA64W = 64;
constexpr int kTmemA64RowsST = 6, kTmemA64RowsSP = 12, kTmemA64RowsSD = 3;
constexpr int kTmemA64SamplesST = 3, kTmemA64SamplesSP = 12, kTmemA64SamplesSD = 4;
// TMEMA = 3: the rows pass on CTA pairs with A in TMEM, column tiles of at most 64 (each CTA
// holds half of the B pieces, as in the shared-memory pair form).
constexpr int kTmemAPairRowsST = 8, kTmemAPairRowsSP = 16, kTmemAPairRowsSD = 3;
// TMEMA = 4: the samples pass on CTA pairs over the sample-major copy (six operand sets, each
// CTA holding half of each set).  TMEMA = 5: the same in the five-set form: the decoder
// permutes with the observed-call table (missing -> 0) and a missing-call mask table and ORs
// in q_t from a per-SNP byte array in the decoded K order (a third operation per four codes,
// and the K-block's 128 codes staged with each packed tile); B as in the shared-memory pair
// form.
constexpr int kTmemAPairSamplesST = 4, kTmemAPairSamplesSP = 16, kTmemAPairSamplesSD = 4;
constexpr uint32_t kTmemAStage = 64;

template <bool ROWS, bool PAIR, bool NARROW = false, int TMEMA = 0>
struct Layout {
    static_assert(!(PAIR && NARROW), "narrow layouts are single-CTA");
    static_assert(!TMEMA || (TMEMA == 3 ? (ROWS && PAIR && !NARROW)
                             : TMEMA >= 4 ? (!ROWS && PAIR && !NARROW) : (NARROW && !PAIR)),
                  "A in TMEM: the narrow single-CTA passes, or the passes on CTA pairs");
    // samples passes over the sample-major copy with the fixed dosage table: W and mu o W
    static constexpr bool kSixSets = !ROWS && (TMEMA == 1 || TMEMA == 2 || TMEMA == 4);
    static constexpr int kPieces = ROWS ? 3 : (kSixSets ? 6 : 5);  // per column tile, over the pair
    static constexpr int kMaxW = TMEMA >= 2 ? kTmemA64W
                                 : NARROW ? (ROWS ? kNarrowRowsW : kNarrowSamplesW)
                                 : PAIR ? (ROWS ? kPairRowsW : kPairSamplesW) : (ROWS ? kRowsW : kSamplesW);
    static constexpr int kTmaStages = TMEMA >= 4 ? kTmemAPairSamplesST
                                      : TMEMA == 3 ? kTmemAPairRowsST
                                      : TMEMA == 2 ? (ROWS ? kTmemA64RowsST : kTmemA64SamplesST)
                                      : TMEMA ? (ROWS ? kTmemARowsST : kTmemASamplesST)
                                      : NARROW ? (ROWS ? kNarrowRowsST : kNarrowSamplesST)
                                      : PAIR ? (ROWS ? kPairRowsST : kPairSamplesST) : (ROWS ? kRowsST : kSamplesST);
    static constexpr int kPackedStages = TMEMA >= 4 ? kTmemAPairSamplesSP
                                         : TMEMA == 3 ? kTmemAPairRowsSP
                                         : TMEMA == 2 ? (ROWS ? kTmemA64RowsSP : kTmemA64SamplesSP)
                                         : TMEMA ? (ROWS ? kTmemARowsSP : kTmemASamplesSP)
                                         : NARROW ? (ROWS ? kNarrowRowsSP : kNarrowSamplesSP)
                                         : PAIR ? (ROWS ? kPairRowsSP : kPairSamplesSP) : (ROWS ? kRowsSP : kSamplesSP);
    static constexpr int kDecodeStages = TMEMA >= 4 ? kTmemAPairSamplesSD
                                         : TMEMA == 3 ? kTmemAPairRowsSD
                                         : TMEMA == 2 ? (ROWS ? kTmemA64RowsSD : kTmemA64SamplesSD)
                                         : TMEMA ? (ROWS ? kTmemARowsSD : kTmemASamplesSD)
                                         : NARROW ? (ROWS ? kNarrowRowsSD : kNarrowSamplesSD)
                                         : PAIR ? (ROWS ? kPairRowsSD : kPairSamplesSD) : (ROWS ? kRowsSD : kSamplesSD);
    static constexpr int kAccCols = ROWS ? 5 * kMaxW : 3 * kMaxW;
    static constexpr int kAccBufs = ((ROWS && !NARROW) || TMEMA >= 2) ? 1 : 2;
    static constexpr uint32_t kAccStride = TMEMA ? (uint32_t)kAccCols : 256;
    // TMEM columns of decode stage d's imputed-code / missing-indicator tiles (TMEMA)
    static constexpr uint32_t kTmemA0 = kAccBufs * kAccStride;
    static __host__ __device__ constexpr uint32_t ta(int d) { return kTmemA0 + d * kTmemAStage; }
    static __host__ __device__ constexpr uint32_t tam(int d) { return ta(d) + kTmemAStage / 2; }
    static constexpr int kBBytes = kPieces * kMaxW * 128 / (PAIR ? 2 : 1);  // this CTA's share
    static constexpr int kTmaBytes = kBBytes;
    static constexpr int kDecBytes = 2 * kATileBytes;
    static constexpr int kDecodeRegion = TMEMA ? 0 : kDecodeStages * kDecBytes;
    // samples pass over the sample-major copy: the K-block's 128 imputed codes (P.qperm) ride
    // in each packed stage, so the decoders read them from shared memory
    static constexpr int kQBytes = TMEMA == 5 ? kKBlock : 0;
    // barriers: full / empty per B, packed and decode stage, full / empty per accumulator,
    // `drained`, then the TMEM slot
    static constexpr int kBarBytes =
        (2 * (kTmaStages + kPackedStages + kDecodeStages + kAccBufs) + 1) * 8 + 8;
    static constexpr int kSmem = kDecodeRegion + kTmaStages * kTmaBytes +
                                 kPackedStages * (kPackedBytes + kQBytes) + 1024 + kBarBytes;
    static __host__ __device__ constexpr int a(int d) { return d * kDecBytes; }
    static __host__ __device__ constexpr int am(int d) { return d * kDecBytes + kATileBytes; }
    static __host__ __device__ constexpr int b(int s) { return kDecodeRegion + s * kTmaBytes; }
    static __host__ __device__ constexpr int p(int s) {
        return kDecodeRegion + kTmaStages * kTmaBytes + s * kPackedBytes;
    }
    static __host__ __device__ constexpr int q(int s) {
        return kDecodeRegion + kTmaStages * kTmaBytes + kPackedStages * kPackedBytes + s * kQBytes;
    }
    static __host__ __device__ constexpr int bars() {
        return kDecodeRegion + kTmaStages * kTmaBytes + kPackedStages * (kPackedBytes + kQBytes);
    }
    static_assert(kSmem <= 227 * 1024, "mixed pass exceeds shared memory");
    static_assert(kTmaBytes % 1024 == 0, "TMA stages must keep 1024-byte alignment");
    static_assert(kAccBufs == 1 ? kAccCols <= (int)kTmemCols : kAccCols <= (int)kAccStride,
                  "accumulators exceed TMEM");
    static_assert(!TMEMA || ta(kDecodeStages) <= kTmemCols, "A stages exceed TMEM");
    static_assert(kMaxW % 16 == 0 && kMaxW <= kMaxKc, "column tiles are multiples of 16, at most 80");
};

struct PassArgs {
    int n_tiles, n_ctiles, n_splits;
    int kb_total, kb_per_split;  // K-blocks of the contraction, per slice
    int kc, kp;                  // column tile width, padded column count
    int kc_last;                 // width of the last column tile (a multiple of 16, <= kc)
    const uint32_t* lut;         // per SNP row: imputed code of each 2-bit code (byte-permute table)
    const uint4* qperm;          // samples pass over the sample-major copy: q_t of each SNP at
                                 // its position in the decoded K order, 16 SNPs per uint4
    const double* resid;         // rows pass: r_t = mu_t - q_t / Q per SNP row (epilogue)
    const double* inv_f;         // samples pass: 1 / (Q f) per column
    double* part;                // [n_splits][kp][ld] FP64 slice partials
    int64_t ld;                  // padded output rows
    int* status;
    uint32_t poll_ns;            // pairs: pause between polls of the long, off-critical-path waits
    uint32_t poll_dec_ns;        // pairs: pause between the decoders' polls for a free stage
    int decode_alt;              // TMEMA: two groups of four decoder warps take alternate K-blocks
};

// 16 codes (one 32-bit word, code j in bits 2j..2j+1) -> 16 int8 imputed codes (byte c of
// the row's table `lut` for code c) and 16 missing indicators in the interleaved sample order
// 0 2 4 .. 14 1 3 .. 15 within the group: the even codes, masked in place, are already
// byte-permute selectors (one nibble each), and so are the odd codes after one shift.
// sample_at(p) / position_of(s) convert.
__device__ __forceinline__ void decode_word_interleaved(uint32_t w, uint32_t lut, uint4& dos, uint4& mis) {
    const uint32_t se = w & 0x33333333u, so = (w >> 2) & 0x33333333u;
    dos.x = __byte_perm(lut, 0u, se);
    dos.y = __byte_perm(lut, 0u, se >> 16);
    dos.z = __byte_perm(lut, 0u, so);
    dos.w = __byte_perm(lut, 0u, so >> 16);
    mis.x = __byte_perm(0x00000100u, 0u, se);
    mis.y = __byte_perm(0x00000100u, 0u, se >> 16);
    mis.z = __byte_perm(0x00000100u, 0u, so);
    mis.w = __byte_perm(0x00000100u, 0u, so >> 16);
}
// The same for 16 codes of 16 different SNPs (a word of the sample-major copy): the observed
// calls through the fixed table 2Q / 0 / Q / 0, a 0xFF byte per missing call, and the SNPs'
// imputed codes q (four per word, in the interleaved order) put in under that mask.  The mask
// itself is the missing-indicator tile, as int8 -1: the samples operand of this form carries
// the residual pieces negated, so the products are those of the +1 tile.
constexpr uint32_t kObservedCodes = (uint32_t)(2 * kImputeQ) | ((uint32_t)kImputeQ << 16);
__device__ __forceinline__ void decode_word_imputed(uint32_t w, const uint4& q, uint4& dos, uint4& mis) {
    const uint32_t se = w & 0x33333333u, so = (w >> 2) & 0x33333333u;
    mis.x = __byte_perm(0x0000FF00u, 0u, se);
    mis.y = __byte_perm(0x0000FF00u, 0u, se >> 16);
    mis.z = __byte_perm(0x0000FF00u, 0u, so);
    mis.w = __byte_perm(0x0000FF00u, 0u, so >> 16);
    dos.x = __byte_perm(kObservedCodes, 0u, se) | (mis.x & q.x);
    dos.y = __byte_perm(kObservedCodes, 0u, se >> 16) | (mis.y & q.y);
    dos.z = __byte_perm(kObservedCodes, 0u, so) | (mis.z & q.z);
    dos.w = __byte_perm(kObservedCodes, 0u, so >> 16) | (mis.w & q.w);
}
// position p (0..15) of the interleaved order -> sample offset in the group, and back
__host__ __device__ __forceinline__ int sample_at(int p) { return p < 8 ? 2 * p : 2 * (p - 8) + 1; }
__host__ __device__ __forceinline__ int position_of(int s) { return (s & 1) ? 8 + (s >> 1) : s >> 1; }

template <bool ROWS, bool PAIR, bool NARROW, int TMEMA>
__global__ void __launch_bounds__(kThreads, 1)
k_mixed_pass(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b,
             const __grid_constant__ CUtensorMap tm_bt, PassArgs P) {
    using L = Layout<ROWS, PAIR, NARROW, TMEMA>;
    // K-major A tiles decoded from rows of K elements: the rows pass, and the samples pass over
    // the sample-major copy
    constexpr bool KMAJOR = ROWS || TMEMA != 0;
    constexpr int ST = L::kTmaStages, SP = L::kPackedStages, SD = L::kDecodeStages, NB = L::kAccBufs;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::bars());
    uint64_t* full_t = bars;              // B stage landed (1 arrival + tx bytes)
    uint64_t* empty_t = full_t + ST;      // MMAs reading the B stage done (commit)
    uint64_t* full_p = empty_t + ST;      // packed tile landed (1 arrival + tx bytes)
    uint64_t* empty_p = full_p + SP;      // packed tile decoded (one arrival per decode warp)
    uint64_t* full_d = empty_p + SP;      // decoded (one arrival per decode warp; pair: the
                                          // leader's counts both CTAs' warps and the other
                                          // CTA's B-stage-landed arrival)
    uint64_t* empty_d = full_d + SD;      // MMAs reading the decoded tile done (commit)
    uint64_t* acc_full = empty_d + SD;    // accumulator ready for the epilogue (commit)
    uint64_t* acc_empty = acc_full + NB;  // accumulator drained (one arrival per epilogue warp)
    uint64_t* drained = acc_empty + NB;   // MMA thread's own work complete at exit
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kc = P.kc, kp = P.kp;
    const uint32_t rank = PAIR ? cluster_ctarank() : 0u;
    // TMEMA: the decoder warps either share every K-block (each its lane quarter and one half of
    // K) or split into two groups of four that take alternate K-blocks whole, so that two
    // K-blocks are in decode at once
    const bool alt = TMEMA != 0 && P.decode_alt != 0;
    const uint32_t dec_arrivals = alt ? 4u : (uint32_t)kDecodeWarps;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&full_t[s], 1);
            mbar_init(&empty_t[s], 1);
        }
        for (int s = 0; s < SP; ++s) {
            mbar_init(&full_p[s], 1);
            mbar_init(&empty_p[s], dec_arrivals);
        }
        for (int d = 0; d < SD; ++d) {
            mbar_init(&full_d[d], PAIR ? 2 * dec_arrivals + 1 : dec_arrivals);
            mbar_init(&empty_d[d], 1);
        }
        for (int b = 0; b < NB; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], PAIR ? 8 : 4);
        }
        mbar_init(drained, 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        if (PAIR)
            tmem_alloc_pair(tmem_slot, kTmemCols);
        else
            tmem_alloc(tmem_slot, kTmemCols);
    }
    tc_fence_before();
    if (PAIR)
        cluster_sync_all();
    else
        __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    // A unit is one M tile (pair: two, one per CTA) x one column tile x one K slice; both
    // CTAs of a pair walk the same units.  The column tile varies fastest, so the CTAs that
    // run at the same time share each packed tile through L2 instead of re-reading the packed
    // matrix from HBM once per column tile.
    const int groups = PAIR ? P.n_tiles / 2 : P.n_tiles;
    const int units = groups * P.n_ctiles * P.n_splits;
    const int u0 = PAIR ? (int)cluster_id_x() : (int)blockIdx.x;
    const int ustep = PAIR ? (int)cluster_count_x() : (int)gridDim.x;
    auto unit_coords = [&](int u, int& tile, int& ct, int& split, int& kb0, int& kb1) {
        ct = u % P.n_ctiles;
        const int rest = u / P.n_ctiles;
        const int g = rest % groups;
        tile = PAIR ? 2 * g + (int)rank : g;
        split = rest / groups;
        kb0 = split * P.kb_per_split;
        kb1 = min(P.kb_total, kb0 + P.kb_per_split);
    };
    // columns [ct kc, ct kc + w) of the padded kp; only the last tile may be narrower
    auto width = [&](int ct) { return ct == P.n_ctiles - 1 ? P.kc_last : kc; };
    // Waits on barriers that the MMA commits arrive on (pair: multicast from the leader) or
    // that the other CTA arrives on: pairs poll without suspending (see mbar_poll); the
    // cluster form also acquires what the other CTA released.
    auto wait_commit = [&](uint64_t* bar, uint32_t parity, int code) {
        return PAIR ? mbar_poll(bar, parity, P.status, code) : mbar_wait(bar, parity, P.status, code);
    };
    auto wait_peer = [&](uint64_t* bar, uint32_t parity, int code) {
        return PAIR ? mbar_poll_cluster(bar, parity, P.status, code)
                    : mbar_wait(bar, parity, P.status, code);
    };
    // commit barriers that a warp waits on long and off the critical path (the epilogue's
    // accumulator, the B producer's free stage, the partner CTA's forwarding)
    auto wait_idle = [&](uint64_t* bar, uint32_t parity, int code) {
        return PAIR ? mbar_poll_sleep(bar, parity, P.status, code, P.poll_ns)
                    : mbar_wait(bar, parity, P.status, code);
    };

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer (B)
        if (elect_one()) {
            prefetch_tensormap(&tm_b);
            prefetch_tensormap(&tm_bt);
            uint32_t j = 0;
            bool ok = true;
            for (int u = u0; u < units && ok; u += ustep) {
                int tile, ct, split, kb0, kb1;
                unit_coords(u, tile, ct, split, kb0, kb1);
                const int w = width(ct);
                // the narrower last tile has its own map (box of kc_last rows, pair: half)
                const CUtensorMap* mb = ct == P.n_ctiles - 1 ? &tm_bt : &tm_b;
                const uint32_t bytes = (uint32_t)(L::kPieces * w * 128 / (PAIR ? 2 : 1));
                for (int kb = kb0; kb < kb1; ++kb, ++j) {
                    const int s = j % ST;
                    if (!(ok = wait_idle(&empty_t[s], ((j / ST) & 1) ^ 1, kTimeoutTma))) break;
                    mbar_arrive_expect_tx(&full_t[s], bytes);
                    if (PAIR) {
                        const int hw = w / 2;  // rows of one half-piece
                        if (ROWS) {
                            // half r of each piece, [p0(r) p1(r) p2(r)]: the missing-call MMA
                            // (N = 2 w) then finds [p0(r) p1(r)] at the start of each CTA's stage
#pragma unroll
                            for (int c = 0; c < 3; ++c)
                                tma_load_2d(smem + L::b(s) + c * hw * 128, mb, kb * kKBlock,
                                            c * kp + ct * kc + (int)rank * hw, &full_t[s]);
                        } else {
                            // main set: half-pieces [p0a p0b p1a p1b p2a p2b], this CTA loads
                            // 3 r .. 3 r + 2; residual set: piece 3 + r whole (six sets: the
                            // mu o W set split like the main one)
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                const int h = 3 * (int)rank + c, q = h >> 1;
                                tma_load_2d(smem + L::b(s) + c * hw * 128, mb, kb * kKBlock,
                                            q * kp + ct * kc + (h & 1) * hw, &full_t[s]);
                            }
                            if constexpr (L::kSixSets) {
#pragma unroll
                                for (int c = 0; c < 3; ++c) {
                                    const int h = 3 * (int)rank + c, q = h >> 1;
                                    tma_load_2d(smem + L::b(s) + (3 + c) * hw * 128, mb, kb * kKBlock,
                                                (3 + q) * kp + ct * kc + (h & 1) * hw, &full_t[s]);
                                }
                            } else {
#pragma unroll
                                for (int c = 0; c < 2; ++c)
                                    tma_load_2d(smem + L::b(s) + (3 + c) * hw * 128, mb, kb * kKBlock,
                                                (3 + (int)rank) * kp + ct * kc + c * hw, &full_t[s]);
                            }
                        }
                    } else {
                        for (int q = 0; q < L::kPieces; ++q)
                            tma_load_2d(smem + L::b(s) + q * w * 128, mb, kb * kKBlock,
                                        q * kp + ct * kc, &full_t[s]);
                    }
                }
            }
            // leave no copy in flight
            for (uint32_t q = (j >= (uint32_t)ST ? j - ST : 0); q < j; ++q)
                mbar_wait(&full_t[q % ST], (q / ST) & 1, P.status, kTimeoutTma, 1u << 20);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer (pair: leader)
        if ((!PAIR || rank == 0) && elect_one()) {
            // s8 x s8 -> s32; rows pass: K-major A (SNP rows x samples); samples pass:
            // MN-major A (the same tile read as samples x SNPs); N = 3 w (the three pieces
            // of a column tile side by side) for the imputed codes and 2 w for the missing
            // indicators, M = 128 (pair: 256)
            const uint32_t idesc0 = (2u << 4) | (1u << 7) | (1u << 10) | ((KMAJOR ? 0u : 1u) << 15) |
                                    ((uint32_t)((PAIR ? 2 : 1) * kTile >> 4) << 24);
            uint32_t j = 0;
            int ui = 0;
            bool ok = true;
            for (int u = u0; u < units && ok; u += ustep, ++ui) {
                int tile, ct, split, kb0, kb1;
                unit_coords(u, tile, ct, split, kb0, kb1);
                const int w = width(ct);
                const uint32_t idesc = idesc0 | ((uint32_t)((3 * w) >> 3) << 17);
                // the missing-indicator MMA: two pieces, or the three of mu o W (six sets)
                const uint32_t idesc_m = idesc0 | ((uint32_t)(((L::kSixSets ? 3 : 2) * w) >> 3) << 17);
                const int buf = ui % NB;
                if (!(ok = wait_peer(&acc_empty[buf], ((ui / NB) & 1) ^ 1, kTimeoutMma))) break;
                tc_fence_after();
                const uint32_t acc_main = tmem_base + buf * L::kAccStride;
                const uint32_t acc_miss = ROWS ? acc_main + 3 * w : acc_main;
                for (int kb = kb0; kb < kb1; ++kb, ++j) {
                    const int s = j % ST, d = j % SD;
                    if (!(ok = mbar_wait(&full_t[s], (j / ST) & 1, P.status, kTimeoutMma))) break;
                    if (!(ok = wait_peer(&full_d[d], (j / SD) & 1, kTimeoutMma))) break;
                    tc_fence_after();
                    const uint32_t a = smem_addr(smem + L::a(d));
                    const uint32_t am = smem_addr(smem + L::am(d));
                    const uint32_t b = smem_addr(smem + L::b(s));
                    // rows pass: the first two pieces (this CTA's halves of them); samples
                    // pass: the residual set after the W set (this CTA's share)
                    const uint32_t bm = ROWS ? b : b + 3 * w * 128 / (PAIR ? 2 : 1);
#pragma unroll
                    for (int ks = 0; ks < kKBlock / 32; ++ks) {
                        const uint32_t first = (kb == kb0 && ks == 0) ? 0u : 1u;
                        const uint64_t db = smem_desc_sw128(b + ks * 32, 16, 1024);
                        const uint64_t dbm = smem_desc_sw128(bm + ks * 32, 16, 1024);
                        if constexpr (TMEMA != 0) {
                            // A from TMEM: 32 K elements = 8 columns per MMA
                            if constexpr (PAIR) {
                                mma_i8_pair_tmem_a(acc_main, tmem_base + L::ta(d) + ks * 8, db, idesc, first);
                                mma_i8_pair_tmem_a(acc_miss, tmem_base + L::tam(d) + ks * 8, dbm, idesc_m,
                                                   ROWS ? first : 1u);
                            } else {
                                mma_i8_tmem_a(acc_main, tmem_base + L::ta(d) + ks * 8, db, idesc, first);
                                mma_i8_tmem_a(acc_miss, tmem_base + L::tam(d) + ks * 8, dbm, idesc_m,
                                              ROWS ? first : 1u);
                            }
                            continue;
                        }
                        const uint32_t aoff = ROWS ? ks * 32 : ks * 4096;  // 32 K elements
                        const uint64_t da = smem_desc_sw128(a + aoff, 16, 1024);
                        const uint64_t dm = smem_desc_sw128(am + aoff, 16, 1024);
                        // rows pass: separate missing-call sums; samples pass: the first two
                        // piece columns of the same accumulator
                        if (PAIR) {
                            mma_i8_pair(acc_main, da, db, idesc, first);
                            mma_i8_pair(acc_miss, dm, dbm, idesc_m, ROWS ? first : 1u);
                        } else {
                            mma_i8(acc_main, da, db, idesc, first);
                            mma_i8(acc_miss, dm, dbm, idesc_m, ROWS ? first : 1u);
                        }
                    }
                    if (PAIR) {
                        mma_commit_pair(&empty_t[s], 3);
                        mma_commit_pair(&empty_d[d], 3);
                    } else {
                        mma_commit(&empty_t[s]);
                        mma_commit(&empty_d[d]);
                    }
                }
                if (ok) {
                    if (PAIR)
                        mma_commit_pair(&acc_full[buf], 3);
                    else
                        mma_commit(&acc_full[buf]);
                }
            }
            if (PAIR)
                mma_commit_pair(drained, 1);
            else
                mma_commit(drained);
            mbar_wait(drained, 0, P.status, kTimeoutMma, 1u << 20);
        } else if (PAIR && rank == 1 && elect_one()) {
            // The leader's MMA also reads this CTA's half of each B stage: once the stage has
            // landed here, tell the leader (one arrival on its full_d, after the decoders'),
            // so that no decoder waits for the B copy of the K-block it has just decoded.
            // Like a decoder, wait until the decode stage is free so that the arrival counts
            // toward that stage's next phase.
            uint32_t j = 0;
            bool ok = true;
            for (int u = u0; u < units && ok; u += ustep) {
                int tile, ct, split, kb0, kb1;
                unit_coords(u, tile, ct, split, kb0, kb1);
                for (int kb = kb0; kb < kb1; ++kb, ++j) {
                    const int s = j % ST, d = j % SD;
                    if (!(ok = wait_idle(&empty_d[d], ((j / SD) & 1) ^ 1, kTimeoutDecode))) break;
                    if (!(ok = mbar_wait(&full_t[s], (j / ST) & 1, P.status, kTimeoutDecode))) break;
                    mbar_arrive_remote(mapa_shared(&full_d[d], 0));
                }
            }
        }
    } else if (warp < kEpiWarp0) {
        // ------------------------------------------------------------ decoders
        // thread dt: SNP row dt % 128, 64 samples (16 packed bytes) starting at 64 * (dt / 128);
        // TMEMA: row 32 (warp % 4) + lane, the TMEM lane quarter this warp may access
        const int dt = threadIdx.x - kDecodeWarp0 * 32;
        const int r = TMEMA ? 32 * (warp & 3) + lane : dt & 127;
        const int h = TMEMA ? (warp - kDecodeWarp0) >> 2 : dt >> 7;  // alt: the warp's group
        const int rbase = (r >> 3) * 1024 + (r & 7) * 128;
        uint32_t j = 0;
        bool ok = true;
        for (int u = u0; u < units && ok; u += ustep) {
            int tile, ct, split, kb0, kb1;
            unit_coords(u, tile, ct, split, kb0, kb1);
            // the row's imputed-code table: rows pass SNP tile * 128 + r, samples pass
            // kb * 128 + r (the packed tile's row); over the sample-major copy the fixed dosage
            // table 2 / 0 / 1 / 0 (six sets) or the K-block's imputed codes staged with the
            // packed tile (TMEMA = 5)
            uint32_t lut = ROWS ? __ldg(P.lut + (int64_t)tile * kTile + r) : 0x00010002u;
            for (int kb = kb0; kb < kb1; ++kb, ++j) {
                if (alt && (int)(j & 1u) != h) continue;  // the other group's K-block
                const int sp = j % SP, d = j % SD;
                if (!KMAJOR) lut = __ldg(P.lut + (int64_t)kb * kKBlock + r);
                if (!(ok = PAIR ? mbar_poll_sleep(&empty_d[d], ((j / SD) & 1) ^ 1, P.status,
                                                  kTimeoutDecode, P.poll_dec_ns)
                                : mbar_wait(&empty_d[d], ((j / SD) & 1) ^ 1, P.status, kTimeoutDecode)))
                    break;
                if (!(ok = mbar_wait(&full_p[sp], (j / SP) & 1, P.status, kTimeoutDecode))) break;
                if constexpr (TMEMA) {
                    tc_fence_after();  // after the MMA's release of this stage (empty_d)
                    // one K half of this lane: 64 K elements = 16 TMEM columns of each tile
                    auto decode_half = [&](int hq) {
                        const uint4 packed = *reinterpret_cast<const uint4*>(smem + L::p(sp) + r * 32 + hq * 16);
                        const uint32_t words[4] = {packed.x, packed.y, packed.z, packed.w};
                        // imputed codes of these 64 SNPs (the same for every lane of the warp:
                        // shared-memory broadcasts)
                        uint4 qv[4];
                        if constexpr (TMEMA == 5) {
#pragma unroll
                            for (int cj = 0; cj < 4; ++cj)
                                qv[cj] = *reinterpret_cast<const uint4*>(smem + L::q(sp) + hq * 64 + cj * 16);
                        }
                        uint32_t ev[16], mv[16];
#pragma unroll
                        for (int cj = 0; cj < 4; ++cj) {
                            uint4 dos, mis;
                            if constexpr (TMEMA == 5)
                                decode_word_imputed(words[cj], qv[cj], dos, mis);
                            else
                                decode_word_interleaved(words[cj], lut, dos, mis);
                            ev[4 * cj] = dos.x; ev[4 * cj + 1] = dos.y; ev[4 * cj + 2] = dos.z; ev[4 * cj + 3] = dos.w;
                            mv[4 * cj] = mis.x; mv[4 * cj + 1] = mis.y; mv[4 * cj + 2] = mis.z; mv[4 * cj + 3] = mis.w;
                        }
                        const uint32_t lane_base = tmem_base + ((uint32_t)(32 * (warp & 3)) << 16) + 16 * hq;
                        tmem_st16(lane_base + L::ta(d), ev);
                        tmem_st16(lane_base + L::tam(d), mv);
                    };
                    if (alt) {  // both halves of the K-block (this group's K-blocks only)
                        decode_half(0);
                        decode_half(1);
                    } else {
                        decode_half(h);
                    }
                    tmem_wait_st();
                    tc_fence_before();
                } else {
                    const uint4 packed = *reinterpret_cast<const uint4*>(smem + L::p(sp) + r * 32 + h * 16);
                    const uint32_t words[4] = {packed.x, packed.y, packed.z, packed.w};
                    unsigned char* a = smem + L::a(d);
                    unsigned char* am = smem + L::am(d);
#pragma unroll
                    for (int cj = 0; cj < 4; ++cj) {
                        uint4 dos, mis;
                        decode_word_interleaved(words[cj], lut, dos, mis);
                        const int chunk = 4 * h + cj;  // 16 samples per 16-byte chunk
                        const int off = rbase + ((chunk ^ (r & 7)) << 4);
                        *reinterpret_cast<uint4*>(a + off) = dos;
                        *reinterpret_cast<uint4*>(am + off) = mis;
                    }
                    fence_proxy_async_smem();
                }
                __syncwarp();
                if (lane == 0) {
                    if (PAIR)
                        mbar_arrive_remote(mapa_shared(&full_d[d], 0));
                    else
                        mbar_arrive(&full_d[d]);
                    mbar_arrive(&empty_p[sp]);  // the packed tile has been read
                }
            }
        }
    } else if (warp == kPackedWarp) {
        // ------------------------------------------------------------ TMA producer (packed)
        if (elect_one()) {
            prefetch_tensormap(&tm_a);
            uint32_t j = 0;
            bool ok = true;
            for (int u = u0; u < units && ok; u += ustep) {
                int tile, ct, split, kb0, kb1;
                unit_coords(u, tile, ct, split, kb0, kb1);
                for (int kb = kb0; kb < kb1; ++kb, ++j) {
                    const int sp = j % SP;
                    if (!(ok = mbar_wait(&empty_p[sp], ((j / SP) & 1) ^ 1, P.status, kTimeoutTma))) break;
                    mbar_arrive_expect_tx(&full_p[sp], (uint32_t)(kPackedBytes + L::kQBytes));
                    // packed tile: 128 rows x 32 bytes (128 K elements)
                    if (KMAJOR)
                        tma_load_2d(smem + L::p(sp), &tm_a, kb * 32, tile * kTile, &full_p[sp]);
                    else
                        tma_load_2d(smem + L::p(sp), &tm_a, tile * 32, kb * kKBlock, &full_p[sp]);
                    if constexpr (L::kQBytes != 0)
                        bulk_load_1d(smem + L::q(sp), reinterpret_cast<const unsigned char*>(P.qperm) +
                                                          (int64_t)kb * kKBlock,
                                     (uint32_t)L::kQBytes, &full_p[sp]);
                }
            }
            // leave no copy in flight
            for (uint32_t q = (j >= (uint32_t)SP ? j - SP : 0); q < j; ++q)
                mbar_wait(&full_p[q % SP], (q / SP) & 1, P.status, kTimeoutTma, 1u << 20);
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        int ui = 0;
        bool ok = true;
        const double ib = 1.0 / kBase, ib2 = 1.0 / (kBase * kBase);
        for (int u = u0; u < units && ok; u += ustep, ++ui) {
            int tile, ct, split, kb0, kb1;
            unit_coords(u, tile, ct, split, kb0, kb1);
            const int buf = ui % NB;
            if (!(ok = wait_idle(&acc_full[buf], (ui / NB) & 1, kTimeoutEpilogue))) break;
            tc_fence_after();
            // rows pass: TMEM lane = SNP row; samples pass: lane = position in the decoded
            // tile, whose samples are interleaved within each group of 16
            const int lp = 32 * q + lane;
            const int64_t row = (int64_t)tile * kTile + (KMAJOR ? lp : (lp & ~15) + sample_at(lp & 15));
            const uint32_t tb = tmem_base + buf * L::kAccStride + ((uint32_t)(32 * q) << 16);
            const int w = width(ct);
            double* dst = P.part + ((int64_t)split * kp + (int64_t)ct * kc) * P.ld + row;
            if (ROWS) {
                // TMEM columns: single CTA [p0 p1 p2 | m0 m1] (w each); pair, w / 2 = hw each,
                // [p0a p1a p2a p0b p1b p2b | m0a m1a m0b m1b] (half a from the leader's B)
                constexpr int CH = PAIR ? 8 : 16;
                const double rt = P.resid[row];
                const double inv_q = 1.0 / (double)kImputeQ;
                const int hw = w / 2;
                for (int c0 = 0; c0 < w; c0 += CH) {
                    const bool hb = PAIR && c0 >= hw;
                    const int cc = hb ? c0 - hw : c0;
                    const int step = PAIR ? hw : w;
                    const uint32_t cm = PAIR ? (hb ? 3 * hw : 0) + cc : c0;
                    const uint32_t cx = 3 * w + (PAIR ? (hb ? 2 * hw : 0) + cc : c0);
                    int32_t m1[CH], m2[CH], m3[CH];
                    tmem_ld_cols<CH>(tb + cm, m1);
                    tmem_ld_cols<CH>(tb + cm + step, m2);
                    tmem_ld_cols<CH>(tb + cm + 2 * step, m3);
                    // main sums first, then the missing-call sums (fewer live registers)
                    double mv[CH];
#pragma unroll
                    for (int i = 0; i < CH; ++i)
                        mv[i] = (double)m1[i] + (double)m2[i] * ib + (double)m3[i] * ib2;
                    tmem_ld_cols<CH>(tb + cx, m1);
                    tmem_ld_cols<CH>(tb + cx + step, m2);
#pragma unroll
                    for (int i = 0; i < CH; ++i) {
                        const double xv = (double)m1[i] + (double)m2[i] * ib;
                        dst[(int64_t)(c0 + i) * P.ld] = mv[i] * inv_q + rt * xv;
                    }
                }
            } else {
                for (int c0 = 0; c0 < w; c0 += 16) {
                    int32_t m1[16], m2[16], m3[16];
                    tmem_ld16i(tb + c0, m1);
                    tmem_ld16i(tb + w + c0, m2);
                    tmem_ld16i(tb + 2 * w + c0, m3);
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const double mv = (double)m1[i] + (double)m2[i] * ib + (double)m3[i] * ib2;
                        dst[(int64_t)(c0 + i) * P.ld] = mv * P.inv_f[ct * kc + c0 + i];
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                if (PAIR)
                    mbar_arrive_remote(mapa_shared(&acc_empty[buf], 0));
                else
                    mbar_arrive(&acc_empty[buf]);
            }
        }
    }
    tc_fence_before();
    if (PAIR)
        cluster_sync_all();
    else
        __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        if (PAIR)
            tmem_dealloc_pair(tmem_base, kTmemCols);
        else
            tmem_dealloc(tmem_base, kTmemCols);
    }
}

// ---------------------------------------------------------------- operand preparation
// All reductions here are deterministic: block-level trees in a fixed order, per-block
// partials summed in block order, and maxima through atomicMax on non-negative doubles
// (order independent).  Tiles are 32 columns x 64 rows so that row-major FP64 inputs are
// read with coalesced 256-byte rows and column-major outputs written with coalesced runs.
constexpr int kPrepCols = 32, kPrepRows = 64;

// Quantises v (centred and multiplied by 127 / max) into three int8 pieces of base 254;
// returns the represented value.
__device__ __forceinline__ double quantise3(double v, int8_t& q1, int8_t& q2, int8_t& q3) {
    const double a = rint(v);
    const double r1 = (v - a) * kBase;
    const double b = rint(r1);
    const double r2 = (r1 - b) * kBase;
    const double c = rint(r2);
    q1 = (int8_t)a;
    q2 = (int8_t)b;
    q3 = (int8_t)c;
    return a + b / kBase + c / (kBase * kBase);
}

// Two int8 pieces of base 254 (the residual operand of the samples pass, |v| <= 63.5).
__device__ __forceinline__ void quantise2(double v, int8_t& q1, int8_t& q2) {
    const double a = rint(v);
    q1 = (int8_t)a;
    q2 = (int8_t)rint((v - a) * kBase);
}

__device__ __forceinline__ double quant_factor(unsigned long long bits) {
    const double m = __longlong_as_double((long long)bits);
    return m > 0.0 ? 127.0 / m : 0.0;
}

// Per-column sums, minima and maxima of a row-major FP64 matrix over tiles of 64 rows x 32
// columns (blockIdx.x, blockIdx.y): part[b][c], part[nb + b][c], part[2 nb + b][c], b the row
// tile, nb = gridDim.x.  Warps read 32 consecutive columns of a row (256-byte segments).
__global__ void __launch_bounds__(256)
k_col_stats(const double* __restrict__ X, int64_t ld, int64_t n, int64_t k, double* __restrict__ part) {
    __shared__ double red[3][8][kPrepCols];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int64_t c = (int64_t)blockIdx.y * kPrepCols + tx;
    const int64_t r0 = (int64_t)blockIdx.x * kPrepRows;
    double sm = 0.0, mn = INFINITY, mx = -INFINITY;
    if (c < k)
        for (int64_t r = r0 + ty; r < min(n, r0 + kPrepRows); r += 8) {
            const double v = X[r * ld + c];
            sm += v;
            mn = fmin(mn, v);
            mx = fmax(mx, v);
        }
    red[0][ty][tx] = sm;
    red[1][ty][tx] = mn;
    red[2][ty][tx] = mx;
    __syncthreads();
    if (ty == 0 && c < k) {
        for (int j = 1; j < 8; ++j) {
            sm += red[0][j][tx];
            mn = fmin(mn, red[1][j][tx]);
            mx = fmax(mx, red[2][j][tx]);
        }
        const int64_t nb = gridDim.x;
        part[(int64_t)blockIdx.x * k + c] = sm;
        part[(nb + blockIdx.x) * k + c] = mn;
        part[(2 * nb + blockIdx.x) * k + c] = mx;
    }
}

// mean[c] = (sum over row tiles) / n and maxbits[c] = the bits of max |x - mean[c]| =
// max(max x - mean, mean - min x) (rounding is monotonic, so this equals the maximum of the
// rounded differences).  One warp per column: lane l takes tiles l, l + 32, ..., then a fixed
// shuffle tree (deterministic).
__global__ void __launch_bounds__(256)
k_col_finalize(const double* __restrict__ part, int nb, int64_t k, int64_t n,
               double* __restrict__ mean, unsigned long long* __restrict__ maxbits) {
    const int lane = threadIdx.x & 31;
    const int64_t c = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (c >= k) return;
    double sm = 0.0, mn = INFINITY, mx = -INFINITY;
    for (int b = lane; b < nb; b += 32) {
        sm += part[(int64_t)b * k + c];
        mn = fmin(mn, part[(int64_t)(nb + b) * k + c]);
        mx = fmax(mx, part[(int64_t)(2 * nb + b) * k + c]);
    }
    for (int off = 16; off; off >>= 1) {
        sm += __shfl_xor_sync(0xffffffffu, sm, off);
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, off));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    }
    if (lane == 0) {
        const double m = sm / (double)n;
        mean[c] = m;
        const double a = fmax(fmax(mx - m, m - mn), 0.0);
        maxbits[c] = (unsigned long long)__double_as_longlong(a);
    }
}

// out[c] = scale * sum_b part[b][c]: one warp per column, lane l takes b = l, l + 32, ...,
// then a fixed shuffle tree (deterministic).  Launch with (k + 7) / 8 blocks of 256 threads.
__global__ void __launch_bounds__(256)
k_sum_partials(const double* __restrict__ part, int nb, int64_t k, double scale, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t c = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (c >= k) return;
    double sm = 0.0;
    for (int b = lane; b < nb; b += 32) sm += part[(int64_t)b * k + c];
    for (int off = 16; off; off >>= 1) sm += __shfl_xor_sync(0xffffffffu, sm, off);
    if (lane == 0) out[c] = sm * scale;
}

// Rows-pass operand: B1[q*kp + c][pos(i)] (int8 pieces of (x_ic - mean_c) 127 / max_c, i < n_pad;
// pos interleaves each group of 16 samples as the decoded tiles do) and per-tile sums of the
// represented values qpart[blockIdx.x][c].
__global__ void __launch_bounds__(256)
k_split_rows_operand(const double* __restrict__ X, int64_t ld, int64_t n, int64_t k, int64_t kp,
                     int64_t n_pad, const double* __restrict__ mean,
                     const unsigned long long* __restrict__ maxbits, int8_t* __restrict__ B,
                     double* __restrict__ qpart) {
    __shared__ double tile[kPrepRows][kPrepCols + 1];
    __shared__ double red[8][kPrepCols];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int64_t c0 = (int64_t)blockIdx.y * kPrepCols, r0 = (int64_t)blockIdx.x * kPrepRows;
    for (int rr = ty; rr < kPrepRows; rr += 8) {
        const int64_t r = r0 + rr, c = c0 + tx;
        tile[rr][tx] = (r < n && c < k) ? X[r * ld + c] : 0.0;
    }
    __syncthreads();
    // each warp handles 4 columns; lane covers rows lane and lane + 32
    double qs[4] = {0.0, 0.0, 0.0, 0.0};
    for (int cc = 0; cc < 4; ++cc) {
        const int col = ty * 4 + cc;
        const int64_t c = c0 + col;
        if (c >= kp) continue;
        const double f = c < k ? quant_factor(maxbits[c]) : 0.0;
        const double mc = c < k ? mean[c] : 0.0;
        for (int rr = tx; rr < kPrepRows; rr += 32) {
            const int64_t i = r0 + rr;
            if (i >= n_pad) continue;
            int8_t q1 = 0, q2 = 0, q3 = 0;
            if (c < k && i < n) qs[cc] += quantise3((tile[rr][col] - mc) * f, q1, q2, q3);
            // K position of sample i: the decoded tiles interleave each group of 16 samples
            const int64_t pos = (i & ~(int64_t)15) + position_of((int)(i & 15));
            B[c * n_pad + pos] = q1;
            B[(kp + c) * n_pad + pos] = q2;
            B[(2 * kp + c) * n_pad + pos] = q3;
        }
    }
    for (int cc = 0; cc < 4; ++cc) {
        double v = qs[cc];
        for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (tx == 0) red[0][ty * 4 + cc] = v;  // lane 0 of warp ty owns columns 4ty..4ty+3
    }
    __syncthreads();
    if (threadIdx.x < kPrepCols) {
        const int64_t c = c0 + threadIdx.x;
        if (c < k) qpart[(int64_t)blockIdx.x * k + c] = red[0][threadIdx.x];
    }
}

// Rows-pass reduction, one column per blockIdx.y and 2048 rows per blockIdx.x:
//   inner_tc = (sum_z part[z][c][t] - mu_t Q_c) / f_c + mean_c exc_t
// out = inner * s_t^spow written column-major (out[c * out_ld + t]) or row-major
// (out[t * out_ld + c]); optional maxima of |out| per column.
__global__ void __launch_bounds__(256)
k_reduce_rows(const double* __restrict__ part, int splits, int64_t kp, int64_t ld, int64_t R,
              int64_t k, const double* __restrict__ s_row, int spow,
              const double* __restrict__ exc_row, const double* __restrict__ mu,
              const double* __restrict__ mean, const double* __restrict__ qsum,
              const unsigned long long* __restrict__ maxbits_in, double* __restrict__ out,
              int64_t out_ld, int colmajor, unsigned long long* __restrict__ max_w) {
    __shared__ double red_w[8];
    const int64_t c = blockIdx.y;
    const double f = quant_factor(maxbits_in[c]);
    const double inv_f = f > 0.0 ? 1.0 / f : 0.0;
    const double mc = mean[c], qc = qsum[c];
    double mw = 0.0;
    const int64_t t0 = (int64_t)blockIdx.x * 2048;
    for (int64_t t = t0 + threadIdx.x; t < min(R, t0 + 2048); t += 256) {
        double acc = 0.0;
        for (int z = 0; z < splits; ++z) acc += part[((int64_t)z * kp + c) * ld + t];
        double v = (acc - mu[t] * qc) * inv_f + mc * exc_row[t];
        if (s_row) {
            v *= s_row[t];
            if (spow == 2) v *= s_row[t];
        }
        if (colmajor) out[c * out_ld + t] = v;
        else out[t * out_ld + c] = v;
        mw = fmax(mw, fabs(v));
    }
    if (max_w) {
        for (int off = 16; off; off >>= 1) mw = fmax(mw, __shfl_xor_sync(0xffffffffu, mw, off));
        if ((threadIdx.x & 31) == 0) red_w[threadIdx.x >> 5] = mw;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int j = 1; j < 8; ++j) mw = fmax(mw, red_w[j]);
            atomicMax(max_w + c, (unsigned long long)__double_as_longlong(mw));
        }
    }
}

// Samples-pass operand from W^T (column-major, k x R): three pieces of W f (rows q kp + c)
// and two of (Q r o W) f (rows (3 + q) kp + c), t < r_pad, with ONE factor f = 127 / max|W|
// per column so that both MMAs accumulate into the same TMEM columns (|Q r_t| <= 1/2); 1/(Q f)
// per column; and per-block sums of mu_t W[t][c] (the centring term) in cpart[blockIdx.x][c].
// `interleave` (A in TMEM, over the sample-major copy): SNP t sits at K position
// (t & ~15) + position_of(t & 15), the order in which the decoder writes each group of 16, and
// the residual pieces are negated (that decoder's missing-indicator tile holds -1).
// Grid: (r_pad / 2048, kp).
__global__ void __launch_bounds__(256)
k_split_samples_operand(const double* __restrict__ Wt, int64_t R, int64_t k, int64_t kp,
                        int64_t r_pad, const double* __restrict__ mu,
                        const double* __restrict__ resid,
                        const unsigned long long* __restrict__ max_w, int interleave,
                        int8_t* __restrict__ B, double* __restrict__ inv_f,
                        double* __restrict__ cpart) {
    __shared__ double red[8];
    const int64_t c = blockIdx.y;
    const double f = c < k ? quant_factor(max_w[c]) : 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) inv_f[c] = f > 0.0 ? 1.0 / (f * kImputeQ) : 0.0;
    double cs = 0.0;
    const int64_t t0 = (int64_t)blockIdx.x * 2048;
    for (int64_t t = t0 + threadIdx.x; t < min(r_pad, t0 + 2048); t += 256) {
        int8_t a1 = 0, a2 = 0, a3 = 0, b1 = 0, b2 = 0;
        if (c < k && t < R) {
            const double w = Wt[c * R + t];
            quantise3(w * f, a1, a2, a3);
            quantise2((interleave ? -kImputeQ : kImputeQ) * resid[t] * w * f, b1, b2);
            cs += mu[t] * w;
        }
        const int64_t pos = interleave ? (t & ~(int64_t)15) + position_of((int)(t & 15)) : t;
        B[c * r_pad + pos] = a1;
        B[(kp + c) * r_pad + pos] = a2;
        B[(2 * kp + c) * r_pad + pos] = a3;
        B[(3 * kp + c) * r_pad + pos] = b1;
        B[(4 * kp + c) * r_pad + pos] = b2;
    }
    for (int off = 16; off; off >>= 1) cs += __shfl_xor_sync(0xffffffffu, cs, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cs;
    __syncthreads();
    if (threadIdx.x == 0 && c < k) {
        for (int j = 1; j < 8; ++j) cs += red[j];
        cpart[(int64_t)blockIdx.x * k + c] = cs;
    }
}

// Sample-major copy of a packed view for the samples pass with A in TMEM: dst row i (sample,
// i < n_pad) holds the 2-bit codes of SNPs 0..r_pad-1, four per byte (SNP t at bits
// 2 (t % 4) of byte t / 4), stride r_pad / 4.  SNP rows past R read as code 0 (they meet zero
// B rows); samples past the analysed ones keep the rows' missing-code padding.  One CTA per
// 128-SNP x 128-sample tile: the tile's 128 x 32 packed bytes through shared memory, each
// thread writing 16 bytes of one output row.
__global__ void __launch_bounds__(256)
k_transpose_packed(const uint8_t* __restrict__ src, int64_t R, int64_t stride,
                   uint8_t* __restrict__ dst, int64_t stride_t) {
    __shared__ uint8_t tile[kTile][32];
    const int64_t t0 = (int64_t)blockIdx.x * kTile, b0 = (int64_t)blockIdx.y * 32;
    for (int e = threadIdx.x; e < kTile * 32; e += 256) {
        const int rr = e >> 5, cb = e & 31;
        tile[rr][cb] = (t0 + rr < R) ? src[(t0 + rr) * stride + b0 + cb] : (uint8_t)0;
    }
    __syncthreads();
    const int i = threadIdx.x >> 1;         // sample within the tile
    const int g0 = (threadIdx.x & 1) * 16;  // first output byte (four SNPs each)
    const int col = i >> 2, sh = 2 * (i & 3);
    uint32_t out[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int g = 0; g < 16; ++g) {
        uint32_t byte = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            byte |= (uint32_t)((tile[4 * (g0 + g) + j][col] >> sh) & 3) << (2 * j);
        out[g >> 2] |= byte << (8 * (g & 3));
    }
    uint8_t* d = dst + (b0 * 4 + i) * stride_t + t0 / 4 + g0;
    *reinterpret_cast<uint4*>(d) = make_uint4(out[0], out[1], out[2], out[3]);
}

// Column maxima of max(|W|, |mu o W|) for a column-major R x k W (the six-set samples operand).
__global__ void __launch_bounds__(256)
k_col_absmax_mu(const double* __restrict__ W, int64_t R, const double* __restrict__ mu,
                unsigned long long* __restrict__ max_w) {
    __shared__ double red_w[8];
    const int64_t c = blockIdx.y;
    double mw = 0.0;
    const int64_t t0 = (int64_t)blockIdx.x * 2048;
    for (int64_t t = t0 + threadIdx.x; t < min(R, t0 + 2048); t += 256) {
        const double v = fabs(W[c * R + t]);
        mw = fmax(mw, fmax(v, mu[t] * v));
    }
    for (int off = 16; off; off >>= 1) mw = fmax(mw, __shfl_xor_sync(0xffffffffu, mw, off));
    if ((threadIdx.x & 31) == 0) red_w[threadIdx.x >> 5] = mw;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 1; j < 8; ++j) mw = fmax(mw, red_w[j]);
        atomicMax(max_w + c, (unsigned long long)__double_as_longlong(mw));
    }
}

// Six-set samples operand (A in TMEM over the sample-major copy): pieces of W f (rows q kp + c)
// and of (mu o W) f (rows (3 + q) kp + c) at the K positions of the decoded tiles (SNPs
// interleaved within groups of 16 like samples in the rows pass), f = 127 / max(|W|, |mu W|)
// per column; 1/f per column; per-block sums of mu_t W[t][c] in cpart[blockIdx.x][c].
// Grid: (r_pad / 2048, kp).
__global__ void __launch_bounds__(256)
k_split_samples_t_operand(const double* __restrict__ Wt, int64_t R, int64_t k, int64_t kp,
                          int64_t r_pad, const double* __restrict__ mu,
                          const unsigned long long* __restrict__ max_wmu, int8_t* __restrict__ B,
                          double* __restrict__ inv_f, double* __restrict__ cpart) {
    __shared__ double red[8];
    const int64_t c = blockIdx.y;
    const double f = c < k ? quant_factor(max_wmu[c]) : 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) inv_f[c] = f > 0.0 ? 1.0 / f : 0.0;
    double cs = 0.0;
    const int64_t t0 = (int64_t)blockIdx.x * 2048;
    for (int64_t t = t0 + threadIdx.x; t < min(r_pad, t0 + 2048); t += 256) {
        int8_t a1 = 0, a2 = 0, a3 = 0, b1 = 0, b2 = 0, b3 = 0;
        if (c < k && t < R) {
            const double w = Wt[c * R + t];
            quantise3(w * f, a1, a2, a3);
            quantise3(mu[t] * w * f, b1, b2, b3);
            cs += mu[t] * w;
        }
        const int64_t pos = (t & ~(int64_t)15) + position_of((int)(t & 15));
        B[c * r_pad + pos] = a1;
        B[(kp + c) * r_pad + pos] = a2;
        B[(2 * kp + c) * r_pad + pos] = a3;
        B[(3 * kp + c) * r_pad + pos] = b1;
        B[(4 * kp + c) * r_pad + pos] = b2;
        B[(5 * kp + c) * r_pad + pos] = b3;
    }
    for (int off = 16; off; off >>= 1) cs += __shfl_xor_sync(0xffffffffu, cs, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cs;
    __syncthreads();
    if (threadIdx.x == 0 && c < k) {
        for (int j = 1; j < 8; ++j) cs += red[j];
        cpart[(int64_t)blockIdx.x * k + c] = cs;
    }
}

// Samples-pass reduction: Y[i][c] = (sum_z part[z][c][i] - c0_c) / M.
__global__ void k_reduce_samples(const double* __restrict__ part, int splits, int64_t kp,
                                 int64_t ld, int64_t n, int64_t k, const double* __restrict__ c0,
                                 double inv_m, double* __restrict__ Y, int64_t ldy) {
    const int64_t total = n * k;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = idx / k, c = idx - i * k;  // c fastest: coalesced Y rows
        double acc = 0.0;
        for (int z = 0; z < splits; ++z) acc += part[((int64_t)z * kp + c) * ld + i];
        Y[i * ldy + c] = (acc - c0[c]) * inv_m;
    }
}

// ---------------------------------------------------------------- tensor maps
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    if (!fn) fail(CS_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    return fn;
}

// 2D uint8 tensor map: inner extent `inner` bytes, `outer` rows of `row_bytes`.
CUtensorMap make_map_u8(const void* base, uint64_t inner, uint64_t outer, uint64_t row_bytes,
                        uint32_t box_inner, uint32_t box_outer, bool swizzle) {
    CUtensorMap m;
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {row_bytes};
    const cuuint32_t box[2] = {box_inner, box_outer};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base),
                                   dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                   swizzle ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        fail(CS_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return m;
}

// Both passes run on CTA pairs (cta_group::2) for more than 32 right-hand sides unless
// CS_B200_CTA_PAIRS=0 selects the single-CTA kernels (=1: pairs for every width).  Measured
// on B200 at N=50k, M=100k: k=266 rows 5.4 vs 5.8 ms, samples 5.7 vs 7.7 ms (pair vs
// single); k=32 1.30 vs 1.14 ms per pass, the pair's cross-CTA handshakes per K-block
// outweighing its narrow MMAs.
constexpr int64_t kPairMinColumns = 33;
int pair_mode() {
    static const int mode = [] {
        const char* v = std::getenv("CS_B200_CTA_PAIRS");
        if (v && std::strcmp(v, "0") == 0) return 0;
        if (v && std::strcmp(v, "1") == 0) return 2;
        return 1;
    }();
    return mode;
}
// The narrow passes with A in TMEM, and the 64-wide form of them for 33 to 64 right-hand sides
// instead of CTA pairs (CS_B200_TMEM_A=0: A in shared memory; =1: the 32-wide form only).
// Measured at N=50k, M=100k, per pass (rows / samples): k <= 16 0.70 / 0.80 ms against
// 1.03 / 1.14 with A in shared memory; k = 34 0.90 / 1.07 against 1.15 / 1.24 on CTA pairs;
// k = 64 1.02 / 1.21 against 1.22 / 1.25.
int tmem_a_mode() {
    static const int mode = [] {
        const char* v = std::getenv("CS_B200_TMEM_A");
        if (v && std::strcmp(v, "0") == 0) return 0;
        if (v && std::strcmp(v, "1") == 0) return 1;
        return 2;
    }();
    return mode;
}
bool tmem_a_default() { return tmem_a_mode() != 0; }
// The passes on CTA pairs with A in TMEM (column tiles of at most 64; the samples pass over the
// sample-major copy, six operand sets) as the default pair plans (CS_B200_TMEM_A_PAIRS=0: A in
// shared memory; =1: the rows pass only; =3: the samples pass in the five-set form, TMEMA = 5).
// Measured at N=50k, M=100k, rows / samples per pass against A in shared memory: k = 96
// 1.75 / 1.93 vs 2.31 / 2.48 ms, k = 128 1.89 / 2.12 vs 2.33 / 2.52, k = 192 2.81 / 3.15 vs
// 3.41 / 3.70, k = 266 4.62 / 5.28 vs 4.92 / 5.47.
int tmem_a_pairs_mode() {
    static const int mode = [] {
        const char* v = std::getenv("CS_B200_TMEM_A_PAIRS");
        if (v && std::strcmp(v, "0") == 0) return 0;
        if (v && std::strcmp(v, "1") == 0) return 1;
        if (v && std::strcmp(v, "3") == 0) return 3;
        return 2;
    }();
    return mode;
}
// Pauses between polls in the pair kernels, in nanoseconds: the long waits (the epilogue's
// accumulator, the B producer's free stage, the partner CTA's forwarding;
// CS_B200_POLL_SLEEP_NS, default 128) and the decoders' waits for a free stage
// (CS_B200_POLL_SLEEP_DEC_NS, default 32).  A warp that polls without pause takes issue slots
// from the decoders and the MMA thread on its scheduler.  Measured per pass (rows / samples)
// at N=50k, M=100k, k=266 against no pauses: 4.46 / 5.24 vs 4.76-4.91 / 5.48-5.63 ms; k=96
// 1.67 / 1.88 vs 1.82 / 2.02; 512 ns pauses are slower than none.
// At most 1 us: a wait gives up after 2^26 polls, so the pause sets how long a stalled pass
// takes to report its timeout (about 12 s at the 128 ns default, 70 s at the cap).
uint32_t env_ns(const char* name, uint32_t def) {
    const char* v = std::getenv(name);
    if (!v || !*v) return def;
    const long x = std::strtol(v, nullptr, 10);
    return (uint32_t)std::max(0L, std::min(x, 1000L));
}
uint32_t poll_sleep_ns() {
    static const uint32_t ns = env_ns("CS_B200_POLL_SLEEP_NS", 128u);
    return ns;
}
uint32_t poll_dec_sleep_ns() {
    static const uint32_t ns = env_ns("CS_B200_POLL_SLEEP_DEC_NS", 32u);
    return ns;
}
// Passes with A in TMEM: the decoder warps in two groups of four taking alternate K-blocks
// whole (default), or all eight on every K-block, each one half of K for its lane quarter
// (CS_B200_DECODE_ALT=0).  With one K-block per warp at a time, a K-block's decode latency
// (the packed-tile read, the byte permutes, two tcgen05.st and their wait) set the pace of the
// TMEM passes; two groups keep two K-blocks in decode.  Measured at N=50k, M=100k, rows /
// samples per pass (ms), alternate vs shared, same box: k=16 0.70 / 0.73 vs 1.00 / 1.07; k=48
// 0.93 / 1.06 vs 1.01 / 1.09; k=96 1.66 / 1.97 vs 2.09 / 2.25; k=266 4.23 / 5.06 vs 5.24 / 5.75.
int decode_alt_mode() {
    static const int mode = [] {
        const char* v = std::getenv("CS_B200_DECODE_ALT");
        return (v && std::strcmp(v, "0") == 0) ? 0 : 1;
    }();
    return mode;
}
bool tmem_a_pairs_default() { return tmem_a_pairs_mode() != 0; }
// The narrow single-CTA layout for 32 or fewer right-hand sides (CS_B200_NARROW=0: never).
bool narrow_layouts() {
    static const bool on = [] {
        const char* v = std::getenv("CS_B200_NARROW");
        return !(v && std::strcmp(v, "0") == 0);
    }();
    return on;
}
bool use_cta_pairs(int64_t k) {
    const int mode = pair_mode();
    return mode != 0 && (mode == 2 || k >= kPairMinColumns) && num_sms() >= 2;
}

int blocks_for(int64_t work) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 16LL * num_sms()));
}

// Number of K slices so that about `target` work units cover the GPU, and at least enough that
// no slice holds more than kMaxKbPerAccum K-blocks (the int32 accumulators' exact range).
int choose_splits(int64_t units_per_split, int kb_total, int64_t target) {
    int64_t s = (target + units_per_split - 1) / units_per_split;
    s = std::max<int64_t>(1, std::min<int64_t>(s, std::max(1, kb_total / 8)));
    s = std::max<int64_t>(s, (kb_total + kMaxKbPerAccum - 1) / kMaxKbPerAccum);
    return (int)s;
}

}  // namespace

struct MixedRows {
    // a packed view with per-row centring statistics, ready for the rows pass
    int64_t R = 0, n = 0, r_pad = 0, n_pad = 0;
    DeviceBuffer<double> mu, exc, s, resid;
    DeviceBuffer<uint32_t> lut;  // imputed code of each 2-bit code, one byte per code
    // q_t (byte 1 of lut[t]) at K position (t & ~15) + position_of(t & 15): the samples pass
    // over the sample-major copy reads the imputed codes of 16 SNPs per uint4
    DeviceBuffer<uint4> qperm;
    CUtensorMap tm{};
    const uint8_t* rows = nullptr;  // the view's packed rows (owned by the operator)
    int64_t stride = 0;
    // sample-major copy for the narrow samples pass with A in TMEM (made on first use)
    DeviceBuffer<uint8_t> packed_t;
    CUtensorMap tm_t{};
};

struct MixedWorkspace {
    DeviceBuffer<int8_t> b1, b2;
    DeviceBuffer<double> part, colpart, mean1, qsum, c0, W, inv_f;
    DeviceBuffer<unsigned long long> max1, max_w, max_wmu;
    CUtensorMap tm_b1{}, tm_b2{};
    CUtensorMap tm_b1t{}, tm_b2t{};  // boxes of the last column tile's width
    const void* tm_b1_base = nullptr;
    const void* tm_b2_base = nullptr;
    int64_t tm_b1_key = -1, tm_b2_key = -1;
    DeviceBuffer<int> status;
};

struct MixedOperator {
    MixedRows rows;
    MixedWorkspace ws;
    int64_t last_k = 0;  // columns of ws.W from the last apply (0: none yet)
};

void destroy_mixed(MixedOperator* m) { delete m; }

namespace {

template <bool ROWS, bool PAIR, bool NARROW = false, int TMEMA = 0>
cudaError_t allow_smem() {
    return cudaFuncSetAttribute(k_mixed_pass<ROWS, PAIR, NARROW, TMEMA>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                Layout<ROWS, PAIR, NARROW, TMEMA>::kSmem);
}

void configure_kernels() {
    static PerDeviceOnce configured;
    once_per_device(configured, [] {
        cudaError_t err = allow_smem<true, false>();
        if (err == cudaSuccess) err = allow_smem<false, false>();
        if (err == cudaSuccess) err = allow_smem<true, true>();
        if (err == cudaSuccess) err = allow_smem<false, true>();
        if (err == cudaSuccess) err = allow_smem<true, false, true>();
        if (err == cudaSuccess) err = allow_smem<false, false, true>();
        if (err == cudaSuccess) err = allow_smem<true, false, true, 1>();
        if (err == cudaSuccess) err = allow_smem<false, false, true, 1>();
        if (err == cudaSuccess) err = allow_smem<true, false, true, 2>();
        if (err == cudaSuccess) err = allow_smem<false, false, true, 2>();
        if (err == cudaSuccess) err = allow_smem<true, true, false, 3>();
        if (err == cudaSuccess) err = allow_smem<false, true, false, 4>();
        if (err == cudaSuccess) err = allow_smem<false, true, false, 5>();
        return err;
    }, "configure tensor-core kernels");
}

// Clusters of two CTAs that can be resident at once (an SM without a partner in its GPC
// stays idle): the persistent pair kernels launch exactly that many, since clusters beyond
// it would run as a second wave after the first has finished all its units.
template <bool ROWS>
int resident_pairs() {
    static int cached[64] = {};  // per device ordinal
    int dev = 0;
    CS_CUDA(cudaGetDevice(&dev));
    int& n = cached[dev < 64 ? dev : 0];
    if (n == 0) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(num_sms() & ~1));
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = Layout<ROWS, true>::kSmem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        CS_CUDA(cudaOccupancyMaxActiveClusters(&clusters, k_mixed_pass<ROWS, true, false, 0>, &cfg));
        n = std::max(1, std::min(clusters, num_sms() / 2));
    }
    return n;
}

// One CTA per SM, or (PAIR) as many clusters of two CTAs as are resident together.
template <bool ROWS, bool PAIR, bool NARROW = false, int TMEMA = 0>
void launch_pass(const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& tbt,
                 const PassArgs& P, cudaStream_t s) {
    if constexpr (PAIR) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(2 * resident_pairs<ROWS>()));
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = Layout<ROWS, true, false, TMEMA>::kSmem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CS_CUDA(cudaLaunchKernelEx(&cfg, k_mixed_pass<ROWS, true, false, TMEMA>, ta, tb, tbt, P));
    } else {
        k_mixed_pass<ROWS, false, NARROW, TMEMA>
            <<<num_sms(), kThreads, Layout<ROWS, false, NARROW, TMEMA>::kSmem, s>>>(
            ta, tb, tbt, P);
    }
}

// Per-row statistics: mu_t, exc_t = S_t - mu_t n_t (from code counts c00, c01, c10, c11),
// optional multiplier s_t, and the imputed-code table: codes 00 / 01 (missing) / 10 / 11 ->
// 2Q / q_t / Q / 0 with q_t = rint(Q mu_t), and the residual r_t = mu_t - q_t / Q.  Padding
// rows decode to zeros.
void init_rows(MixedRows& r, const cs_packed_view& v, const double* mean, const int32_t* counts,
               const double* s_or_null) {
    configure_kernels();
    r.R = v.n_rows;
    r.n = v.n_samples;
    // SNP rows padded to 256 as well: the rows pass runs on pairs of 128-row tiles
    r.r_pad = round_up(std::max<int64_t>(r.R, 1), 2 * kTile);
    // samples padded to 256: the samples pass runs on pairs of 128-sample tiles (packed rows
    // hold a multiple of 256 samples, so the padding tiles read missing codes)
    r.n_pad = round_up(std::max<int64_t>(r.n, 1), 2 * kTile);
    std::vector<double> mu(r.r_pad, 0.0), ex(r.r_pad, 0.0), sv(r.r_pad, 0.0), rs(r.r_pad, 0.0);
    std::vector<uint32_t> lut(r.r_pad, 0u);
    std::vector<uint8_t> qp(r.r_pad, 0u);
    for (int64_t t = 0; t < r.R; ++t) {
        const double mt = mean[t];
        mu[t] = mt;
        const double qd = std::isfinite(mt) ? std::rint(kImputeQ * mt) : 0.0;
        const uint32_t q = (uint32_t)std::min(std::max(qd, 0.0), 2.0 * kImputeQ);
        lut[t] = (uint32_t)(2 * kImputeQ) | (q << 8) | ((uint32_t)kImputeQ << 16);
        qp[(t & ~(int64_t)15) + position_of((int)(t & 15))] = (uint8_t)q;
        rs[t] = std::isfinite(mt) ? mt - (double)q / kImputeQ : 0.0;
        const int64_t c00 = counts[4 * t], c10 = counts[4 * t + 2], c11 = counts[4 * t + 3];
        ex[t] = (double)(2 * c00 + c10) - mt * (double)(c00 + c10 + c11);
        sv[t] = s_or_null ? s_or_null[t] : 1.0;
    }
    r.mu.resize(r.r_pad);
    r.exc.resize(r.r_pad);
    r.s.resize(r.r_pad);
    r.resid.resize(r.r_pad);
    r.lut.resize(r.r_pad);
    r.qperm.resize(r.r_pad / 16);
    CS_CUDA(cudaMemcpy(r.resid.get(), rs.data(), 8 * r.r_pad, cudaMemcpyHostToDevice));
    CS_CUDA(cudaMemcpy(r.lut.get(), lut.data(), 4 * r.r_pad, cudaMemcpyHostToDevice));
    CS_CUDA(cudaMemcpy(r.qperm.get(), qp.data(), r.r_pad, cudaMemcpyHostToDevice));
    CS_CUDA(cudaMemcpy(r.mu.get(), mu.data(), 8 * r.r_pad, cudaMemcpyHostToDevice));
    CS_CUDA(cudaMemcpy(r.exc.get(), ex.data(), 8 * r.r_pad, cudaMemcpyHostToDevice));
    CS_CUDA(cudaMemcpy(r.s.get(), sv.data(), 8 * r.r_pad, cudaMemcpyHostToDevice));
    // packed tiles: 32 bytes (128 samples) x 128 SNP rows; rows past R read as zeros and
    // either land in discarded output rows (rows pass) or meet zero B rows (samples pass)
    r.tm = make_map_u8(v.rows, v.stride, std::max<int64_t>(r.R, 1), v.stride, 32, kTile, false);
    r.rows = v.rows;
    r.stride = v.stride;
}

// The sample-major copy of the view (once per context): n_pad rows of r_pad / 4 bytes.
void ensure_transposed(MixedRows& r, cudaStream_t s) {
    if (r.packed_t.get()) return;
    const int64_t stride_t = r.r_pad / 4;
    r.packed_t.resize((size_t)(r.n_pad * stride_t));
    {
        prof::Scope ps("transpose_packed", s, 0.0, 2.0 * (double)r.n_pad * (double)stride_t);
        dim3 g((unsigned)(r.r_pad / kTile), (unsigned)(r.n_pad / kTile));
        k_transpose_packed<<<g, 256, 0, s>>>(r.rows, r.R, r.stride, r.packed_t.get(), stride_t);
        CS_LAUNCH("transpose_packed");
    }
    r.tm_t = make_map_u8(r.packed_t.get(), stride_t, r.n_pad, stride_t, 32, kTile, false);
}

struct Tiling {
    int n_ctiles, kc, kc_last;
    int64_t kp;
};

// Column tiles of max_w columns and a last tile of the remainder rounded up to 16 (the MMA's
// N granularity), so that k = 266 runs 80 + 80 + 80 + 32 columns in the rows pass.  `uniform`
// (the CTA-pair kernel) gives every tile the same width instead.
Tiling tiling_for(int64_t k, int max_w, bool uniform = false) {
    Tiling t;
    t.n_ctiles = (int)((k + max_w - 1) / max_w);
    if (uniform || t.n_ctiles == 1) {
        t.kc = (int)round_up((k + t.n_ctiles - 1) / t.n_ctiles, 16);
        t.kc_last = t.kc;
    } else {
        t.kc = max_w;
        t.kc_last = (int)round_up(k - (int64_t)(t.n_ctiles - 1) * max_w, 16);
    }
    t.kp = (int64_t)t.kc * (t.n_ctiles - 1) + t.kc_last;
    return t;
}

void check_status(MixedWorkspace& ws, cudaStream_t s) {
    int status = 0;
    CS_CUDA(cudaMemcpyAsync(&status, ws.status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    if (status != 0) {
        // cleared on the caller's stream: a non-blocking stream does not wait for the legacy one
        cudaMemsetAsync(ws.status.get(), 0, sizeof(int), s);
        cudaStreamSynchronize(s);
        fail(CS_ERR_CUDA, "tensor-core kinship kernel gave up waiting (status " +
                              std::to_string(status) + ")");
    }
}

// ---------------------------------------------------------------- pass plans and the autotuner
// A pass runs with a plan: CTA pairs or single CTAs, the layout (A in shared memory or in TMEM),
// the column-tile width cap and the number of K slices.  The default plan is the heuristic: up
// to 32 right-hand sides the narrow single-CTA layout with A in TMEM, 33 to 64 its 64-wide
// form, above that CTA pairs with A in TMEM (tiles of at most 64); slices so that about 8
// units per CTA cover the GPU.  The autotuner times the layout x width candidates of a shape
// once (shapes bucketed: rows and samples by factors of 1.25, columns to multiples of 16) and
// keeps the fastest.  It never changes the slice count (the order of the slice sums) nor, in
// the samples pass, the arithmetic form (five or six operand sets), so a tuned pass returns
// the same bits as the default one.  CS_B200_AUTOTUNE=0 turns it off.
struct PassPlan {
    bool pairs = false;
    bool narrow = false;  // single-CTA layout for column tiles of at most 32
    int tmem_a = 0;       // A operand in TMEM: 1 / 2 single CTA (tiles <= 32 / 64), 3 / 4 CTA
                          // pairs (rows / samples, tiles <= 64), 5 the five-set samples pairs
    int max_w = 0;
    int splits = 1;
    bool same_kernel(const PassPlan& o) const {
        return pairs == o.pairs && narrow == o.narrow && tmem_a == o.tmem_a && max_w == o.max_w;
    }
};

// the samples-pass form of a plan: six operand sets over the sample-major copy with the fixed
// dosage table (TMEMA 1, 2, 4), five otherwise
bool six_set_samples(const PassPlan& p) { return p.tmem_a == 1 || p.tmem_a == 2 || p.tmem_a == 4; }

PassPlan default_plan(bool rows, int64_t tiles, int kb, int64_t k) {
    PassPlan p;
    p.pairs = use_cta_pairs(k) && tiles % 2 == 0;
    p.narrow = !p.pairs && k <= kNarrowRowsW && narrow_layouts();
    p.tmem_a = p.narrow && tmem_a_default() ? 1 : 0;
    if (tmem_a_mode() == 2 && narrow_layouts() && k > kNarrowRowsW && k <= kTmemA64W &&
        pair_mode() != 2) {
        p.pairs = false;
        p.narrow = true;
        p.tmem_a = 2;
    }
    if (rows && p.pairs && tmem_a_default() && tmem_a_pairs_default()) p.tmem_a = 3;
    if (!rows && p.pairs && tmem_a_default() && tmem_a_pairs_mode() >= 2)
        p.tmem_a = tmem_a_pairs_mode() == 3 ? 5 : 4;
    p.max_w = p.tmem_a >= 2 ? kTmemA64W
              : p.narrow ? kNarrowRowsW
                       : rows ? (p.pairs ? kPairRowsW : kRowsW) : (p.pairs ? kPairSamplesW : kSamplesW);
    const Tiling tl = tiling_for(k, p.max_w);
    p.splits = p.pairs ? choose_splits(tiles / 2 * tl.n_ctiles, kb, 4LL * num_sms())
                       : choose_splits(tiles * tl.n_ctiles, kb, 8LL * num_sms());
    return p;
}

bool autotune_env() {
    static const bool on = [] {
        const char* v = std::getenv("CS_B200_AUTOTUNE");
        return !(v && std::strcmp(v, "0") == 0);
    }();
    return on;
}

struct TuneKey {
    int rows;
    int64_t rb, nb, kb16;
    bool operator<(const TuneKey& o) const {
        return std::tie(rows, rb, nb, kb16) < std::tie(o.rows, o.rb, o.nb, o.kb16);
    }
};
struct TuneEntry {
    PassPlan plan;
    double ms_best = 0.0, ms_default = 0.0;
    int64_t R = 0, n = 0, k = 0;  // the shape it was tuned on
    int candidates = 0;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneEntry> g_tuned;

int64_t bucket(int64_t x) { return (int64_t)std::floor(std::log((double)std::max<int64_t>(x, 1)) / std::log(1.25)); }

// The plan for a pass of this shape: the tuned one (tuning it now when the shape is new and the
// pass may be timed: autotuning on, the stream not capturing, the work large enough to matter),
// or the default.  `run` executes the pass with a plan.
template <class Run>
PassPlan choose_plan(bool rows, bool allow, int64_t R, int64_t n, int64_t k, int64_t tiles, int kb,
                     cudaStream_t s, Run&& run) {
    const PassPlan def = default_plan(rows, tiles, kb, k);
    if (!allow || !autotune_env() || 2.0 * (double)R * (double)n * (double)k < 2e10) return def;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return def;
    const TuneKey key{rows ? 1 : 0, bucket(R), bucket(n), (k + 15) / 16};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            PassPlan p = it->second.plan;
            p.splits = def.splits;
            return p;
        }
    }
    std::vector<PassPlan> cands;
    const int mode = pair_mode();
    if (mode != 2 && narrow_layouts())
        for (int w = 16; w <= kNarrowRowsW; w += 16)
            for (int t = 0; t < (tmem_a_default() ? 2 : 1); ++t) {
                PassPlan p;
                p.narrow = true;
                p.tmem_a = t;
                p.max_w = w;
                p.splits = def.splits;
                cands.push_back(p);
            }
    if (mode != 0 && tiles % 2 == 0 && num_sms() >= 2 && tmem_a_default())
        for (int w = 48; w <= kTmemA64W; w += 16) {
            PassPlan p;
            p.pairs = true;
            p.tmem_a = rows ? 3 : (def.tmem_a == 5 ? 5 : 4);
            p.max_w = w;
            p.splits = def.splits;
            cands.push_back(p);
        }
    if (mode != 2 && narrow_layouts() && tmem_a_default() && k > kNarrowRowsW)
        for (int w = 48; w <= kTmemA64W; w += 16) {
            PassPlan p;
            p.narrow = true;
            p.tmem_a = 2;
            p.max_w = w;
            p.splits = def.splits;
            cands.push_back(p);
        }
    for (int pr = 0; pr < 2; ++pr) {
        if (pr == 1 && (mode == 0 || tiles % 2 != 0 || num_sms() < 2)) continue;
        if (pr == 0 && mode == 2) continue;
        const int cap_w = rows ? (pr ? kPairRowsW : kRowsW) : (pr ? kPairSamplesW : kSamplesW);
        int last_kc = -1, last_kl = -1, last_ct = -1;
        for (int w = 32; w <= cap_w; w += 16) {
            const Tiling tl = tiling_for(k, w);
            // a wider cap that gives the same tiling as a narrower one is the same plan
            if (tl.kc == last_kc && tl.kc_last == last_kl && tl.n_ctiles == last_ct &&
                !(pr == (def.pairs ? 1 : 0) && !def.narrow && w == def.max_w))
                continue;
            last_kc = tl.kc;
            last_kl = tl.kc_last;
            last_ct = tl.n_ctiles;
            PassPlan p;
            p.pairs = pr == 1;
            p.max_w = w;
            p.splits = def.splits;
            cands.push_back(p);
        }
    }
    // Samples-pass plans over the sample-major copy with the fixed dosage table compute the
    // six-set form (W and mu o W), the others the five-set form: only plans of the default's
    // form are candidates, so a tuned pass returns the same bits as the default one.
    if (!rows) {
        const bool six = six_set_samples(def);
        cands.erase(std::remove_if(cands.begin(), cands.end(),
                                   [six](const PassPlan& p) { return six_set_samples(p) != six; }),
                    cands.end());
    }
    cudaEvent_t e0, e1;
    CS_CUDA(cudaEventCreate(&e0));
    CS_CUDA(cudaEventCreate(&e1));
    TuneEntry best;
    best.plan = def;
    best.ms_best = 1e30;
    try {
        run(def);  // warm: maps, function attributes, operand buffers
        bool have_default = false;
        for (const PassPlan& p : cands) have_default = have_default || p.same_kernel(def);
        if (!have_default) cands.insert(cands.begin(), def);
        for (const PassPlan& p : cands) {
            CS_CUDA(cudaEventRecord(e0, s));
            run(p);
            CS_CUDA(cudaEventRecord(e1, s));
            CS_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            CS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (p.same_kernel(def)) best.ms_default = ms;
            if (ms < best.ms_best) {
                best.ms_best = ms;
                best.plan = p;
            }
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    best.R = R;
    best.n = n;
    best.k = k;
    best.candidates = (int)cands.size();
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned.emplace(key, best);
    }
    return best.plan;
}

// Rows pass over a MixedRows context: for X (n x k, row-major ldx),
//   out_tc = s_t^spow ( sum_i (G_ti - mu_t)[obs] x_ic )  (mean-imputed centred dosages)
// written column-major (out[c * out_ld + t]) or row-major.  With want_max, also the
// per-column maxima of |out| and |mu out| (samples-pass operand scales).
void rows_pass_plan(const PassPlan& plan, MixedRows& r, MixedWorkspace& ws, const double* X,
                    int64_t ldx, int64_t k, double* out, int64_t out_ld, bool colmajor, int spow,
                    bool want_max, cudaStream_t s) {
    const int64_t tiles = r.r_pad / kTile;
    const bool pairs = plan.pairs;
    const Tiling tl = tiling_for(k, plan.max_w);
    const int64_t n = r.n, R = r.R, n_pad = r.n_pad, r_pad = r.r_pad, kp = tl.kp;
    const int kb = (int)(n_pad / kKBlock);
    const int kbs = (kb + plan.splits - 1) / plan.splits;
    const int splits = (kb + kbs - 1) / kbs;  // no empty slice
    if (kbs > kMaxKbPerAccum) fail(CS_ERR_UNSUPPORTED, "rows pass: K slice exceeds the exact int32 range");
    const int rt = (int)((n_pad + kPrepRows - 1) / kPrepRows);
    const int nst = (int)((n + kPrepRows - 1) / kPrepRows);  // row tiles of the column stats
    ws.b1.resize(3 * kp * n_pad);
    ws.part.resize((int64_t)splits * kp * r_pad);
    ws.colpart.resize((int64_t)std::max(rt, 3 * nst) * k);
    ws.mean1.resize(k);
    ws.qsum.resize(k);
    ws.max1.resize(k);
    ws.max_w.resize(k);
    if (!ws.status.get()) {
        ws.status.resize(1);
        // on the pass's own stream, so the kernel never reads the pool's previous contents
        CS_CUDA(cudaMemsetAsync(ws.status.get(), 0, sizeof(int), s));
    }
    // boxes of one column tile's rows (pairs: half of them)
    const int box = pairs ? tl.kc / 2 : tl.kc, box_last = pairs ? tl.kc_last / 2 : tl.kc_last;
    const int64_t key = ((kp * 1000003 + n_pad) * 131 + box_last) * 131 + box;
    if (ws.tm_b1_base != ws.b1.get() || ws.tm_b1_key != key) {
        ws.tm_b1 = make_map_u8(ws.b1.get(), n_pad, 3 * kp, n_pad, kKBlock, box, true);
        ws.tm_b1t = make_map_u8(ws.b1.get(), n_pad, 3 * kp, n_pad, kKBlock, box_last, true);
        ws.tm_b1_base = ws.b1.get();
        ws.tm_b1_key = key;
    }
    {
        prof::Scope ps("mixed_prep_rows_operand", s, 0.0, 24.0 * n * k + 3.0 * kp * n_pad);
        dim3 g1((unsigned)nst, (unsigned)((k + kPrepCols - 1) / kPrepCols));
        k_col_stats<<<g1, 256, 0, s>>>(X, ldx, n, k, ws.colpart.get());
        k_col_finalize<<<(unsigned)((k + 7) / 8), 256, 0, s>>>(ws.colpart.get(), nst, k, n,
                                                               ws.mean1.get(), ws.max1.get());
        dim3 g2((unsigned)rt, (unsigned)((kp + kPrepCols - 1) / kPrepCols));
        k_split_rows_operand<<<g2, 256, 0, s>>>(X, ldx, n, k, kp, n_pad, ws.mean1.get(),
                                                ws.max1.get(), ws.b1.get(), ws.colpart.get());
        k_sum_partials<<<(unsigned)((k + 7) / 8), 256, 0, s>>>(ws.colpart.get(), rt, k, 1.0, ws.qsum.get());
        CS_LAUNCH("mixed rows operand");
    }
    PassArgs P{};
    P.n_tiles = (int)tiles;
    P.n_ctiles = tl.n_ctiles;
    P.n_splits = splits;
    P.kb_total = kb;
    P.kb_per_split = kbs;
    P.kc = tl.kc;
    P.kc_last = tl.kc_last;
    P.kp = (int)kp;
    P.lut = r.lut.get();
    P.resid = r.resid.get();
    P.part = ws.part.get();
    P.ld = r_pad;
    P.status = ws.status.get();
    P.poll_ns = poll_sleep_ns();
    P.poll_dec_ns = poll_dec_sleep_ns();
    P.decode_alt = decode_alt_mode();
    {
        // algorithmic work: 2 n R k flops, one pass over the packed rows
        prof::Scope ps("kinship_rows_tc", s, 2.0 * (double)n * (double)R * (double)k,
                       (double)R * (double)((n + 3) / 4));
        if (pairs && plan.tmem_a == 3)
            launch_pass<true, true, false, 3>(r.tm, ws.tm_b1, ws.tm_b1t, P, s);
        else if (pairs)
            launch_pass<true, true>(r.tm, ws.tm_b1, ws.tm_b1t, P, s);
        else if (plan.narrow && plan.tmem_a == 2)
            launch_pass<true, false, true, 2>(r.tm, ws.tm_b1, ws.tm_b1t, P, s);
        else if (plan.narrow && plan.tmem_a)
            launch_pass<true, false, true, 1>(r.tm, ws.tm_b1, ws.tm_b1t, P, s);
        else if (plan.narrow)
            launch_pass<true, false, true>(r.tm, ws.tm_b1, ws.tm_b1t, P, s);
        else
            launch_pass<true, false>(r.tm, ws.tm_b1, ws.tm_b1t, P, s);
        CS_LAUNCH("kinship_rows_tc");
    }
    if (want_max) CS_CUDA(cudaMemsetAsync(ws.max_w.get(), 0, 8 * k, s));
    {
        prof::Scope ps("mixed_reduce_rows", s, 0.0, 8.0 * splits * kp * R + 8.0 * R * k);
        dim3 g((unsigned)((R + 2047) / 2048), (unsigned)k);
        k_reduce_rows<<<g, 256, 0, s>>>(ws.part.get(), splits, kp, r_pad, R, k, r.s.get(), spow,
                                        r.exc.get(), r.mu.get(), ws.mean1.get(), ws.qsum.get(),
                                        ws.max1.get(), out, out_ld, colmajor ? 1 : 0,
                                        want_max ? ws.max_w.get() : nullptr);
        CS_LAUNCH("reduce_rows");
    }
}

// Samples pass: Y (n x k, row-major ldy) = (Z W) / M for W^T (k x R, column-major) with the
// per-column maxima computed by rows_pass(want_max).
void samples_pass_plan(const PassPlan& plan, MixedRows& r, MixedWorkspace& ws, const double* Wt,
                       int64_t k, double inv_m, double* Y, int64_t ldy, cudaStream_t s) {
    const int64_t tiles = r.n_pad / kTile;
    const bool pairs = plan.pairs;
    const Tiling tl = tiling_for(k, plan.max_w);
    const int64_t n = r.n, R = r.R, n_pad = r.n_pad, r_pad = r.r_pad, kp = tl.kp;
    const int kb = (int)(r_pad / kKBlock);
    const int kbs = (kb + plan.splits - 1) / plan.splits;
    const int splits = (kb + kbs - 1) / kbs;  // no empty slice
    if (kbs > kMaxKbPerAccum) fail(CS_ERR_UNSUPPORTED, "samples pass: K slice exceeds the exact int32 range");
    const int nrb = (int)((r_pad + 2047) / 2048);
    // A in TMEM: over the sample-major copy, B in the decoded K order; six sets with the fixed
    // dosage table, five with the imputed codes (TMEMA = 5)
    const bool tmem_a = plan.tmem_a != 0;  // narrow single-CTA forms, or 4 / 5 on CTA pairs
    const bool six = six_set_samples(plan);
    const int pieces = six ? 6 : 5;
    if (tmem_a) ensure_transposed(r, s);
    ws.b2.resize(pieces * kp * r_pad);
    ws.part.resize((int64_t)splits * kp * n_pad);
    ws.colpart.resize((int64_t)nrb * k);
    ws.inv_f.resize(kp);
    ws.c0.resize(k);
    // boxes of one column tile's rows (pairs: half of them)
    const int box = pairs ? tl.kc / 2 : tl.kc, box_last = pairs ? tl.kc_last / 2 : tl.kc_last;
    const int64_t key = (((kp * 1000003 + r_pad) * 131 + box_last) * 131 + box) * 7 + pieces;
    if (ws.tm_b2_base != ws.b2.get() || ws.tm_b2_key != key) {
        ws.tm_b2 = make_map_u8(ws.b2.get(), r_pad, pieces * kp, r_pad, kKBlock, box, true);
        ws.tm_b2t = make_map_u8(ws.b2.get(), r_pad, pieces * kp, r_pad, kKBlock, box_last, true);
        ws.tm_b2_base = ws.b2.get();
        ws.tm_b2_key = key;
    }
    {
        prof::Scope ps("mixed_prep_samples_operand", s, 0.0, 8.0 * R * k + pieces * kp * r_pad);
        dim3 g((unsigned)nrb, (unsigned)kp);
        if (six) {
            ws.max_wmu.resize(k);
            CS_CUDA(cudaMemsetAsync(ws.max_wmu.get(), 0, 8 * k, s));
            k_col_absmax_mu<<<dim3((unsigned)nrb, (unsigned)k), 256, 0, s>>>(Wt, R, r.mu.get(),
                                                                            ws.max_wmu.get());
            k_split_samples_t_operand<<<g, 256, 0, s>>>(Wt, R, k, kp, r_pad, r.mu.get(),
                                                        ws.max_wmu.get(), ws.b2.get(),
                                                        ws.inv_f.get(), ws.colpart.get());
        } else {
            k_split_samples_operand<<<g, 256, 0, s>>>(Wt, R, k, kp, r_pad, r.mu.get(), r.resid.get(),
                                                      ws.max_w.get(), tmem_a ? 1 : 0, ws.b2.get(),
                                                      ws.inv_f.get(), ws.colpart.get());
        }
        k_sum_partials<<<(unsigned)((k + 7) / 8), 256, 0, s>>>(ws.colpart.get(), nrb, k, 1.0, ws.c0.get());
        CS_LAUNCH("mixed samples operand");
    }
    PassArgs P{};
    P.n_tiles = (int)tiles;
    P.n_ctiles = tl.n_ctiles;
    P.n_splits = splits;
    P.kb_total = kb;
    P.kb_per_split = kbs;
    P.kc = tl.kc;
    P.kc_last = tl.kc_last;
    P.kp = (int)kp;
    P.lut = r.lut.get();
    P.qperm = r.qperm.get();
    P.inv_f = ws.inv_f.get();
    P.part = ws.part.get();
    P.ld = n_pad;
    P.status = ws.status.get();
    P.poll_ns = poll_sleep_ns();
    P.poll_dec_ns = poll_dec_sleep_ns();
    P.decode_alt = decode_alt_mode();
    {
        prof::Scope ps("kinship_samples_tc", s, 2.0 * (double)n * (double)R * (double)k,
                       (double)R * (double)((n + 3) / 4));
        if (pairs && plan.tmem_a == 5)
            launch_pass<false, true, false, 5>(r.tm_t, ws.tm_b2, ws.tm_b2t, P, s);
        else if (pairs && tmem_a)
            launch_pass<false, true, false, 4>(r.tm_t, ws.tm_b2, ws.tm_b2t, P, s);
        else if (pairs)
            launch_pass<false, true>(r.tm, ws.tm_b2, ws.tm_b2t, P, s);
        else if (tmem_a && plan.tmem_a == 2)
            launch_pass<false, false, true, 2>(r.tm_t, ws.tm_b2, ws.tm_b2t, P, s);
        else if (tmem_a)
            launch_pass<false, false, true, 1>(r.tm_t, ws.tm_b2, ws.tm_b2t, P, s);
        else if (plan.narrow)
            launch_pass<false, false, true>(r.tm, ws.tm_b2, ws.tm_b2t, P, s);
        else
            launch_pass<false, false>(r.tm, ws.tm_b2, ws.tm_b2t, P, s);
        CS_LAUNCH("kinship_samples_tc");
    }
    {
        prof::Scope ps("mixed_reduce_samples", s, 0.0, 8.0 * splits * kp * n + 8.0 * n * k);
        k_reduce_samples<<<blocks_for(n * k), 256, 0, s>>>(ws.part.get(), splits, kp, n_pad, n, k,
                                                           ws.c0.get(), inv_m, Y, ldy);
        CS_LAUNCH("reduce_samples");
    }
}

void rows_pass(MixedRows& r, MixedWorkspace& ws, const double* X, int64_t ldx, int64_t k,
               double* out, int64_t out_ld, bool colmajor, int spow, bool want_max,
               cudaStream_t s, bool allow_tune) {
    const int64_t tiles = r.r_pad / kTile;
    const int kb = (int)(r.n_pad / kKBlock);
    const PassPlan plan = choose_plan(true, allow_tune, r.R, r.n, k, tiles, kb, s, [&](const PassPlan& p) {
        rows_pass_plan(p, r, ws, X, ldx, k, out, out_ld, colmajor, spow, want_max, s);
    });
    rows_pass_plan(plan, r, ws, X, ldx, k, out, out_ld, colmajor, spow, want_max, s);
}

void samples_pass(MixedRows& r, MixedWorkspace& ws, const double* Wt, int64_t k, double inv_m,
                  double* Y, int64_t ldy, cudaStream_t s, bool allow_tune, bool sample_major_copy) {
    const int64_t tiles = r.n_pad / kTile;
    const int kb = (int)(r.r_pad / kKBlock);
    PassPlan plan = choose_plan(false, allow_tune && sample_major_copy, r.R, r.n, k, tiles, kb, s,
                                [&](const PassPlan& p) {
                                    samples_pass_plan(p, r, ws, Wt, k, inv_m, Y, ldy, s);
                                });
    if (!sample_major_copy && plan.tmem_a) {
        // A in shared memory (narrow up to 32 columns, otherwise the general layouts): the same
        // int32 sums without the copy; the slice count stays the default plan's
        plan.tmem_a = 0;
        if (plan.max_w > kNarrowSamplesW) {
            plan.narrow = false;
            plan.pairs = use_cta_pairs(k) && tiles % 2 == 0;
            plan.max_w = plan.pairs ? kPairSamplesW : kSamplesW;
        }
    }
    samples_pass_plan(plan, r, ws, Wt, k, inv_m, Y, ldy, s);
}

}  // namespace

static MixedOperator* mixed_for(cs_kinship* op) {
    if (op->mixed) return op->mixed;
    auto* m = new MixedOperator();
    try {
        init_rows(m->rows, op->view, op->mean.data(), op->counts.data(), op->inv_std.data());
    } catch (...) {
        delete m;
        throw;
    }
    op->mixed = m;
    return m;
}

void kinship_apply_mixed(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                         int64_t ldy, cudaStream_t s) {
    if (k <= 0) return;
    const int64_t n = op->rows, R = op->n_active;
    if (R == 0) {
        CS_CUDA(cudaMemset2DAsync(Y, ldy * 8, 0, k * 8, n, s));
        return;
    }
    MixedOperator* m = mixed_for(op);
    m->ws.W.resize(R * k);
    // W^T = s o s o (Z-centred)^T X: the rows pass output already scaled for the samples pass
    m->last_k = 0;
    rows_pass(m->rows, m->ws, X, ldx, k, m->ws.W.get(), R, true, 2, true, s, op->autotune);
    samples_pass(m->rows, m->ws, m->ws.W.get(), k, 1.0 / (double)op->num_variants, Y, ldy, s,
                 op->autotune, op->sample_major_copy);
    check_status(m->ws, s);
    m->last_k = k;
}

// Column maxima of |W| for a column-major R x k W (the samples-pass operand scales):
// atomicMax on the bits of non-negative doubles (order independent).
__global__ void __launch_bounds__(256)
k_col_absmax(const double* __restrict__ W, int64_t R, int64_t k, unsigned long long* __restrict__ max_w) {
    __shared__ double red_w[8];
    const int64_t c = blockIdx.y;
    double mw = 0.0;
    const int64_t t0 = (int64_t)blockIdx.x * 2048;
    for (int64_t t = t0 + threadIdx.x; t < min(R, t0 + 2048); t += 256) mw = fmax(mw, fabs(W[c * R + t]));
    for (int off = 16; off; off >>= 1) mw = fmax(mw, __shfl_xor_sync(0xffffffffu, mw, off));
    if ((threadIdx.x & 31) == 0) red_w[threadIdx.x >> 5] = mw;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 1; j < 8; ++j) mw = fmax(mw, red_w[j]);
        atomicMax(max_w + c, (unsigned long long)__double_as_longlong(mw));
    }
}

// GenotypeMatrix::multiply_Zt_v on tensor cores: U (R x k, row-major ldu) = Z^T X over the
// operator's view rows, X (rows x k, row-major ldx).
void mixed_multiply_zt(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* U,
                       int64_t ldu, cudaStream_t s) {
    if (k <= 0 || op->n_active == 0) return;
    MixedOperator* m = mixed_for(op);
    m->last_k = 0;
    rows_pass(m->rows, m->ws, X, ldx, k, U, ldu, false, 1, false, s, op->autotune);
    check_status(m->ws, s);
}

// GenotypeMatrix::multiply_Z_v on tensor cores: Y (rows x k, row-major ldy) = Z V with
// W = s o V over the view rows given column-major (R x k, leading dimension R).
void mixed_multiply_z(cs_kinship* op, const double* Wcol, int64_t k, double* Y, int64_t ldy,
                      cudaStream_t s) {
    if (k <= 0) return;
    const int64_t R = op->n_active;
    MixedOperator* m = mixed_for(op);
    m->last_k = 0;
    MixedWorkspace& ws = m->ws;
    ws.max_w.resize(k);
    if (!ws.status.get()) {
        ws.status.resize(1);
        CS_CUDA(cudaMemsetAsync(ws.status.get(), 0, sizeof(int), s));
    }
    CS_CUDA(cudaMemsetAsync(ws.max_w.get(), 0, 8 * k, s));
    {
        prof::Scope ps("mixed_col_absmax", s, 0.0, 8.0 * R * k);
        dim3 g((unsigned)((R + 2047) / 2048), (unsigned)k);
        k_col_absmax<<<g, 256, 0, s>>>(Wcol, R, k, ws.max_w.get());
        CS_LAUNCH("col_absmax");
    }
    samples_pass(m->rows, ws, Wcol, k, 1.0, Y, ldy, s, op->autotune, op->sample_major_copy);
    check_status(ws, s);
}

// The autotuner's table as JSON (reported with the profile summary).
std::string autotune_json() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::string out = "[";
    char buf[384];
    bool first = true;
    for (const auto& kv : g_tuned) {
        const TuneEntry& e = kv.second;
        std::snprintf(buf, sizeof buf,
                      "%s{\"pass\": \"%s\", \"R\": %lld, \"n\": %lld, \"k\": %lld, "
                      "\"pairs\": %s, \"narrow\": %s, \"tmem_a\": %s, \"max_width\": %d, \"slices\": %d, "
                      "\"candidates\": %d, \"ms_best\": %.4f, \"ms_default\": %.4f}",
                      first ? "" : ", ", kv.first.rows ? "rows" : "samples", (long long)e.R,
                      (long long)e.n, (long long)e.k, e.plan.pairs ? "true" : "false",
                      e.plan.narrow ? "true" : "false",
                      e.plan.tmem_a == 5 ? "\"pair64_five\"" : e.plan.tmem_a >= 3 ? "\"pair64\""
                      : e.plan.tmem_a == 2 ? "64" : e.plan.tmem_a ? "32" : "false",
                      e.plan.max_w,
                      e.plan.splits, e.candidates,
                      e.ms_best, e.ms_default);
        out += buf;
        first = false;
    }
    return out + "]";
}

const double* mixed_rows_output(const cs_kinship* op, int64_t* R, int64_t* k) {
    if (!op->mixed || op->mixed->last_k == 0) return nullptr;
    *R = op->n_active;
    *k = op->mixed->last_k;
    return op->mixed->ws.W.get();
}

// Scan projection on tensor cores: T[t][c] = sum_i (g_ti - m_t)[observed] B[i][c] for every row
// of a packed view (the analysed samples), m_t = per-row mean of the observed dosages.
struct MixedScan {
    MixedRows rows;
    MixedWorkspace ws;
};

MixedScan* mixed_scan_create(const cs_packed_view& v, const double* row_mean, const int32_t* counts) {
    auto* m = new MixedScan();
    try {
        init_rows(m->rows, v, row_mean, counts, nullptr);
    } catch (...) {
        delete m;
        throw;
    }
    return m;
}

void mixed_scan_destroy(MixedScan* m) { delete m; }

void mixed_scan_project(MixedScan* m, const double* B, int64_t ldb, int64_t k, double* T,
                        int64_t ldt, cudaStream_t s) {
    rows_pass(m->rows, m->ws, B, ldb, k, T, ldt, false, 1, false, s, true);
    check_status(m->ws, s);
}

}  // namespace cs
