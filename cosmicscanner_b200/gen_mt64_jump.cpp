// Build-time generator of the jump table for the 64-bit Mersenne Twister (mt19937_64 as the
// C++ standard defines it: n = 312, m = 156, r = 31, a = 0xB5026F5AA96619E9).
//
// The engine's untempered words x[t] follow a linear recurrence over GF(2) whose state has
// 19937 bits, so every bit position of x satisfies x[t + 19937] = sum_i p_i x[t + i] with
// p(X) the characteristic polynomial (degree 19937, found here by Berlekamp-Massey on one
// bit of the sequence).  Consequently the 312-word window that starts D words later is
//   W_D[w] = XOR over i with g_i = 1 of x[i + w],   g(X) = X^D mod p(X),
// a correlation of the first 19937 + 311 words of the stream with the bits of g.  The table
// holds g for D = c * J, c = 1 .. kChunks - 1, J = 156 * 6720 = 1,048,320 words (a multiple
// of the 156 words the device generator produces per step, so that a chunk ends exactly where
// the next begins): the device draws chunk c from window W_{c J} without generating the words
// before it.  The generator checks one jump against direct generation before writing.
//
// usage: gen_mt64_jump <output .inc>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

constexpr int kN = 312, kM = 156;
constexpr uint64_t kA = 0xB5026F5AA96619E9ull, kUpper = 0xFFFFFFFF80000000ull, kLower = 0x7FFFFFFFull;
constexpr int kDeg = 19937;
constexpr int kWords = (kDeg + 63) / 64;  // 312
constexpr int kChunks = 64;
constexpr int64_t kChunkWords = 156 * 6720;

// untempered stream: x[0..311] = seeded state, then x[t] = x[t-312+156] ^ twist(x[t-312], x[t-311])
std::vector<uint64_t> stream(uint64_t seed, size_t count) {
    std::vector<uint64_t> x(count);
    x[0] = seed;
    for (int i = 1; i < kN && (size_t)i < count; ++i)
        x[i] = 6364136223846793005ull * (x[i - 1] ^ (x[i - 1] >> 62)) + (uint64_t)i;
    for (size_t t = kN; t < count; ++t) {
        const uint64_t y = (x[t - kN] & kUpper) | (x[t - kN + 1] & kLower);
        x[t] = x[t - kN + kM] ^ (y >> 1) ^ ((y & 1) ? kA : 0);
    }
    return x;
}

using Poly = std::vector<uint64_t>;  // bit i = coefficient of X^i

int degree(const Poly& a) {
    for (int w = (int)a.size() - 1; w >= 0; --w)
        if (a[w]) return w * 64 + 63 - __builtin_clzll(a[w]);
    return -1;
}
bool bit(const Poly& a, int i) { return (a[i >> 6] >> (i & 63)) & 1; }
void flip(Poly& a, int i) { a[i >> 6] ^= 1ull << (i & 63); }

// a ^= b << s
void xor_shifted(Poly& a, const Poly& b, int s) {
    const int ws = s >> 6, bs = s & 63;
    int bd = degree(b);
    if (bd < 0) return;
    const size_t need = (size_t)((bd + s) >> 6) + 2;
    if (a.size() < need) a.resize(need, 0);
    for (size_t w = 0; w < b.size(); ++w) {
        if (!b[w]) continue;
        a[w + ws] ^= b[w] << bs;
        if (bs) a[w + ws + 1] ^= b[w] >> (64 - bs);
    }
}

// Berlekamp-Massey over GF(2): connection polynomial C of the shortest LFSR generating s.
Poly berlekamp_massey(const std::vector<uint8_t>& s) {
    const int n = (int)s.size();
    Poly C(n / 64 + 2, 0), B(n / 64 + 2, 0);
    C[0] = B[0] = 1;
    int L = 0, m = 1;
    for (int k = 0; k < n; ++k) {
        int d = s[k];
        for (int i = 1; i <= L; ++i)
            if (bit(C, i)) d ^= s[k - i];
        if (d == 0) {
            ++m;
        } else if (2 * L <= k) {
            Poly T = C;
            xor_shifted(C, B, m);
            L = k + 1 - L;
            B = T;
            m = 1;
        } else {
            xor_shifted(C, B, m);
            ++m;
        }
    }
    C.resize((size_t)(L / 64 + 1));
    // reciprocal: p(X) = X^L C(1/X)
    Poly p((size_t)(L / 64 + 1), 0);
    for (int i = 0; i <= L; ++i)
        if (bit(C, i)) flip(p, L - i);
    return p;
}

// a mod p (p monic of degree kDeg)
void reduce(Poly& a, const Poly& p) {
    for (int d = degree(a); d >= kDeg; d = degree(a)) xor_shifted(a, p, d - kDeg);
    a.resize(kWords, 0);
}

Poly mulmod(const Poly& a, const Poly& b, const Poly& p) {
    Poly r(2 * kWords + 2, 0);
    for (int i = 0; i < kDeg; ++i)
        if (bit(a, i)) xor_shifted(r, b, i);
    reduce(r, p);
    return r;
}

// X^e mod p
Poly xpow(uint64_t e, const Poly& p) {
    Poly result(kWords, 0), base(kWords, 0);
    result[0] = 1;
    base[0] = 2;  // X
    while (e) {
        if (e & 1) result = mulmod(result, base, p);
        e >>= 1;
        if (e) base = mulmod(base, base, p);
    }
    return result;
}

// window of 312 words D later, by the correlation with g = X^D mod p
std::vector<uint64_t> jump(const std::vector<uint64_t>& x, const Poly& g) {
    std::vector<uint64_t> w(kN, 0);
    for (int i = 0; i < kDeg; ++i)
        if (bit(g, i))
            for (int k = 0; k < kN; ++k) w[k] ^= x[i + k];
    return w;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s <output .inc>\n", argv[0]);
        return 2;
    }
    // characteristic polynomial from bit 40 of the untempered words (past the seeded window)
    const std::vector<uint64_t> x = stream(5489ull, kN + 2 * kDeg + 64);
    std::vector<uint8_t> s(2 * kDeg);
    for (int k = 0; k < 2 * kDeg; ++k) s[k] = (x[kN + k] >> 40) & 1;
    const Poly p = berlekamp_massey(s);
    if (degree(p) != kDeg) {
        std::fprintf(stderr, "gen_mt64_jump: characteristic polynomial has degree %d\n", degree(p));
        return 1;
    }
    // jump polynomials X^(c J) mod p, c = 1 .. kChunks - 1
    const Poly step = xpow((uint64_t)kChunkWords, p);
    std::vector<Poly> table(kChunks);
    table[1] = step;
    for (int c = 2; c < kChunks; ++c) table[c] = mulmod(table[c - 1], step, p);
    // check: a jump of 3 J + 1000 words equals direct generation, for another seed
    {
        const int64_t D = 3 * kChunkWords + 1000;
        const std::vector<uint64_t> y = stream(42ull, (size_t)(D + kN + 8));
        const std::vector<uint64_t> w = jump(y, xpow((uint64_t)D, p));
        for (int k = 1; k < kN; ++k)
            if (w[k] != y[D + k]) {
                std::fprintf(stderr, "gen_mt64_jump: jump check failed at word %d\n", k);
                return 1;
            }
        if ((w[0] & kUpper) != (y[D] & kUpper)) {
            std::fprintf(stderr, "gen_mt64_jump: jump check failed at word 0\n");
            return 1;
        }
    }
    FILE* f = std::fopen(argv[1], "w");
    if (!f) return 1;
    std::fprintf(f, "// generated by gen_mt64_jump.cpp: X^(c J) mod p(X), J = %lld, c = 0 .. %d (row 0 unused)\n",
                 (long long)kChunkWords, kChunks - 1);
    std::fprintf(f, "static constexpr long long kMt64JumpWords = %lldLL;\n", (long long)kChunkWords);
    std::fprintf(f, "static constexpr int kMt64JumpChunks = %d;\n", kChunks);
    std::fprintf(f, "__device__ const unsigned long long kMt64Jump[%d][%d] = {\n", kChunks, kWords);
    for (int c = 0; c < kChunks; ++c) {
        std::fprintf(f, "{");
        for (int k = 0; k < kWords; ++k)
            std::fprintf(f, "0x%016llxull%s", (unsigned long long)(c ? table[c][k] : 0ull),
                         k + 1 < kWords ? "," : "");
        std::fprintf(f, "},\n");
    }
    std::fprintf(f, "};\n");
    std::fclose(f);
    return 0;
}
