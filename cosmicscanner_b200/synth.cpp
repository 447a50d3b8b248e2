// Synthetic PLINK .bed generator (host, OpenMP) for tests and benchmarks.
//
// Genotypes are Binomial(2, p) draws from a counter-based generator keyed by
// (seed, snp, sample), so the bytes do not depend on the thread count.  Codes follow the
// PLINK convention the reference reads (libCosmicCore/src/plink_reader.cpp:12-21):
// 2 copies of A1 -> 00, 1 -> 10, 0 -> 11, missing -> 01.
#include <stdint.h>

#include <cstring>

namespace {

inline uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

inline double unit(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace

extern "C" {

// freq: n_snps x n_pops allele-1 frequencies (row-major); pop: population of each sample.
// bed_out receives 3 + n_snps * ceil(n/4) bytes (magic included).
void cs_synth_bed(int64_t n, int64_t n_snps, uint64_t seed, const double* freq, int32_t n_pops,
                  const int32_t* pop, double missing_rate, uint8_t* bed_out) {
    const int64_t stride = (n + 3) / 4;
    bed_out[0] = 0x6C;
    bed_out[1] = 0x1B;
    bed_out[2] = 0x01;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t j = 0; j < n_snps; ++j) {
        uint8_t* row = bed_out + 3 + j * stride;
        std::memset(row, 0, stride);
        const uint64_t key = splitmix(seed ^ splitmix((uint64_t)j * 0x632BE59BD9B4E019ull));
        for (int64_t i = 0; i < n; ++i) {
            const uint64_t h1 = splitmix(key + (uint64_t)i * 3);
            const uint64_t h2 = splitmix(key + (uint64_t)i * 3 + 1);
            const uint64_t h3 = splitmix(key + (uint64_t)i * 3 + 2);
            const double p = freq[j * n_pops + (n_pops > 1 ? pop[i] : 0)];
            const int g = (unit(h1) < p) + (unit(h2) < p);
            uint32_t code;
            if (unit(h3) < missing_rate) code = 1;
            else code = g == 2 ? 0u : (g == 1 ? 2u : 3u);
            row[i >> 2] |= (uint8_t)(code << (2 * (i & 3)));
        }
    }
}

// Decodes selected SNPs to dosages (NaN for missing), n x n_sel column-major.
void cs_synth_decode(const uint8_t* bed, int64_t n, const int32_t* snps, int64_t n_sel,
                     double* out) {
    const int64_t stride = (n + 3) / 4;
    const double nan = __builtin_nan("");
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n_sel; ++c) {
        const uint8_t* row = bed + 3 + (int64_t)snps[c] * stride;
        for (int64_t i = 0; i < n; ++i) {
            const int code = (row[i >> 2] >> (2 * (i & 3))) & 3;
            out[i + c * n] = code == 1 ? nan : (code == 0 ? 2.0 : (code == 2 ? 1.0 : 0.0));
        }
    }
}

}  // extern "C"
