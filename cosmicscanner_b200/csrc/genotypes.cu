// Resident packed genotypes: upload, per-SNP statistics, code counts, repacking.
//
// Reference behaviour restated here:
//   libCosmicCore/src/plink_reader.cpp:67-92   openBed (magic 6C 1B 01, SNP-major only)
//   libCosmicCore/src/plink_reader.cpp:187-239 computeStats (mean, 1/sqrt(2p(1-p)))
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>

#include "cs_internal.h"

namespace cs {

namespace {

// Counts of the four 2-bit codes in a 32-bit word (16 samples).
__device__ __forceinline__ void count_codes(uint32_t w, int& c00, int& c01, int& c10, int& c11) {
    const uint32_t lo = w & 0x55555555u;
    const uint32_t hi = (w >> 1) & 0x55555555u;
    c01 += __popc(lo & ~hi);
    c10 += __popc(hi & ~lo);
    c11 += __popc(hi & lo);
    c00 += __popc(~(lo | hi) & 0x55555555u);
}

// One warp per row: counts of codes 00 (two A1), 01 (missing), 10 (het), 11 (zero A1).
__global__ void k_row_code_counts(const uint8_t* __restrict__ rows, int64_t n_rows,
                                  int64_t stride, int32_t* __restrict__ counts) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = warp; t < n_rows; t += n_warps) {
        const uint4* row = reinterpret_cast<const uint4*>(rows + t * stride);
        int c00 = 0, c01 = 0, c10 = 0, c11 = 0;
        for (int64_t q = lane; q < stride / 16; q += 32) {
            const uint4 v = __ldg(row + q);
            count_codes(v.x, c00, c01, c10, c11);
            count_codes(v.y, c00, c01, c10, c11);
            count_codes(v.z, c00, c01, c10, c11);
            count_codes(v.w, c00, c01, c10, c11);
        }
        c00 = __reduce_add_sync(0xffffffffu, c00);
        c01 = __reduce_add_sync(0xffffffffu, c01);
        c10 = __reduce_add_sync(0xffffffffu, c10);
        c11 = __reduce_add_sync(0xffffffffu, c11);
        if (lane == 0) {
            counts[4 * t + 0] = c00;
            counts[4 * t + 1] = c01;
            counts[4 * t + 2] = c10;
            counts[4 * t + 3] = c11;
        }
    }
}

// plink_reader.cpp:213-233 with the same operation order and no contraction:
// mean = sum / count; p = mean / 2; var = 2 * p * (1 - p); inv_std = 1 / sqrt(var).
__global__ void k_stats_from_counts(const int32_t* __restrict__ counts, int64_t n,
                                    double* __restrict__ mean, double* __restrict__ inv_std,
                                    int32_t* __restrict__ count_out, double* __restrict__ sum_out) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int32_t c00 = counts[4 * j + 0], c10 = counts[4 * j + 2], c11 = counts[4 * j + 3];
    const int32_t count = c00 + c10 + c11;
    const double sum = (double)(2 * (int64_t)c00 + c10);
    count_out[j] = count;
    sum_out[j] = sum;
    if (count > 0) {
        const double m = __ddiv_rn(sum, (double)count);
        const double p = __ddiv_rn(m, 2.0);
        const double var = __dmul_rn(__dmul_rn(2.0, p), __dsub_rn(1.0, p));
        mean[j] = m;
        inv_std[j] = (var < 1e-9) ? 0.0 : __ddiv_rn(1.0, __dsqrt_rn(var));
    } else {
        mean[j] = 0.0;
        inv_std[j] = 0.0;
    }
}

// Samples at or beyond n_samples in the last byte of each row become "missing".
__global__ void k_sanitize_tail(uint8_t* rows, int64_t n_rows, int64_t stride, int64_t last_byte,
                                int used_codes) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n_rows) return;
    uint8_t b = rows[t * stride + last_byte];
    for (int q = used_codes; q < 4; ++q) b = (uint8_t)((b & ~(3u << (2 * q))) | (1u << (2 * q)));
    rows[t * stride + last_byte] = b;
}

__global__ void k_repack(const uint8_t* __restrict__ src, int64_t src_stride,
                         const int32_t* __restrict__ rows, int64_t n_rows,
                         const int32_t* __restrict__ keep, int64_t n_keep,
                         uint8_t* __restrict__ dst, int64_t dst_stride) {
    const int64_t total = n_rows * dst_stride;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = idx / dst_stride;
        const int64_t b = idx - t * dst_stride;
        const uint8_t* srow = src + (int64_t)(rows ? rows[t] : t) * src_stride;
        uint32_t out = 0;
        for (int q = 0; q < 4; ++q) {
            const int64_t r = 4 * b + q;
            uint32_t code = 1;
            if (r < n_keep) {
                const int64_t s = keep ? keep[r] : r;
                code = (srow[s >> 2] >> ((s & 3) * 2)) & 3u;
            }
            out |= code << (2 * q);
        }
        dst[idx] = (uint8_t)out;
    }
}

__global__ void k_col_to_row(const double* __restrict__ src, int64_t ld, int64_t n, int64_t k,
                             double* __restrict__ dst, int64_t kp) {
    const int64_t total = n * kp;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = idx / kp, c = idx - i * kp;
        dst[idx] = c < k ? src[i + c * ld] : 0.0;
    }
}

__global__ void k_row_to_col(const double* __restrict__ src, int64_t kp, int64_t n, int64_t k,
                             double* __restrict__ dst, int64_t ld) {
    const int64_t total = n * k;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = idx / n, i = idx - c * n;
        dst[i + c * ld] = src[i * kp + c];
    }
}

int grid_for(int64_t work, int threads) {
    const int64_t blocks = (work + threads - 1) / threads;
    const int64_t cap = (int64_t)num_sms() * 32;
    return (int)std::max<int64_t>(1, std::min(blocks, cap));
}

}  // namespace

int num_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

void row_code_counts(const cs_packed_view& v, int32_t* d_counts, cudaStream_t s) {
    if (v.n_rows == 0) return;
    const int threads = 256;
    prof::Scope ps("row_code_counts", s, 0.0, (double)v.n_rows * ((v.n_samples + 3) / 4));
    k_row_code_counts<<<grid_for(v.n_rows * 32, threads), threads, 0, s>>>(v.rows, v.n_rows,
                                                                          v.stride, d_counts);
    CS_LAUNCH("row_code_counts");
}

void repack(const uint8_t* src, int64_t src_stride, const int32_t* d_rows, int64_t n_rows,
            const int32_t* d_keep, int64_t n_keep, uint8_t* dst, int64_t dst_stride,
            cudaStream_t s) {
    if (n_rows == 0) return;
    prof::Scope ps("repack", s, 0.0, (double)n_rows * dst_stride);
    k_repack<<<grid_for(n_rows * dst_stride, 256), 256, 0, s>>>(src, src_stride, d_rows, n_rows,
                                                               d_keep, n_keep, dst, dst_stride);
    CS_LAUNCH("repack");
}

void colmajor_to_rowmajor(const double* src, int64_t ld, int64_t n, int64_t k, double* dst,
                          int64_t kp, cudaStream_t s) {
    if (n * kp == 0) return;
    prof::Scope ps("colmajor_to_rowmajor", s, 0.0, 16.0 * n * kp);
    k_col_to_row<<<grid_for(n * kp, 256), 256, 0, s>>>(src, ld, n, k, dst, kp);
    CS_LAUNCH("colmajor_to_rowmajor");
}

void rowmajor_to_colmajor(const double* src, int64_t kp, int64_t n, int64_t k, double* dst,
                          int64_t ld, cudaStream_t s) {
    if (n * k == 0) return;
    prof::Scope ps("rowmajor_to_colmajor", s, 0.0, 16.0 * n * k);
    k_row_to_col<<<grid_for(n * k, 256), 256, 0, s>>>(src, kp, n, k, dst, ld);
    CS_LAUNCH("rowmajor_to_colmajor");
}

// Builds the device-resident matrix from the .bed bytes (magic included).
cs_genotypes* genotypes_from_bed(const uint8_t* bed, size_t n_bytes, int64_t n_samples,
                                 int64_t n_snps) {
    if (n_samples <= 0) fail(CS_ERR_INVALID_ARGUMENT, "No samples found in .fam file");
    if (n_snps < 0) fail(CS_ERR_INVALID_ARGUMENT, "negative SNP count");
    if (bed == nullptr || n_bytes < 3) fail(CS_ERR_FORMAT, "Invalid .bed file (too small)");
    if (bed[0] != 0x6C || bed[1] != 0x1B) fail(CS_ERR_FORMAT, "Invalid .bed file magic number");
    if (bed[2] != 0x01)
        fail(CS_ERR_FORMAT, "Only SNP-major mode (0x01) .bed files are supported");
    const int64_t bps = (n_samples + 3) / 4;
    if ((int64_t)n_bytes < 3 + n_snps * bps)
        fail(CS_ERR_FORMAT, "Invalid .bed file: " + std::to_string(n_bytes) +
                                " bytes < expected " + std::to_string(3 + n_snps * bps));
    prof::HostScope hs("genotypes_upload_stats");
    auto* g = new cs_genotypes();
    static std::atomic<uint64_t> next_uid{1};
    g->uid = next_uid.fetch_add(1);
    try {
        CS_CUDA(cudaGetDevice(&g->device));
        g->n_samples = n_samples;
        g->n_snps = n_snps;
        g->bytes_per_snp = bps;
        g->stride = round_up(bps, kRowAlign);
        const int64_t M = n_snps;
        g->packed.resize(std::max<int64_t>(1, M * g->stride));
        cudaStream_t s = 0;
        if (M > 0) {
            CS_CUDA(cudaMemsetAsync(g->packed.get(), kMissingByte, M * g->stride, s));
            CS_CUDA(cudaMemcpy2DAsync(g->packed.get(), g->stride, bed + 3, bps, bps, M,
                                      cudaMemcpyHostToDevice, s));
            if (n_samples % 4) {
                prof::Scope ps("sanitize_tail", s);
                k_sanitize_tail<<<(unsigned)((M + 255) / 256), 256, 0, s>>>(
                    g->packed.get(), M, g->stride, bps - 1, (int)(n_samples % 4));
                CS_LAUNCH("sanitize_tail");
            }
        }
        g->d_mean.resize(std::max<int64_t>(1, M));
        g->d_inv_std.resize(std::max<int64_t>(1, M));
        g->mean.assign(M, 0.0);
        g->inv_std.assign(M, 0.0);
        g->count.assign(M, 0);
        g->sum.assign(M, 0.0);
        g->code_counts.assign(4 * M, 0);
        if (M > 0) {
            DeviceBuffer<int32_t> counts, cnt;
            DeviceBuffer<double> sum;
            counts.resize(4 * M);
            cnt.resize(M);
            sum.resize(M);
            cs_packed_view v{g->packed.get(), M, n_samples, g->stride};
            row_code_counts(v, counts.get(), s);
            prof::Scope ps("stats_from_counts", s);
            k_stats_from_counts<<<(unsigned)((M + 255) / 256), 256, 0, s>>>(
                counts.get(), M, g->d_mean.get(), g->d_inv_std.get(), cnt.get(), sum.get());
            CS_LAUNCH("stats_from_counts");
            CS_CUDA(cudaMemcpyAsync(g->mean.data(), g->d_mean.get(), M * 8, cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaMemcpyAsync(g->inv_std.data(), g->d_inv_std.get(), M * 8,
                                    cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaMemcpyAsync(g->count.data(), cnt.get(), M * 4, cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaMemcpyAsync(g->sum.data(), sum.get(), M * 8, cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaMemcpyAsync(g->code_counts.data(), counts.get(), M * 16,
                                    cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaStreamSynchronize(s));
        }
    } catch (...) {
        delete g;
        throw;
    }
    return g;
}

static int64_t count_lines(const std::string& path) {
    std::ifstream ifs(path);
    if (!ifs) fail(CS_ERR_IO, "Cannot open file: " + path);
    std::string line;
    int64_t n = 0;
    while (std::getline(ifs, line))
        if (!line.empty()) ++n;
    return n;
}

cs_genotypes* genotypes_open_plink(const std::string& prefix) {
    const int64_t n = count_lines(prefix + ".fam");
    if (n == 0) fail(CS_ERR_INVALID_ARGUMENT, "No samples found in .fam file");
    const int64_t m = count_lines(prefix + ".bim");
    std::ifstream bed(prefix + ".bed", std::ios::binary);
    if (!bed) fail(CS_ERR_IO, "Could not open file for mmap: " + prefix + ".bed");
    bed.seekg(0, std::ios::end);
    const std::streamoff size = bed.tellg();
    bed.seekg(0);
    std::vector<uint8_t> bytes(static_cast<size_t>(size));
    if (size > 0) bed.read(reinterpret_cast<char*>(bytes.data()), size);
    return genotypes_from_bed(bytes.data(), bytes.size(), n, m);
}

}  // namespace cs
