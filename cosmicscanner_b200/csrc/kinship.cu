// Kinship operator K = Z Z^T / M over a sample / variant selection
// (src/kinship_operator.h:53-95, src/kinship_operator.cpp:29-374).
//
// Layout: the operator reads one packed matrix `view` whose rows are the selected
// variants and whose samples are the selected samples, padded to kRowAlign bytes with the
// missing code.  With the identity selection it is the resident genotype matrix itself;
// otherwise the selection is materialised once at construction by a repack kernel, so
// every apply streams contiguous rows (a keep list becomes a gather only once, not on
// every apply as in kinship_operator.cpp:127-134).  Selected variants with 1/sd == 0
// contribute nothing and are dropped from the copy, while the 1/M scaling still counts
// them, as the reference does (kinship_operator.cpp:63-64, 96).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "cs_internal.h"

namespace cs {

cs_kinship* kinship_create(const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                           const int32_t* variants, int64_t n_var) {
    prof::HostScope hs("kinship_create");
    if (g == nullptr) fail(CS_ERR_INVALID_ARGUMENT, "PlinkKinshipOperator: null reader");
    const int64_t N = g->n_samples, M = g->n_snps;
    bool identity = true;
    if (keep && n_keep > 0) {
        for (int64_t i = 0; i < n_keep; ++i)
            if (keep[i] < 0 || keep[i] >= N)
                fail(CS_ERR_INVALID_ARGUMENT, "PlinkKinshipOperator: sample index out of range");
        identity = (n_keep == N);
        for (int64_t i = 0; identity && i < N; ++i) identity = keep[i] == i;
    } else {
        keep = nullptr;
        n_keep = 0;
    }
    if (variants && n_var > 0) {
        bool all = (n_var == M);
        for (int64_t j = 0; j < n_var; ++j) {
            if (variants[j] < 0 || variants[j] >= M)
                fail(CS_ERR_INVALID_ARGUMENT, "PlinkKinshipOperator: variant index out of range");
            all = all && variants[j] == j;
        }
        if (all) {  // every SNP in file order: the resident matrix serves as is
            variants = nullptr;
            n_var = 0;
        }
    } else {
        variants = nullptr;
        n_var = 0;
    }
    auto* op = new cs_kinship();
    try {
        op->g = g;
        op->rows = keep ? n_keep : N;
        op->num_variants = variants ? n_var : M;
        if (op->num_variants == 0) fail(CS_ERR_INVALID_ARGUMENT, "PlinkKinshipOperator: no variants selected");
        cudaStream_t s = 0;
        std::vector<int32_t> active;
        op->keep_identity = identity;
        if (!variants && identity) {
            op->view = cs_packed_view{g->packed.get(), M, N, g->stride};
            op->n_active = M;
            op->mean = g->mean;
            op->inv_std = g->inv_std;
            op->view_snp.resize(M);
            for (int64_t t = 0; t < M; ++t) op->view_snp[t] = (int32_t)t;
            op->view_pos = op->view_snp;
        } else {
            active.reserve(op->num_variants);
            for (int64_t t = 0; t < op->num_variants; ++t) {
                const int32_t j = variants ? variants[t] : (int32_t)t;
                if (g->inv_std[j] != 0.0) {
                    active.push_back(j);
                    op->view_pos.push_back((int32_t)t);
                }
            }
            op->n_active = (int64_t)active.size();
            const int64_t stride = round_up((op->rows + 3) / 4, kRowAlign);
            op->own_packed.resize(std::max<int64_t>(1, op->n_active * stride));
            DeviceBuffer<int32_t> d_rows, d_keep;
            d_rows.resize(std::max<int64_t>(1, op->n_active));
            if (op->n_active)
                CS_CUDA(cudaMemcpyAsync(d_rows.get(), active.data(), op->n_active * 4,
                                        cudaMemcpyHostToDevice, s));
            if (!identity) {
                d_keep.resize(n_keep);
                CS_CUDA(cudaMemcpyAsync(d_keep.get(), keep, n_keep * 4, cudaMemcpyHostToDevice, s));
            }
            repack(g->packed.get(), g->stride, d_rows.get(), op->n_active,
                   identity ? nullptr : d_keep.get(), op->rows, op->own_packed.get(), stride, s);
            CS_CUDA(cudaStreamSynchronize(s));
            op->view = cs_packed_view{op->own_packed.get(), op->n_active, op->rows, stride};
            op->mean.resize(op->n_active);
            op->inv_std.resize(op->n_active);
            for (int64_t t = 0; t < op->n_active; ++t) {
                op->mean[t] = g->mean[active[t]];
                op->inv_std[t] = g->inv_std[active[t]];
            }
            op->view_snp = active;
        }
        const int64_t R = op->n_active;
        if (identity && (int64_t)g->code_counts.size() != 4 * g->n_snps)
            fail(CS_ERR_INVALID_ARGUMENT, "PlinkKinshipOperator: genotype statistics missing");
        // code counts over the operator's samples (trace, mixed-form corrections)
        op->counts.assign(4 * R, 0);
        if (identity) {
            // every sample: the counts the statistics pass kept
            for (int64_t t = 0; t < R; ++t)
                std::copy_n(&g->code_counts[4 * (int64_t)op->view_snp[t]], 4, &op->counts[4 * t]);
        } else if (R) {
            op->d_counts.resize(std::max<int64_t>(1, 4 * R));
            row_code_counts(op->view, op->d_counts.get(), s);
            CS_CUDA(cudaMemcpyAsync(op->counts.data(), op->d_counts.get(), 16 * R,
                                    cudaMemcpyDeviceToHost, s));
        }
        std::vector<double> lut(4 * R), lut_sq(4 * R);
        double total = 0.0;
        CS_CUDA(cudaStreamSynchronize(s));
        for (int64_t t = 0; t < R; ++t) {
            const double mu = op->mean[t], is = op->inv_std[t];
            // kinship_operator.cpp:276-277 decode values; code 01 (missing) -> 0
            lut[4 * t + 0] = (2.0 - mu) * is;
            lut[4 * t + 1] = 0.0;
            lut[4 * t + 2] = (1.0 - mu) * is;
            lut[4 * t + 3] = -mu * is;
            for (int q = 0; q < 4; ++q) lut_sq[4 * t + q] = lut[4 * t + q] * lut[4 * t + q];
            // trace(): sum over observed calls of z^2 (kinship_operator.cpp:306-344)
            total += op->counts[4 * t + 0] * lut_sq[4 * t + 0] +
                     op->counts[4 * t + 2] * lut_sq[4 * t + 2] +
                     op->counts[4 * t + 3] * lut_sq[4 * t + 3];
        }
        op->trace = total / (double)op->num_variants;
        op->d_view_pos.resize(std::max<int64_t>(1, R));
        if (R)
            CS_CUDA(cudaMemcpy(op->d_view_pos.get(), op->view_pos.data(), 4 * R,
                               cudaMemcpyHostToDevice));
        op->d_lut.resize(std::max<int64_t>(1, 4 * R));
        op->d_lut_sq.resize(std::max<int64_t>(1, 4 * R));
        op->d_mean.resize(std::max<int64_t>(1, R));
        op->d_inv_std.resize(std::max<int64_t>(1, R));
        if (R) {
            CS_CUDA(cudaMemcpy(op->d_lut.get(), lut.data(), 32 * R, cudaMemcpyHostToDevice));
            CS_CUDA(cudaMemcpy(op->d_lut_sq.get(), lut_sq.data(), 32 * R, cudaMemcpyHostToDevice));
            CS_CUDA(cudaMemcpy(op->d_mean.get(), op->mean.data(), 8 * R, cudaMemcpyHostToDevice));
            CS_CUDA(cudaMemcpy(op->d_inv_std.get(), op->inv_std.data(), 8 * R, cudaMemcpyHostToDevice));
        }
    } catch (...) {
        delete op;
        throw;
    }
    return op;
}

// FP64 form: U = Z^T X (pass over rows), Y = Z U / M (pass over samples).
static void kinship_apply_fp64(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                               int64_t ldy, cudaStream_t s) {
    const int64_t R = op->n_active;
    const double scale = 1.0 / (double)op->num_variants;
    if (R == 0) {
        // every selected variant is monomorphic: K = 0
        CS_CUDA(cudaMemset2DAsync(Y, ldy * 8, 0, k * 8, op->rows, s));
        return;
    }
    op->buf_u.resize(R * k);
    decode_gemm_rows_fp64(op->view, op->d_lut.get(), X, ldx, k, op->buf_u.get(), k, op->ws, s);
    decode_gemm_samples_fp64(op->view, op->d_lut.get(), op->buf_u.get(), k, k, Y, ldy, scale,
                             op->ws, s);
}

void kinship_apply_rowmajor(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                            int64_t ldy, int precision, cudaStream_t s) {
    if (k <= 0) return;
    if (precision == CS_PRECISION_MIXED)
        kinship_apply_mixed(op, X, ldx, k, Y, ldy, s);
    else if (precision == CS_PRECISION_FP64)
        kinship_apply_fp64(op, X, ldx, k, Y, ldy, s);
    else
        fail(CS_ERR_INVALID_ARGUMENT, "unknown precision mode");
}

// FP32 column-major (ld) <-> FP64 row-major (n x k) around the FP32 entry point.
__global__ void k_f32col_to_f64row(const float* __restrict__ src, int64_t ld, int64_t n,
                                   int64_t k, double* __restrict__ dst) {
    const int64_t total = n * k;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = idx / k, c = idx - i * k;
        dst[idx] = (double)src[i + c * ld];
    }
}

__global__ void k_f64row_to_f32col(const double* __restrict__ src, int64_t n, int64_t k,
                                   float* __restrict__ dst, int64_t ld) {
    const int64_t total = n * k;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = idx / n, i = idx - c * n;
        dst[i + c * ld] = (float)src[i * k + c];
    }
}

// FP32 apply (device pointers): the inputs widened to FP64, the FP64 or mixed apply, the
// result rounded to FP32.  Y may alias X.
void kinship_apply_f32(cs_kinship* op, const float* X, int64_t ldx, int64_t k, float* Y,
                       int64_t ldy, int precision, cudaStream_t s) {
    if (k < 0) fail(CS_ERR_INVALID_ARGUMENT, "negative column count");
    if (k == 0) return;
    if (ldx < op->rows || ldy < op->rows)
        fail(CS_ERR_INVALID_ARGUMENT, "PlinkKinshipOperator::apply: dimension mismatch");
    const int64_t n = op->rows;
    op->buf_x.resize(n * k);
    op->buf_y.resize(n * k);
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n * k + 255) / 256, 32LL * num_sms()));
    {
        prof::Scope ps("f32_to_f64", s, 0.0, 12.0 * n * k);
        k_f32col_to_f64row<<<blocks, 256, 0, s>>>(X, ldx, n, k, op->buf_x.get());
        CS_LAUNCH("f32_to_f64");
    }
    kinship_apply_rowmajor(op, op->buf_x.get(), k, k, op->buf_y.get(), k, precision, s);
    {
        prof::Scope ps("f64_to_f32", s, 0.0, 12.0 * n * k);
        k_f64row_to_f32col<<<blocks, 256, 0, s>>>(op->buf_y.get(), n, k, Y, ldy);
        CS_LAUNCH("f64_to_f32");
    }
}

// Public column-major apply (device pointers): transposes in and out around the kernels.
void kinship_apply_colmajor(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                            int64_t ldy, int precision, cudaStream_t s) {
    if (k < 0) fail(CS_ERR_INVALID_ARGUMENT, "negative column count");
    if (k == 0) return;
    if (ldx < op->rows || ldy < op->rows)
        fail(CS_ERR_INVALID_ARGUMENT, "PlinkKinshipOperator::apply: dimension mismatch");
    const int64_t n = op->rows;
    op->buf_x.resize(n * k);
    op->buf_y.resize(n * k);
    colmajor_to_rowmajor(X, ldx, n, k, op->buf_x.get(), k, s);
    kinship_apply_rowmajor(op, op->buf_x.get(), k, k, op->buf_y.get(), k, precision, s);
    rowmajor_to_colmajor(op->buf_y.get(), k, n, k, Y, ldy, s);
}

// ---------------------------------------------------------------- GenotypeMatrix half-passes
// PlinkReader::multiply_Zt_v / multiply_Z_v (libCosmicCore/src/plink_reader.cpp:241-438, the
// GenotypeMatrix interface of libCosmicCore/src/matrix_adapter.h:40-53) over the operator's
// selection: Z is rows() x numVariants(), standardised with the all-sample statistics, missing
// calls 0, variants with 1/sd == 0 all zero; no 1/M scaling.

// out[pos[t] * ldo + c] = in[t * ldi + c] (view row t -> its selection position), c < k.
__global__ void k_scatter_rows(const double* __restrict__ in, int64_t ldi, int64_t R, int64_t k,
                               const int32_t* __restrict__ pos, double* __restrict__ out,
                               int64_t ldo) {
    const int64_t total = R * k;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = idx / k, c = idx - t * k;
        out[(int64_t)pos[t] * ldo + c] = in[t * ldi + c];
    }
}

// FP64 operand: W[t * k + c] = V[pos[t] * ldv + c]; tensor-core operand (column-major,
// s-scaled): W[c * R + t] = s_t V[pos[t] * ldv + c].
__global__ void k_gather_rows(const double* __restrict__ V, int64_t ldv, int64_t R, int64_t k,
                              const int32_t* __restrict__ pos, const double* __restrict__ s_row,
                              double* __restrict__ W, int colmajor) {
    const int64_t total = R * k;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        if (colmajor) {
            const int64_t c = idx / R, t = idx - c * R;
            W[idx] = s_row[t] * V[(int64_t)pos[t] * ldv + c];
        } else {
            const int64_t t = idx / k, c = idx - t * k;
            W[idx] = V[(int64_t)pos[t] * ldv + c];
        }
    }
}

static unsigned grid_for(int64_t work) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 32LL * num_sms()));
}

// U (numVariants x k, row-major ldu) = Z^T X for X (rows x k, row-major ldx).
void genotype_multiply_zt_rowmajor(cs_kinship* op, const double* X, int64_t ldx, int64_t k,
                                   double* U, int64_t ldu, int precision, cudaStream_t s) {
    const int64_t R = op->n_active, nv = op->num_variants;
    CS_CUDA(cudaMemset2DAsync(U, ldu * 8, 0, k * 8, nv, s));
    if (R == 0 || k == 0) return;
    op->buf_u.resize(R * k);
    if (precision == CS_PRECISION_MIXED)
        mixed_multiply_zt(op, X, ldx, k, op->buf_u.get(), k, s);
    else if (precision == CS_PRECISION_FP64)
        decode_gemm_rows_fp64(op->view, op->d_lut.get(), X, ldx, k, op->buf_u.get(), k, op->ws, s);
    else
        fail(CS_ERR_INVALID_ARGUMENT, "unknown precision mode");
    prof::Scope ps("scatter_rows", s, 0.0, 16.0 * R * k);
    k_scatter_rows<<<grid_for(R * k), 256, 0, s>>>(op->buf_u.get(), k, R, k, op->d_view_pos.get(),
                                                   U, ldu);
    CS_LAUNCH("scatter_rows");
}

// Y (rows x k, row-major ldy) = Z V for V (numVariants x k, row-major ldv).
void genotype_multiply_z_rowmajor(cs_kinship* op, const double* V, int64_t ldv, int64_t k,
                                  double* Y, int64_t ldy, int precision, cudaStream_t s) {
    const int64_t R = op->n_active;
    if (k == 0) return;
    if (R == 0) {
        CS_CUDA(cudaMemset2DAsync(Y, ldy * 8, 0, k * 8, op->rows, s));
        return;
    }
    if (precision != CS_PRECISION_MIXED && precision != CS_PRECISION_FP64)
        fail(CS_ERR_INVALID_ARGUMENT, "unknown precision mode");
    const bool mixed = precision == CS_PRECISION_MIXED;
    op->buf_u.resize(R * k);
    {
        prof::Scope ps("gather_rows", s, 0.0, 16.0 * R * k);
        k_gather_rows<<<grid_for(R * k), 256, 0, s>>>(V, ldv, R, k, op->d_view_pos.get(),
                                                      op->d_inv_std.get(), op->buf_u.get(),
                                                      mixed ? 1 : 0);
        CS_LAUNCH("gather_rows");
    }
    if (mixed)
        mixed_multiply_z(op, op->buf_u.get(), k, Y, ldy, s);
    else
        decode_gemm_samples_fp64(op->view, op->d_lut.get(), op->buf_u.get(), k, k, Y, ldy, 1.0,
                                 op->ws, s);
}

// Column-major public forms (device pointers): transposes around the row-major passes.
void genotype_multiply_zt(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* U,
                          int64_t ldu, int precision, cudaStream_t s) {
    if (k < 0) fail(CS_ERR_INVALID_ARGUMENT, "negative column count");
    if (ldx < op->rows || ldu < op->num_variants)
        fail(CS_ERR_INVALID_ARGUMENT, "Dimension mismatch in multiply_Zt_v");
    if (k == 0) return;
    const int64_t n = op->rows, nv = op->num_variants;
    op->buf_x.resize(n * k);
    op->buf_y.resize(nv * k);
    colmajor_to_rowmajor(X, ldx, n, k, op->buf_x.get(), k, s);
    genotype_multiply_zt_rowmajor(op, op->buf_x.get(), k, k, op->buf_y.get(), k, precision, s);
    rowmajor_to_colmajor(op->buf_y.get(), k, nv, k, U, ldu, s);
}

void genotype_multiply_z(cs_kinship* op, const double* V, int64_t ldv, int64_t k, double* Y,
                         int64_t ldy, int precision, cudaStream_t s) {
    if (k < 0) fail(CS_ERR_INVALID_ARGUMENT, "negative column count");
    if (ldv < op->num_variants || ldy < op->rows)
        fail(CS_ERR_INVALID_ARGUMENT, "Dimension mismatch in multiply_Z_v");
    if (k == 0) return;
    const int64_t n = op->rows, nv = op->num_variants;
    op->buf_x.resize(nv * k);
    op->buf_y.resize(n * k);
    colmajor_to_rowmajor(V, ldv, nv, k, op->buf_x.get(), k, s);
    genotype_multiply_z_rowmajor(op, op->buf_x.get(), k, k, op->buf_y.get(), k, precision, s);
    rowmajor_to_colmajor(op->buf_y.get(), k, n, k, Y, ldy, s);
}

void kinship_diagonal(cs_kinship* op, double* diag_host) {
    const int64_t n = op->rows, R = op->n_active;
    if (R == 0) {
        std::fill(diag_host, diag_host + n, 0.0);
        return;
    }
    cudaStream_t s = 0;
    DeviceBuffer<double> ones, d;
    ones.resize(R);
    d.resize(n);
    std::vector<double> h(R, 1.0);
    CS_CUDA(cudaMemcpy(ones.get(), h.data(), 8 * R, cudaMemcpyHostToDevice));
    decode_gemm_samples_fp64(op->view, op->d_lut_sq.get(), ones.get(), 1, 1, d.get(), 1,
                             1.0 / (double)op->num_variants, op->ws, s);
    CS_CUDA(cudaMemcpy(diag_host, d.get(), 8 * n, cudaMemcpyDeviceToHost));
}

}  // namespace cs
