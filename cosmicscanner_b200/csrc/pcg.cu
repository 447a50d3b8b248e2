// Multi-right-hand-side preconditioned CG on the mixed-model covariance
// V = vg * Zr K Zr^T + vpe * Zr Zr^T + ve * I, and the record <-> genotype-row maps around
// the kinship operator.
//
// The reference solves one right-hand side at a time (libCosmicCore/src/matrix_free_pcg.h:
// 20-68, driven by libCosmicCore/src/stcg_vce.cpp:117-126), so every CG iteration streams
// the whole packed genotype matrix for one vector.  Here all right-hand sides that share a
// V advance together: one kinship apply per iteration carries every active column (the
// tensor-core operator needs width to be efficient), each column keeps its own alpha/beta
// recurrence, and columns whose residual meets the tolerance are compacted out of the
// block so later applies only carry live columns.  Reductions use a fixed row chunking, so
// a column's arithmetic does not depend on which other columns share the block.
#include <algorithm>
#include <cmath>
#include <utility>

#include "vce_internal.h"

namespace cs {

namespace {

constexpr int kColTile = 32, kRowLanes = 8;

int64_t reduction_chunks(int64_t n) { return std::min<int64_t>(128, std::max<int64_t>(1, (n + 511) / 512)); }

// partial[b * k + c] = sum over rows of chunk b of A[r, c] * B[r, c]
__global__ void k_dot_partial(const double* __restrict__ A, int64_t lda, const double* __restrict__ B,
                              int64_t ldb, int64_t n, int64_t k, int64_t chunk,
                              double* __restrict__ partial) {
    __shared__ double red[kRowLanes][kColTile];
    const int64_t c = (int64_t)blockIdx.y * kColTile + threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * chunk, r1 = min(n, r0 + chunk);
    double acc = 0.0;
    if (c < k)
        for (int64_t r = r0 + threadIdx.y; r < r1; r += kRowLanes) acc += A[r * lda + c] * B[r * ldb + c];
    red[threadIdx.y][threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.y == 0 && c < k) {
        double s = red[0][threadIdx.x];
        for (int q = 1; q < kRowLanes; ++q) s += red[q][threadIdx.x];
        partial[blockIdx.x * k + c] = s;
    }
}

__global__ void k_sum_partials(const double* __restrict__ partial, int64_t nb, int64_t k,
                               double* __restrict__ out) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= k) return;
    double s = 0.0;
    for (int64_t b = 0; b < nb; ++b) s += partial[b * k + c];
    out[c] = s;
}

// alpha_c = rsold_c / (p . Ap)_c
__global__ void k_alpha(const double* __restrict__ partial, int64_t nb, int64_t k,
                        const double* __restrict__ rsold, double* __restrict__ alpha) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= k) return;
    double s = 0.0;
    for (int64_t b = 0; b < nb; ++b) s += partial[b * k + c];
    alpha[c] = rsold[c] / s;
}

// x += alpha p, r -= alpha Ap; partial sums of r.r and r.z with z = r / diag
__global__ void k_cg_update(double* __restrict__ X, int64_t ldx, const int32_t* __restrict__ map,
                            const double* __restrict__ P, const double* __restrict__ AP,
                            double* __restrict__ R, int64_t ld, int64_t n, int64_t k, int64_t chunk,
                            const double* __restrict__ alpha, double diag,
                            double* __restrict__ part_rr, double* __restrict__ part_rz) {
    __shared__ double red_a[kRowLanes][kColTile], red_b[kRowLanes][kColTile];
    const int64_t c = (int64_t)blockIdx.y * kColTile + threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * chunk, r1 = min(n, r0 + chunk);
    double rr = 0.0, rz = 0.0;
    if (c < k) {
        const double a = alpha[c];
        const int64_t xc = map[c];
        for (int64_t r = r0 + threadIdx.y; r < r1; r += kRowLanes) {
            X[r * ldx + xc] += a * P[r * ld + c];
            const double rv = R[r * ld + c] - a * AP[r * ld + c];
            R[r * ld + c] = rv;
            rr += rv * rv;
            rz += rv * (rv / diag);
        }
    }
    red_a[threadIdx.y][threadIdx.x] = rr;
    red_b[threadIdx.y][threadIdx.x] = rz;
    __syncthreads();
    if (threadIdx.y == 0 && c < k) {
        double sa = red_a[0][threadIdx.x], sb = red_b[0][threadIdx.x];
        for (int q = 1; q < kRowLanes; ++q) {
            sa += red_a[q][threadIdx.x];
            sb += red_b[q][threadIdx.x];
        }
        part_rr[blockIdx.x * k + c] = sa;
        part_rz[blockIdx.x * k + c] = sb;
    }
}

// rr_c, rz_c; beta_c = rz_c / rsold_c; rsold_c = rz_c
__global__ void k_beta(const double* __restrict__ part_rr, const double* __restrict__ part_rz,
                       int64_t nb, int64_t k, double* __restrict__ rsold, double* __restrict__ beta,
                       double* __restrict__ rr_out) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= k) return;
    double a = 0.0, b = 0.0;
    for (int64_t q = 0; q < nb; ++q) {
        a += part_rr[q * k + c];
        b += part_rz[q * k + c];
    }
    rr_out[c] = a;
    beta[c] = b / rsold[c];
    rsold[c] = b;
}

// p = z + beta p
__global__ void k_direction_z(double* __restrict__ P, const double* __restrict__ Z, int64_t ld,
                              int64_t n, int64_t k, const double* __restrict__ beta) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        P[r * ld + c] = Z[r * ld + c] + beta[c] * P[r * ld + c];
    }
}

// p = r / diag + beta p
__global__ void k_direction(double* __restrict__ P, const double* __restrict__ R, int64_t ld,
                            int64_t n, int64_t k, double diag, const double* __restrict__ beta) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        P[r * ld + c] = R[r * ld + c] / diag + beta[c] * P[r * ld + c];
    }
}

// R = B (columns idx), P = B / diag
__global__ void k_cg_init(const double* __restrict__ B, int64_t ldb, const int32_t* __restrict__ idx,
                          double* __restrict__ R, double* __restrict__ P, int64_t ld, int64_t n,
                          int64_t k, double diag) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        const double b = B[r * ldb + idx[c]];
        R[r * ld + c] = b;
        P[r * ld + c] = b / diag;
    }
}

__global__ void k_gather_cols(const double* __restrict__ src, int64_t lds, int64_t n,
                              const int32_t* __restrict__ idx, int64_t k, double* __restrict__ dst,
                              int64_t ldd) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        dst[r * ldd + c] = src[r * lds + idx[c]];
    }
}

// U[i, c] = sum of the records of row i, in record order (stcg_vce.cpp:64-70)
__global__ void k_records_to_rows(const double* __restrict__ V, int64_t ldv, int64_t k,
                                  const int32_t* __restrict__ row_ptr,
                                  const int32_t* __restrict__ row_recs, int64_t n_rows,
                                  double* __restrict__ U, int64_t ldu) {
    const int64_t total = n_rows * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / k, c = e - i * k;
        double s = 0.0;
        for (int32_t q = row_ptr[i]; q < row_ptr[i + 1]; ++q) s += V[(int64_t)row_recs[q] * ldv + c];
        U[i * ldu + c] = s;
    }
}

// out = vg * fac * KU[row(r)] + vpe * U[row(r)] + ve * V[r]   (stcg_vce.cpp:103-115)
__global__ void k_combine(double* __restrict__ out, int64_t ldo, const double* __restrict__ V,
                          int64_t ldv, const double* __restrict__ KU, int64_t ldk,
                          const double* __restrict__ U, int64_t ldu,
                          const int32_t* __restrict__ rec_to_row, int64_t n_rec, int64_t k,
                          double vg, double fac, double vpe, double ve, int with_pe) {
    const int64_t total = n_rec * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        const int64_t i = rec_to_row ? rec_to_row[r] : r;
        double g = 0.0, pe = 0.0;
        if (i >= 0) {
            g = KU[i * ldk + c];
            if (fac != 1.0) g *= fac;
            pe = U[i * ldu + c];
        }
        double o = vg * g;
        if (with_pe) o += vpe * pe;
        out[r * ldo + c] = o + ve * V[r * ldv + c];
    }
}

// g_out = fac * KU[row(r)], pe_out = U[row(r)]   (stcg_vce.cpp:89-101)
__global__ void k_scatter_rows(double* __restrict__ g_out, int64_t ldg, double* __restrict__ pe_out,
                               int64_t ldp, const double* __restrict__ KU, int64_t ldk,
                               const double* __restrict__ U, int64_t ldu,
                               const int32_t* __restrict__ rec_to_row, int64_t n_rec, int64_t k,
                               double fac) {
    const int64_t total = n_rec * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        const int64_t i = rec_to_row ? rec_to_row[r] : r;
        double g = 0.0, pe = 0.0;
        if (i >= 0) {
            g = KU[i * ldk + c];
            if (fac != 1.0) g *= fac;
            pe = U[i * ldu + c];
        }
        g_out[r * ldg + c] = g;
        if (pe_out) pe_out[r * ldp + c] = pe;
    }
}

__global__ void k_scale_copy(const double* __restrict__ src, int64_t lds, int64_t n, int64_t k,
                             double fac, double* __restrict__ dst, int64_t ldd) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        dst[r * ldd + c] = fac != 1.0 ? src[r * lds + c] * fac : src[r * lds + c];
    }
}

unsigned grid_for(int64_t total) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 16LL * num_sms()));
}

void swap_buffers(DeviceBuffer<double>& a, DeviceBuffer<double>& b) {
    std::swap(a.ptr, b.ptr);
    std::swap(a.count, b.count);
}

}  // namespace

// ---------------------------------------------------------------- record map
void RecordMap::build(const int32_t* rec_to_row_host, int64_t nrec, int64_t nrows) {
    n_rec = nrec;
    n_rows = nrows;
    identity = rec_to_row_host == nullptr;
    rec_to_row.clear();
    if (identity) {
        if (nrec != nrows)
            fail(CS_ERR_INVALID_ARGUMENT, "records without a record map must equal the operator rows");
        return;
    }
    rec_to_row.assign(rec_to_row_host, rec_to_row_host + nrec);
    std::vector<int32_t> ptr(nrows + 1, 0), recs;
    for (int64_t r = 0; r < nrec; ++r) {
        const int32_t i = rec_to_row[r];
        if (i < -1 || i >= nrows)
            fail(CS_ERR_INVALID_ARGUMENT, "record maps to a genotype row out of range");
        if (i >= 0) ++ptr[i + 1];
    }
    for (int64_t i = 0; i < nrows; ++i) ptr[i + 1] += ptr[i];
    recs.resize(ptr[nrows]);
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t r = 0; r < nrec; ++r)
        if (rec_to_row[r] >= 0) recs[fill[rec_to_row[r]]++] = (int32_t)r;
    d_rec_to_row.resize(std::max<int64_t>(1, nrec));
    d_row_ptr.resize(nrows + 1);
    d_row_recs.resize(std::max<size_t>(1, recs.size()));
    CS_CUDA(cudaMemcpy(d_rec_to_row.get(), rec_to_row.data(), 4 * nrec, cudaMemcpyHostToDevice));
    CS_CUDA(cudaMemcpy(d_row_ptr.get(), ptr.data(), 4 * (nrows + 1), cudaMemcpyHostToDevice));
    if (!recs.empty())
        CS_CUDA(cudaMemcpy(d_row_recs.get(), recs.data(), 4 * recs.size(), cudaMemcpyHostToDevice));
}

// ---------------------------------------------------------------- V operator
const double* VOperator::gather(const double* in, int64_t ldi, int64_t k, cudaStream_t s) {
    if (rm->identity) return in;
    u.resize(std::max<int64_t>(1, rm->n_rows * k));
    prof::Scope ps("records_to_rows", s, 0.0, 8.0 * (double)(rm->n_rec + rm->n_rows) * k);
    k_records_to_rows<<<grid_for(rm->n_rows * k), 256, 0, s>>>(
        in, ldi, k, rm->d_row_ptr.get(), rm->d_row_recs.get(), rm->n_rows, u.get(), k);
    CS_LAUNCH("records_to_rows");
    return u.get();
}

void VOperator::apply(const double* in, int64_t ldi, int64_t k, double* out, int64_t ldo,
                      cudaStream_t s) {
    if (k <= 0) return;
    const double* U = gather(in, ldi, k, s);
    const int64_t ldu = rm->identity ? ldi : k;
    ku.resize(std::max<int64_t>(1, rm->n_rows * k));
    kinship_apply_rowmajor(op, U, ldu, k, ku.get(), k, precision, s);
    ++applies;
    apply_cols += k;
    prof::Scope ps("covariance_combine", s, 0.0, 8.0 * 3.0 * (double)rm->n_rec * k);
    k_combine<<<grid_for(rm->n_rec * k), 256, 0, s>>>(
        out, ldo, in, ldi, ku.get(), k, U, ldu, rm->identity ? nullptr : rm->d_rec_to_row.get(),
        rm->n_rec, k, vg, fac, vpe, ve, with_pe ? 1 : 0);
    CS_LAUNCH("covariance_combine");
}

void VOperator::derivatives(const double* in, int64_t ldi, int64_t k, double* g_out, int64_t ldg,
                            double* pe_out, int64_t ldp, cudaStream_t s) {
    if (k <= 0) return;
    const double* U = gather(in, ldi, k, s);
    const int64_t ldu = rm->identity ? ldi : k;
    ku.resize(std::max<int64_t>(1, rm->n_rows * k));
    kinship_apply_rowmajor(op, U, ldu, k, ku.get(), k, precision, s);
    ++applies;
    apply_cols += k;
    prof::Scope ps("records_scatter", s, 0.0, 8.0 * 2.0 * (double)rm->n_rec * k);
    k_scatter_rows<<<grid_for(rm->n_rec * k), 256, 0, s>>>(
        g_out, ldg, pe_out, ldp, ku.get(), k, U, ldu,
        rm->identity ? nullptr : rm->d_rec_to_row.get(), rm->n_rec, k, fac);
    CS_LAUNCH("records_scatter");
}

void VOperator::genetic_rows(const double* in, int64_t ldi, int64_t k, double* rows_out,
                             int64_t ldo, double* zt_out, int64_t ldz, cudaStream_t s) {
    if (k <= 0) return;
    const double* U = gather(in, ldi, k, s);
    const int64_t ldu = rm->identity ? ldi : k;
    ku.resize(std::max<int64_t>(1, rm->n_rows * k));
    kinship_apply_rowmajor(op, U, ldu, k, ku.get(), k, precision, s);
    ++applies;
    apply_cols += k;
    k_scale_copy<<<grid_for(rm->n_rows * k), 256, 0, s>>>(ku.get(), k, rm->n_rows, k, fac,
                                                          rows_out, ldo);
    CS_LAUNCH("scale_copy");
    if (zt_out) {
        k_scale_copy<<<grid_for(rm->n_rows * k), 256, 0, s>>>(U, ldu, rm->n_rows, k, 1.0, zt_out, ldz);
        CS_LAUNCH("scale_copy");
    }
}

// ---------------------------------------------------------------- dots
void column_dots(const double* A, int64_t lda, const double* B, int64_t ldb, int64_t n, int64_t k,
                 double* out_host, PcgWorkspace& ws, cudaStream_t s) {
    if (k <= 0) return;
    const int64_t nb = reduction_chunks(n), chunk = (n + nb - 1) / nb;
    ws.partial_a.resize(nb * k);
    ws.rr.resize(std::max<int64_t>(k, 1));
    {
        prof::Scope ps("column_dots", s, 2.0 * n * k, 16.0 * n * k);
        k_dot_partial<<<dim3((unsigned)nb, (unsigned)((k + kColTile - 1) / kColTile)),
                        dim3(kColTile, kRowLanes), 0, s>>>(A, lda, B, ldb, n, k, chunk,
                                                            ws.partial_a.get());
        CS_LAUNCH("column_dots");
    }
    k_sum_partials<<<(unsigned)((k + 127) / 128), 128, 0, s>>>(ws.partial_a.get(), nb, k, ws.rr.get());
    CS_LAUNCH("sum_partials");
    CS_CUDA(cudaMemcpyAsync(out_host, ws.rr.get(), 8 * k, cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------- low-rank preconditioner
void LowRankPreconditioner::set_components(double vg, double ve, cudaStream_t s) {
    base = 1.0 / std::max(1e-300, vg * r0 + ve);
    std::vector<double> h(std::max<int64_t>(1, r));
    for (int64_t j = 0; j < r; ++j) h[j] = 1.0 / (vg * lambda[j] + ve) - base;
    c.resize(std::max<int64_t>(1, r));
    CS_CUDA(cudaMemcpyAsync(c.get(), h.data(), 8 * r, cudaMemcpyHostToDevice, s));
    CS_CUDA(cudaStreamSynchronize(s));  // h is a local
}

void LowRankPreconditioner::apply(const double* R, int64_t ldr, int64_t k, double* Z, int64_t ldz,
                                  cudaStream_t s) {
    if (k <= 0) return;
    cublasHandle_t blas = shared_blas();
    CS_BLAS(cublasSetStream(blas, s));
    T.resize(std::max<int64_t>(1, r * k));
    prof::Scope ps("lowrank_precondition", s, 4.0 * (double)n * r * k, 8.0 * (2.0 * n * k + n * r));
    // column-major views: R^T (k x n, ld ldr), U^T (r x n, ld r)
    const double one = 1.0, zero = 0.0;
    // T^T (k x r) = R^T U
    CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)k, (int)r, (int)n, &one, R, (int)ldr,
                        U.get(), (int)r, &zero, T.get(), (int)k));
    // T^T[:, j] *= c_j
    CS_BLAS(cublasDdgmm(blas, CUBLAS_SIDE_RIGHT, (int)k, (int)r, T.get(), (int)k, c.get(), 1,
                        T.get(), (int)k));
    // Z^T = base R^T + T^T U^T
    CS_CUDA(cudaMemcpy2DAsync(Z, 8 * ldz, R, 8 * ldr, 8 * k, n, cudaMemcpyDeviceToDevice, s));
    CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)k, (int)n, (int)r, &one, T.get(),
                        (int)k, U.get(), (int)r, &base, Z, (int)ldz));
}

// ---------------------------------------------------------------- block PCG
void pcg_solve_block(VOperator& A, double diag, const double* B, int64_t ldb, int64_t k,
                     double* X, int64_t ldx, double tol, bool relative, int max_iter,
                     PcgWorkspace& ws, PcgStats& st, cudaStream_t s, LowRankPreconditioner* M) {
    st.iterations.assign(k, 0);
    st.sweeps = 0;  // counts of this solve only
    st.column_iterations = 0;
    if (k <= 0) return;
    const int64_t n = A.rm->n_rec;
    CS_CUDA(cudaMemset2DAsync(X, ldx * 8, 0, k * 8, n, s));
    const int64_t nb = reduction_chunks(n), chunk = (n + nb - 1) / nb;
    ws.R.resize(n * k);
    ws.P.resize(n * k);
    ws.AP.resize(n * k);
    ws.T.resize(n * k);
    ws.partial_a.resize(nb * k);
    ws.partial_b.resize(nb * k);
    for (auto* b : {&ws.alpha, &ws.beta, &ws.rsold, &ws.rr, &ws.rz}) b->resize(k);
    ws.map.resize(k);
    ws.idx.resize(k);
    std::vector<int32_t> map(k);
    for (int64_t c = 0; c < k; ++c) map[c] = (int32_t)c;
    CS_CUDA(cudaMemcpyAsync(ws.idx.get(), map.data(), 4 * k, cudaMemcpyHostToDevice, s));
    k_cg_init<<<grid_for(n * k), 256, 0, s>>>(B, ldb, ws.idx.get(), ws.R.get(), ws.P.get(), k, n, k,
                                              diag);
    CS_LAUNCH("cg_init");
    if (M) {
        ws.Zp.resize(n * k);
        M->apply(ws.R.get(), k, k, ws.P.get(), k, s);  // p0 = z0 = M^-1 r0
    }
    // ||b||^2 and rsold = r . z
    std::vector<double> rr(k), rs(k);
    column_dots(ws.R.get(), k, ws.R.get(), k, n, k, rr.data(), ws, s);
    column_dots(ws.R.get(), k, ws.P.get(), k, n, k, rs.data(), ws, s);
    std::vector<double> tol_c(k);
    for (int64_t c = 0; c < k; ++c) tol_c[c] = relative ? tol * std::sqrt(rr[c]) : tol;
    // columns already solved by x = 0 (matrix_free_pcg.h:32)
    std::vector<int32_t> live;
    for (int64_t c = 0; c < k; ++c)
        if (!(std::sqrt(rr[c]) < 1e-20)) live.push_back((int32_t)c);
    int64_t ka = k;
    auto compact = [&](const std::vector<int32_t>& keep_pos, std::vector<double>& rs_host) {
        const int64_t kn = (int64_t)keep_pos.size();
        if (kn == 0) return;
        CS_CUDA(cudaMemcpyAsync(ws.idx.get(), keep_pos.data(), 4 * kn, cudaMemcpyHostToDevice, s));
        k_gather_cols<<<grid_for(n * kn), 256, 0, s>>>(ws.R.get(), ka, n, ws.idx.get(), kn, ws.T.get(), kn);
        CS_LAUNCH("gather_cols");
        swap_buffers(ws.R, ws.T);
        k_gather_cols<<<grid_for(n * kn), 256, 0, s>>>(ws.P.get(), ka, n, ws.idx.get(), kn, ws.T.get(), kn);
        CS_LAUNCH("gather_cols");
        swap_buffers(ws.P, ws.T);
        std::vector<double> r2(kn);
        for (int64_t j = 0; j < kn; ++j) r2[j] = rs_host[keep_pos[j]];
        rs_host = r2;
        CS_CUDA(cudaMemcpyAsync(ws.rsold.get(), rs_host.data(), 8 * kn, cudaMemcpyHostToDevice, s));
        std::vector<int32_t> m2(kn);
        for (int64_t j = 0; j < kn; ++j) m2[j] = map[keep_pos[j]];
        map = m2;
        ka = kn;
    };
    if ((int64_t)live.size() < k) {
        if (live.empty()) return;
        compact(live, rs);
    } else {
        CS_CUDA(cudaMemcpyAsync(ws.rsold.get(), rs.data(), 8 * k, cudaMemcpyHostToDevice, s));
    }
    CS_CUDA(cudaMemcpyAsync(ws.map.get(), map.data(), 4 * ka, cudaMemcpyHostToDevice, s));
    std::vector<double> rr_h(k), rs_h(k);
    for (int it = 0; it < max_iter && ka > 0; ++it) {
        A.apply(ws.P.get(), ka, ka, ws.AP.get(), ka, s);
        ++st.sweeps;
        st.column_iterations += ka;
        const dim3 grid((unsigned)nb, (unsigned)((ka + kColTile - 1) / kColTile));
        const dim3 block(kColTile, kRowLanes);
        {
            prof::Scope ps("cg_step", s, 6.0 * n * ka, 8.0 * 7.0 * n * ka);
            k_dot_partial<<<grid, block, 0, s>>>(ws.P.get(), ka, ws.AP.get(), ka, n, ka, chunk,
                                                 ws.partial_a.get());
            CS_LAUNCH("cg_dot");
            k_alpha<<<(unsigned)((ka + 127) / 128), 128, 0, s>>>(ws.partial_a.get(), nb, ka,
                                                                 ws.rsold.get(), ws.alpha.get());
            CS_LAUNCH("cg_alpha");
            k_cg_update<<<grid, block, 0, s>>>(X, ldx, ws.map.get(), ws.P.get(), ws.AP.get(),
                                               ws.R.get(), ka, n, ka, chunk, ws.alpha.get(), diag,
                                               ws.partial_a.get(), ws.partial_b.get());
            CS_LAUNCH("cg_update");
            if (M) {
                // z = M^-1 r and r . z in place of the scalar form's r . r / diag
                M->apply(ws.R.get(), ka, ka, ws.Zp.get(), ka, s);
                k_dot_partial<<<grid, block, 0, s>>>(ws.R.get(), ka, ws.Zp.get(), ka, n, ka, chunk,
                                                     ws.partial_b.get());
                CS_LAUNCH("cg_rz");
            }
            k_beta<<<(unsigned)((ka + 127) / 128), 128, 0, s>>>(ws.partial_a.get(), ws.partial_b.get(),
                                                                nb, ka, ws.rsold.get(), ws.beta.get(),
                                                                ws.rr.get());
            CS_LAUNCH("cg_beta");
        }
        CS_CUDA(cudaMemcpyAsync(rr_h.data(), ws.rr.get(), 8 * ka, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaStreamSynchronize(s));
        std::vector<int32_t> keep_pos;
        for (int64_t c = 0; c < ka; ++c) {
            st.iterations[map[c]] = it + 1;
            if (!(std::sqrt(rr_h[c]) < tol_c[map[c]])) keep_pos.push_back((int32_t)c);
        }
        if (keep_pos.empty()) break;
        {
            prof::Scope ps("cg_direction", s, 2.0 * n * ka, 24.0 * n * ka);
            if (M)
                k_direction_z<<<grid_for(n * ka), 256, 0, s>>>(ws.P.get(), ws.Zp.get(), ka, n, ka,
                                                               ws.beta.get());
            else
                k_direction<<<grid_for(n * ka), 256, 0, s>>>(ws.P.get(), ws.R.get(), ka, n, ka,
                                                             diag, ws.beta.get());
            CS_LAUNCH("cg_direction");
        }
        if ((int64_t)keep_pos.size() < ka) {
            CS_CUDA(cudaMemcpyAsync(rs_h.data(), ws.rsold.get(), 8 * ka, cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaStreamSynchronize(s));
            compact(keep_pos, rs_h);
            CS_CUDA(cudaMemcpyAsync(ws.map.get(), map.data(), 4 * ka, cudaMemcpyHostToDevice, s));
        }
    }
    CS_CUDA(cudaStreamSynchronize(s));
}

}  // namespace cs
