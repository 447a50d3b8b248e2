// Repeatability GWAS scan after the STCG null model, on the GPU
// (RepeatabilityModel::scanSTCG's scan_stcg_with_grm, src/models/repeatability_scan_stcg.cpp:
// 42-140).
//
// The reference fits the null with a dense q x q subject GRM G (q kept subjects):
// K = vg G + vpe I, M = K^-1 + D / ve (D = records per subject), and applies
// V^-1 v = v / ve - Z M^-1 Z^T v / ve^2 once per SNP (a q x q LDLT solve each).  Here every
// SNP of a block shares one dense GEMM: with e = d - mean (the record-centred dosage at the
// subject level, missing calls at 0 - mean) and g = Z e on records,
//   score      = e^T (Z^T P y)
//   g^T V^-1 g = e^T D e / ve - (D e)^T M^-1 (D e) / ve^2
//   X^T V^-1 g = W^T e / ve - (M^-1 W)^T (D e) / ve^2,  W = Z^T X
//   g^T V^-1 X = e^T (Z^T V^-1 X)
// so the only O(q^2) work is T = M^-1 (D E) for the block (FP64 GEMM); K^-1 and M^-1 come
// from Cholesky factorisations (cuSOLVER) once per scan.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "linalg_host.h"
#include "vce_internal.h"

namespace cs {

namespace {


unsigned grid_for(int64_t total) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 32LL * num_sms()));
}

// A = a G + b I (q x q, column-major)
__global__ void k_scale_plus_diag(double* __restrict__ A, const double* __restrict__ G, int64_t q,
                                  double a, double b) {
    const int64_t total = q * q;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e % q, c = e / q;
        A[e] = a * G[e] + (r == c ? b : 0.0);
    }
}

// Full symmetric matrix from the lower triangle (potri leaves the upper part untouched),
// plus an optional diagonal term diag[r] * scale.
__global__ void k_symmetrize_lower(double* __restrict__ A, int64_t q, const double* __restrict__ diag,
                                   double scale) {
    const int64_t total = q * q;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e % q, c = e / q;
        if (r < c) A[e] = A[c + r * q];
        if (diag && r == c) A[e] += diag[r] * scale;
    }
}

// Per SNP j of the block (one warp each): record-weighted dosage sum and observed-record
// count over the subjects, then E[:, j] = d - mean and DE[:, j] = D o E[:, j]
// (repeatability_scan_stcg.cpp:110-124).
__global__ void k_stcg_encode(const uint8_t* __restrict__ packed, int64_t stride, int64_t first,
                              int64_t m_b, const int32_t* __restrict__ subject_rows, int64_t q,
                              const double* __restrict__ D, double min_maf,
                              double* __restrict__ E, double* __restrict__ DE,
                              double* __restrict__ maf_out, int32_t* __restrict__ pass_out) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= m_b) return;
    const uint8_t* row = packed + (first + warp) * stride;
    double sum = 0.0, valid = 0.0;
    for (int64_t s = lane; s < q; s += 32) {
        const int32_t i = subject_rows[s];
        const int code = (row[i >> 2] >> ((i & 3) * 2)) & 3;
        if (code != 1) {
            const double dos = code == 0 ? 2.0 : (code == 2 ? 1.0 : 0.0);
            sum += D[s] * dos;
            valid += D[s];
        }
    }
    for (int off = 16; off; off >>= 1) {
        sum += __shfl_xor_sync(0xffffffffu, sum, off);
        valid += __shfl_xor_sync(0xffffffffu, valid, off);
    }
    double maf = valid > 0 ? sum / (2.0 * valid) : 0.0;
    if (maf > 0.5) maf = 1.0 - maf;
    const bool pass = valid >= 10.0 && maf >= min_maf;
    const double mean = valid > 0 ? sum / valid : 0.0;
    if (lane == 0) {
        maf_out[warp] = maf;
        pass_out[warp] = pass ? 1 : 0;
    }
    double* e = E + (int64_t)warp * q;
    double* de = DE + (int64_t)warp * q;
    for (int64_t s = lane; s < q; s += 32) {
        const int32_t i = subject_rows[s];
        const int code = (row[i >> 2] >> ((i & 3) * 2)) & 3;
        const double dos = code == 0 ? 2.0 : (code == 2 ? 1.0 : 0.0);  // missing -> 0
        const double v = (code == 1 ? 0.0 : dos) - mean;
        e[s] = v;
        de[s] = D[s] * v;
    }
}

// Per SNP: q1 = e^T D e, q2 = (D e)^T T, score = a^T e (one warp each).
__global__ void k_stcg_quads(const double* __restrict__ E, const double* __restrict__ DE,
                             const double* __restrict__ T, const double* __restrict__ a, int64_t q,
                             int64_t m_b, double* __restrict__ out) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= m_b) return;
    const double* e = E + (int64_t)warp * q;
    const double* de = DE + (int64_t)warp * q;
    const double* t = T + (int64_t)warp * q;
    double q1 = 0.0, q2 = 0.0, sc = 0.0;
    for (int64_t s = lane; s < q; s += 32) {
        q1 += e[s] * de[s];
        q2 += de[s] * t[s];
        sc += a[s] * e[s];
    }
    for (int off = 16; off; off >>= 1) {
        q1 += __shfl_xor_sync(0xffffffffu, q1, off);
        q2 += __shfl_xor_sync(0xffffffffu, q2, off);
        sc += __shfl_xor_sync(0xffffffffu, sc, off);
    }
    if (lane == 0) {
        out[3 * warp] = q1;
        out[3 * warp + 1] = q2;
        out[3 * warp + 2] = sc;
    }
}

// dst (q x k, column-major) = src^T-free product helper: C = A^T B for column-major blocks
void gemm_tn(cublasHandle_t blas, int64_t m, int64_t n, int64_t k, const double* A, int64_t lda,
             const double* B, int64_t ldb, double* C, int64_t ldc, cudaStream_t s) {
    const double one = 1.0, zero = 0.0;
    CS_BLAS(cublasSetStream(blas, s));
    CS_BLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)m, (int)n, (int)k, &one, A, (int)lda,
                        B, (int)ldb, &zero, C, (int)ldc));
}

// In-place inverse of an SPD matrix (q x q, column-major, device) through its Cholesky factor.
void spd_inverse(cusolverDnHandle_t sol, double* A, int64_t q, DeviceBuffer<double>& work,
                 DeviceBuffer<int>& info, const double* add_diag, double scale, cudaStream_t s) {
    CS_SOLVER(cusolverDnSetStream(sol, s));
    int lw1 = 0, lw2 = 0;
    CS_SOLVER(cusolverDnDpotrf_bufferSize(sol, CUBLAS_FILL_MODE_LOWER, (int)q, A, (int)q, &lw1));
    CS_SOLVER(cusolverDnDpotri_bufferSize(sol, CUBLAS_FILL_MODE_LOWER, (int)q, A, (int)q, &lw2));
    work.resize(std::max(1, std::max(lw1, lw2)));
    info.resize(1);
    CS_SOLVER(cusolverDnDpotrf(sol, CUBLAS_FILL_MODE_LOWER, (int)q, A, (int)q, work.get(),
                               std::max(lw1, 1), info.get()));
    int h = 0;
    CS_CUDA(cudaMemcpyAsync(&h, info.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    if (h != 0) fail(CS_ERR_NUMERIC, "scanSTCG: matrix is not positive definite");
    CS_SOLVER(cusolverDnDpotri(sol, CUBLAS_FILL_MODE_LOWER, (int)q, A, (int)q, work.get(),
                               std::max(lw2, 1), info.get()));
    k_symmetrize_lower<<<grid_for(q * q), 256, 0, s>>>(A, q, add_diag, scale);
    CS_LAUNCH("symmetrize");
}

}  // namespace

void stcg_scan(const cs_genotypes* g, const double* G, int64_t q, const int32_t* subject_rows,
               const int32_t* obs_to_subject, int64_t n_obs, const double* y, const double* X,
               int64_t p, double vg, double vpe, double ve, double min_maf, int64_t snp_begin,
               int64_t snp_end, double* beta, double* se, double* pvalue, double* log10p,
               double* maf, int32_t* tested) {
    if (!g || !G || !subject_rows || !obs_to_subject || !y || q <= 0 || n_obs <= 0 || p < 0 ||
        (p > 0 && !X))
        fail(CS_ERR_INVALID_ARGUMENT, "scanSTCG: bad arguments");
    if (snp_begin < 0 || snp_end > g->n_snps || snp_begin > snp_end)
        fail(CS_ERR_INVALID_ARGUMENT, "scanSTCG: SNP window out of range");
    if (!(ve > 0.0)) fail(CS_ERR_INVALID_ARGUMENT, "scanSTCG: V(e) must be positive");
    for (int64_t s = 0; s < q; ++s)
        if (subject_rows[s] < 0 || subject_rows[s] >= g->n_samples)
            fail(CS_ERR_INVALID_ARGUMENT, "scanSTCG: subject row out of range");
    for (int64_t i = 0; i < n_obs; ++i)
        if (obs_to_subject[i] < 0 || obs_to_subject[i] >= q)
            fail(CS_ERR_INVALID_ARGUMENT, "scanSTCG: record maps to no subject");
    cudaStream_t s = 0;
    cublasHandle_t blas = shared_blas();
    cusolverDnHandle_t sol = shared_solver();
    // ---- null model in the subject space (repeatability_scan_stcg.cpp:47-97)
    std::vector<double> D(q, 0.0);
    for (int64_t i = 0; i < n_obs; ++i) D[obs_to_subject[i]] += 1.0;
    DeviceBuffer<double> dG, dK, dD, work, tmp;
    DeviceBuffer<int> info;
    dK.resize(q * q);
    dD.resize(q);
    {
        dG.resize(q * q);
        CS_CUDA(cudaMemcpyAsync(dG.get(), G, 8 * q * q, cudaMemcpyHostToDevice, s));
        CS_CUDA(cudaMemcpyAsync(dD.get(), D.data(), 8 * q, cudaMemcpyHostToDevice, s));
        k_scale_plus_diag<<<grid_for(q * q), 256, 0, s>>>(dK.get(), dG.get(), q, vg, vpe);
        CS_LAUNCH("stcg_k");
        dG.release();
    }
    // K^-1, then M = K^-1 + D / ve and M^-1 (in place)
    spd_inverse(sol, dK.get(), q, work, info, dD.get(), 1.0 / ve, s);
    spd_inverse(sol, dK.get(), q, work, info, nullptr, 0.0, s);
    double* Minv = dK.get();
    // woodbury(v) = v / ve - Z M^-1 Z^T v / ve^2 for the columns [y | X]
    const int64_t nc = 1 + p;
    std::vector<double> ztv(q * nc, 0.0);
    for (int64_t i = 0; i < n_obs; ++i) {
        const int32_t sj = obs_to_subject[i];
        ztv[sj] += y[i];
        for (int64_t a = 0; a < p; ++a) ztv[sj + (1 + a) * q] += X[i + a * n_obs];
    }
    tmp.resize(2 * q * std::max<int64_t>(nc, p + 1));
    DeviceBuffer<double> dz;
    dz.resize(q * nc);
    CS_CUDA(cudaMemcpyAsync(dz.get(), ztv.data(), 8 * q * nc, cudaMemcpyHostToDevice, s));
    {
        const double one = 1.0, zero = 0.0;
        CS_BLAS(cublasSetStream(blas, s));
        CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)q, (int)nc, (int)q, &one, Minv,
                            (int)q, dz.get(), (int)q, &zero, tmp.get(), (int)q));
    }
    std::vector<double> mz(q * nc);
    CS_CUDA(cudaMemcpyAsync(mz.data(), tmp.get(), 8 * q * nc, cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    auto woodbury = [&](const double* v, const double* mzc, double* out) {
        for (int64_t i = 0; i < n_obs; ++i) out[i] = v[i] / ve - mzc[obs_to_subject[i]] / (ve * ve);
    };
    std::vector<double> Vy(n_obs), VX(n_obs * p);
    woodbury(y, mz.data(), Vy.data());
    for (int64_t a = 0; a < p; ++a) woodbury(X + a * n_obs, mz.data() + (1 + a) * q, VX.data() + a * n_obs);
    std::vector<double> XtVX(p * p, 0.0), Xty(p, 0.0);
    for (int64_t a = 0; a < p; ++a) {
        for (int64_t b = 0; b < p; ++b) {
            double acc = 0.0;
            for (int64_t i = 0; i < n_obs; ++i) acc += X[i + a * n_obs] * VX[i + b * n_obs];
            XtVX[a + b * p] = acc;
        }
        double acc = 0.0;
        for (int64_t i = 0; i < n_obs; ++i) acc += X[i + a * n_obs] * Vy[i];
        Xty[a] = acc;
    }
    std::vector<double> L, Dl, inv, bhat(p, 0.0);
    bool xok = p == 0 || la::ldlt(XtVX, (int)p, L, Dl);
    if (p > 0 && xok) {
        inv = la::ldlt_inverse(L, Dl, (int)p);
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b) bhat[a] += inv[a + b * p] * Xty[b];
    }
    if (p > 0 && !xok) fail(CS_ERR_NUMERIC, "scanSTCG: X' V^-1 X is singular");
    std::vector<double> resid(n_obs);
    for (int64_t i = 0; i < n_obs; ++i) {
        double fit = 0.0;
        for (int64_t a = 0; a < p; ++a) fit += X[i + a * n_obs] * bhat[a];
        resid[i] = y[i] - fit;
    }
    // P_y = woodbury(resid); a = Z^T P_y; W = Z^T X; B = Z^T V^-1 X; C = M^-1 W
    std::vector<double> ztr(q, 0.0);
    for (int64_t i = 0; i < n_obs; ++i) ztr[obs_to_subject[i]] += resid[i];
    CS_CUDA(cudaMemcpyAsync(dz.get(), ztr.data(), 8 * q, cudaMemcpyHostToDevice, s));
    {
        const double one = 1.0, zero = 0.0;
        CS_BLAS(cublasDgemv(blas, CUBLAS_OP_N, (int)q, (int)q, &one, Minv, (int)q, dz.get(), 1,
                            &zero, tmp.get(), 1));
    }
    std::vector<double> mr(q);
    CS_CUDA(cudaMemcpyAsync(mr.data(), tmp.get(), 8 * q, cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    std::vector<double> Py(n_obs);
    woodbury(resid.data(), mr.data(), Py.data());
    std::vector<double> av(q, 0.0), Wm(q * std::max<int64_t>(p, 1), 0.0), Bm(q * std::max<int64_t>(p, 1), 0.0);
    for (int64_t i = 0; i < n_obs; ++i) {
        const int32_t sj = obs_to_subject[i];
        av[sj] += Py[i];
        for (int64_t a = 0; a < p; ++a) {
            Wm[sj + a * q] += X[i + a * n_obs];
            Bm[sj + a * q] += VX[i + a * n_obs];
        }
    }
    DeviceBuffer<double> da, dW, dB, dC;
    const int64_t pp = std::max<int64_t>(p, 1);
    da.resize(q);
    dW.resize(q * pp);
    dB.resize(q * pp);
    dC.resize(q * pp);
    CS_CUDA(cudaMemcpyAsync(da.get(), av.data(), 8 * q, cudaMemcpyHostToDevice, s));
    CS_CUDA(cudaMemcpyAsync(dW.get(), Wm.data(), 8 * q * pp, cudaMemcpyHostToDevice, s));
    CS_CUDA(cudaMemcpyAsync(dB.get(), Bm.data(), 8 * q * pp, cudaMemcpyHostToDevice, s));
    if (p > 0) {
        const double one = 1.0, zero = 0.0;
        CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)q, (int)p, (int)q, &one, Minv,
                            (int)q, dW.get(), (int)q, &zero, dC.get(), (int)q));
    }
    // ---- per-SNP blocks
    const int64_t W = snp_end - snp_begin;
    const int64_t mb_max = std::max<int64_t>(1, std::min<int64_t>(2048, (int64_t)(4e8 / (8.0 * q))));
    DeviceBuffer<double> dE, dDE, dT, dq, dUe, dCde, dBe, dmaf;
    DeviceBuffer<int32_t> dpass, dsub;
    dE.resize(q * mb_max);
    dDE.resize(q * mb_max);
    dT.resize(q * mb_max);
    dq.resize(3 * mb_max);
    dUe.resize(pp * mb_max);
    dCde.resize(pp * mb_max);
    dBe.resize(pp * mb_max);
    dmaf.resize(mb_max);
    dpass.resize(mb_max);
    dsub.resize(q);
    CS_CUDA(cudaMemcpyAsync(dsub.get(), subject_rows, 4 * q, cudaMemcpyHostToDevice, s));
    std::vector<double> hq(3 * mb_max), hue(pp * mb_max), hcde(pp * mb_max), hbe(pp * mb_max), hm(mb_max);
    std::vector<int32_t> hp(mb_max);
    for (int64_t b0 = 0; b0 < W; b0 += mb_max) {
        const int64_t mb = std::min(mb_max, W - b0);
        {
            prof::Scope ps("stcg_encode", s, 0.0, (double)mb * q * 20.0);
            k_stcg_encode<<<(unsigned)((mb * 32 + 255) / 256), 256, 0, s>>>(
                g->packed.get(), g->stride, snp_begin + b0, mb, dsub.get(), q, dD.get(), min_maf,
                dE.get(), dDE.get(), dmaf.get(), dpass.get());
            CS_LAUNCH("stcg_encode");
        }
        {
            const double one = 1.0, zero = 0.0;
            CS_BLAS(cublasSetStream(blas, s));
            // T = M^-1 (D E)
            CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)q, (int)mb, (int)q, &one, Minv,
                                (int)q, dDE.get(), (int)q, &zero, dT.get(), (int)q));
            if (p > 0) {
                gemm_tn(blas, p, mb, q, dW.get(), q, dE.get(), q, dUe.get(), pp, s);
                gemm_tn(blas, p, mb, q, dC.get(), q, dDE.get(), q, dCde.get(), pp, s);
                gemm_tn(blas, p, mb, q, dB.get(), q, dE.get(), q, dBe.get(), pp, s);
            }
        }
        k_stcg_quads<<<(unsigned)((mb * 32 + 255) / 256), 256, 0, s>>>(dE.get(), dDE.get(), dT.get(),
                                                                     da.get(), q, mb, dq.get());
        CS_LAUNCH("stcg_quads");
        CS_CUDA(cudaMemcpyAsync(hq.data(), dq.get(), 8 * 3 * mb, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaMemcpyAsync(hm.data(), dmaf.get(), 8 * mb, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaMemcpyAsync(hp.data(), dpass.get(), 4 * mb, cudaMemcpyDeviceToHost, s));
        if (p > 0) {
            CS_CUDA(cudaMemcpyAsync(hue.data(), dUe.get(), 8 * pp * mb, cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaMemcpyAsync(hcde.data(), dCde.get(), 8 * pp * mb, cudaMemcpyDeviceToHost, s));
            CS_CUDA(cudaMemcpyAsync(hbe.data(), dBe.get(), 8 * pp * mb, cudaMemcpyDeviceToHost, s));
        }
        CS_CUDA(cudaStreamSynchronize(s));
        for (int64_t j = 0; j < mb; ++j) {
            const int64_t o = b0 + j;
            const double nan = std::numeric_limits<double>::quiet_NaN();
            if (maf) maf[o] = hm[j];
            bool ok = hp[j] != 0;
            double var = 0.0, score = 0.0;
            if (ok) {
                const double q1 = hq[3 * j], q2 = hq[3 * j + 1];
                score = hq[3 * j + 2];
                var = q1 / ve - q2 / (ve * ve);
                if (p > 0) {
                    std::vector<double> xv(p);
                    for (int64_t a = 0; a < p; ++a)
                        xv[a] = hue[a + j * pp] / ve - hcde[a + j * pp] / (ve * ve);
                    double corr = 0.0;
                    for (int64_t a = 0; a < p; ++a) {
                        double t = 0.0;
                        for (int64_t b = 0; b < p; ++b) t += inv[a + b * p] * xv[b];
                        corr += hbe[a + j * pp] * t;
                    }
                    var -= corr;
                }
                ok = !(var < 1e-15);
            }
            if (tested) tested[o] = ok ? 1 : 0;
            if (!ok) {
                if (beta) beta[o] = nan;
                if (se) se[o] = nan;
                if (pvalue) pvalue[o] = nan;
                if (log10p) log10p[o] = nan;
                continue;
            }
            const double z = score / std::sqrt(var);
            const double pv = std::erfc(std::abs(z) / std::sqrt(2.0));
            if (beta) beta[o] = score / var;
            if (se) se[o] = 1.0 / std::sqrt(var);
            if (pvalue) pvalue[o] = pv;
            if (log10p) log10p[o] = (pv > 0.0 && pv <= 1.0) ? -std::log10(pv) : (pv > 1.0 ? 0.0 : 300.0);
        }
    }
}

}  // namespace cs
