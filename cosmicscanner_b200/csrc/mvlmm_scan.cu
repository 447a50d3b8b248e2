// Multi-trait LMM scan with a fixed null, on the GPU (MvLmmEngine::scan(PlinkReader),
// src/mvlmm_engine.cpp:756-931, with processBlock :210-396 and the information-matrix checks
// of src/mvlmm_numerics.h:27-70).
//
// The null model comes from the caller as the reference's MvLmmEngine::prepareFromVce takes
// it from MvEigenVce (src/mvlmm_engine.cpp:195-207): the eigenbasis W (n x r), eigenvalues D,
// the rotated phenotypes U'y (r x d) and covariates U'X (r x p), and Vg, Ve (d x d).
//
// Per block of SNPs the reference rotates the centred, mean-imputed genotypes S_rot = W' S
// (the dominant O(n r) per SNP work) and accumulates, for every SNP k over rotated samples i,
//   H_SS = sum s_ik^2 Sigma_i^-1,  RHS_S = sum s_ik Sigma_i^-1 y_i,
//   H_XS[j] = sum x_ij s_ik Sigma_i^-1,   Sigma_i = D_i Vg + Ve.
// Here the rotation is a decode-GEMM over the packed rows (FP64, or the int8 tensor-core
// projection), and with Vg, Ve diagonalised together (Ve = R R', R^-1 Vg R^-T = Q L Q',
// T = R^-T Q): Sigma_i^-1 = T diag(w_i) T' with w_il = 1 / (D_i L_l + 1), so every
// accumulation is T diag(.) T' of one column of a GEMM of the rotated block against the
// r x d weight columns [W, W o (T'y), x_j o W].  The d x d Schur complement, the eigenvalue
// checks and the Wald test stay on the host (OpenMP over SNPs).
#include <cublas_v2.h>
#include <cuda_runtime.h>

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

__global__ void k_square(const double* __restrict__ a, int64_t n, double* __restrict__ b) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x)
        b[e] = a[e] * a[e];
}

// src/mvlmm_engine.cpp:12-52 (gamma_q / chisq_prob): series or continued fraction, 1e-7
// relative stopping, at most 100 terms, 0 when neither converges.
double gamma_q(double a, double x) {
    if (x <= 0.0) return 1.0;
    if (x < a + 1.0) {
        double ap = a, sum = 1.0 / a, del = sum;
        for (int i = 0; i < 100; ++i) {
            ap += 1.0;
            del *= x / ap;
            sum += del;
            if (std::abs(del) < std::abs(sum) * 1e-7)
                return 1.0 - sum * std::exp(-x + a * std::log(x) - std::lgamma(a));
        }
    } else {
        double b = x + 1.0 - a, c = 1.0 / 1e-30, d = 1.0 / b, h = d;
        for (int i = 1; i <= 100; ++i) {
            const double an = -i * (i - a);
            b += 2.0;
            d = an * d + b;
            if (std::abs(d) < 1e-30) d = 1e-30;
            c = b + an / c;
            if (std::abs(c) < 1e-30) c = 1e-30;
            d = 1.0 / d;
            const double del = d * c;
            h *= del;
            if (std::abs(del - 1.0) < 1e-7) return std::exp(-x + a * std::log(x) - std::lgamma(a)) * h;
        }
    }
    return 0.0;
}

double chisq_prob(double stat, int df) {
    if (stat <= 0) return 1.0;
    return gamma_q(df / 2.0, stat / 2.0);
}

// mvlmm_numerics.h:27-45 (invertInformation): 0 OK, 3 TRUE_SINGULARITY.
int invert_information(const std::vector<double>& info, int d, std::vector<double>& cov) {
    for (double v : info)
        if (!std::isfinite(v)) return 3;
    std::vector<double> sym(d * d);
    for (int a = 0; a < d; ++a)
        for (int b = 0; b < d; ++b) sym[a + b * d] = 0.5 * (info[a + b * d] + info[b + a * d]);
    std::vector<double> ev, V;
    if (!la::eigh(sym, d, ev, V)) return 3;
    double mn = ev[0], mx = 0.0;
    for (double v : ev) {
        if (!std::isfinite(v)) return 3;
        mn = std::min(mn, v);
        mx = std::max(mx, std::abs(v));
    }
    const double scale = std::max(1.0, mx);
    const double tol = 128.0 * std::numeric_limits<double>::epsilon() * scale * d;
    if (!(mn > tol)) return 3;
    cov.assign(d * d, 0.0);
    for (int a = 0; a < d; ++a)
        for (int b = 0; b < d; ++b) {
            double acc = 0.0;
            for (int l = 0; l < d; ++l) acc += V[a + l * d] * V[b + l * d] / ev[l];
            cov[a + b * d] = acc;
        }
    for (int a = 0; a < d; ++a)
        for (int b = a + 1; b < d; ++b) {
            const double m = 0.5 * (cov[a + b * d] + cov[b + a * d]);
            cov[a + b * d] = cov[b + a * d] = m;
        }
    for (double v : cov)
        if (!std::isfinite(v)) return 3;
    return 0;
}

// mvlmm_numerics.h:47-69 (conditionCovariance): 0 OK, 1 NUMERICAL_ROUNDOFF (clipped),
// 2 BOUNDARY_SOLUTION, 3 TRUE_SINGULARITY.
int condition_covariance(std::vector<double>& cov, int d) {
    for (double v : cov)
        if (!std::isfinite(v)) return 3;
    for (int a = 0; a < d; ++a)
        for (int b = a + 1; b < d; ++b) {
            const double m = 0.5 * (cov[a + b * d] + cov[b + a * d]);
            cov[a + b * d] = cov[b + a * d] = m;
        }
    std::vector<double> ev, V;
    if (!la::eigh(cov, d, ev, V)) return 3;
    double mn = ev[0], mx = 0.0;
    for (double v : ev) {
        if (!std::isfinite(v)) return 3;
        mn = std::min(mn, v);
        mx = std::max(mx, std::abs(v));
    }
    const double scale = std::max(1.0, mx);
    const double tol = 128.0 * std::numeric_limits<double>::epsilon() * scale * d;
    if (mn < -tol) return 3;
    if (mn < 0.0) {
        for (int a = 0; a < d; ++a)
            for (int b = 0; b < d; ++b) {
                double acc = 0.0;
                for (int l = 0; l < d; ++l) acc += V[a + l * d] * V[b + l * d] * std::max(ev[l], 0.0);
                cov[a + b * d] = acc;
            }
        for (int a = 0; a < d; ++a)
            for (int b = a + 1; b < d; ++b) {
                const double m = 0.5 * (cov[a + b * d] + cov[b + a * d]);
                cov[a + b * d] = cov[b + a * d] = m;
            }
        return 1;
    }
    if (mn <= tol) return 2;
    return 0;
}

}  // namespace

// The scan with the eigenbasis already on the device: dW is n x r row-major (ld r), or
// column-major with ld n when w_colmajor (then transposed here, in column chunks).
void mvlmm_scan_device(const cs_genotypes* g, const int32_t* keep, int64_t n, const double* dW,
                       bool w_colmajor, int64_t r, const double* Dv, const double* Uty, int64_t d,
                       const double* UtX, int64_t p, const double* Vg, const double* Ve,
                       int64_t snp_begin, int64_t snp_end, int precision, double* beta,
                       double* cov, double* wald, double* pvalue, double* freq,
                       int32_t* status) {
    const double* Wp = dW;
    if (!g || !keep || !Wp || !Dv || !Uty || !Vg || !Ve || n <= 0 || r <= 0 || d <= 0 || p < 0 ||
        (p > 0 && !UtX))
        fail(CS_ERR_INVALID_ARGUMENT, "MvLmmEngine::scan: bad arguments");
    if (d > 32) fail(CS_ERR_UNSUPPORTED, "at most 32 traits are supported");
    if (snp_begin < 0 || snp_end > g->n_snps || snp_begin > snp_end)
        fail(CS_ERR_INVALID_ARGUMENT, "MvLmmEngine::scan: SNP window out of range");
    for (int64_t i = 0; i < n; ++i)
        if (keep[i] < 0 || keep[i] >= g->n_samples)
            fail(CS_ERR_INVALID_ARGUMENT, "MvLmmEngine::scan: sample index out of range");
    cudaStream_t s = 0;
    cublasHandle_t blas = shared_blas();
    // ---- Sigma_i^-1 = T diag(w_i) T'
    std::vector<double> ve(Ve, Ve + d * d), R;
    if (!la::cholesky_upper(ve, (int)d, R)) fail(CS_ERR_NUMERIC, "MvLmmEngine: Ve is not positive definite");
    // cholesky_upper gives Ve = R' R (R upper); with U = R': Ve = U U'; C = U^-1 Vg U^-T
    const std::vector<double> Rinv = la::upper_inverse(R, (int)d);  // (R)^-1, upper
    std::vector<double> C(d * d, 0.0), tmp(d * d, 0.0);
    // C = R^-T Vg R^-1
    for (int64_t a = 0; a < d; ++a)
        for (int64_t b = 0; b < d; ++b) {
            double acc = 0.0;
            for (int64_t l = 0; l < d; ++l) acc += Vg[a + l * d] * Rinv[l + b * d];
            tmp[a + b * d] = acc;  // Vg R^-1
        }
    for (int64_t a = 0; a < d; ++a)
        for (int64_t b = 0; b < d; ++b) {
            double acc = 0.0;
            for (int64_t l = 0; l < d; ++l) acc += Rinv[l + a * d] * tmp[l + b * d];
            C[a + b * d] = acc;
        }
    std::vector<double> lam, Q;
    if (!la::eigh(C, (int)d, lam, Q)) fail(CS_ERR_NUMERIC, "MvLmmEngine: eigensolver failed");
    // Sigma_i = R' (D_i C + I) R = R' Q (D_i L + I) Q' R  ->  Sigma_i^-1 = T diag(w) T', T = R^-1 Q
    std::vector<double> T(d * d, 0.0);
    for (int64_t a = 0; a < d; ++a)
        for (int64_t b = 0; b < d; ++b) {
            double acc = 0.0;
            for (int64_t l = 0; l < d; ++l) acc += Rinv[a + l * d] * Q[l + b * d];
            T[a + b * d] = acc;
        }
    std::vector<double> w(r * d), yt(r * d);
    for (int64_t i = 0; i < r; ++i)
        for (int64_t l = 0; l < d; ++l) {
            w[i + l * r] = 1.0 / (Dv[i] * lam[l] + 1.0);
            double acc = 0.0;
            for (int64_t a = 0; a < d; ++a) acc += T[a + l * d] * Uty[i + a * r];
            yt[i + l * r] = acc;  // (T' y_i)_l
        }
    auto sigma_inv = [&](int64_t i, double* out) {
        for (int64_t a = 0; a < d; ++a)
            for (int64_t b = 0; b < d; ++b) {
                double acc = 0.0;
                for (int64_t l = 0; l < d; ++l) acc += T[a + l * d] * w[i + l * r] * T[b + l * d];
                out[a + b * d] = acc;
            }
    };
    // ---- H_XX, RHS_X (src/mvlmm_engine.cpp:786-812)
    const int64_t pd = p * d;
    std::vector<double> HXX(pd * pd, 0.0), RHSX(pd, 0.0), Si(d * d), Siy(d);
    for (int64_t i = 0; i < r; ++i) {
        sigma_inv(i, Si.data());
        for (int64_t a = 0; a < d; ++a) {
            double acc = 0.0;
            for (int64_t b = 0; b < d; ++b) acc += Si[a + b * d] * Uty[i + b * r];
            Siy[a] = acc;
        }
        for (int64_t j = 0; j < p; ++j) {
            const double xj = UtX[i + j * r];
            for (int64_t k2 = 0; k2 < p; ++k2) {
                const double xk = UtX[i + k2 * r];
                for (int64_t a = 0; a < d; ++a)
                    for (int64_t b = 0; b < d; ++b)
                        HXX[(j * d + a) + (k2 * d + b) * pd] += xj * xk * Si[a + b * d];
            }
            for (int64_t a = 0; a < d; ++a) RHSX[j * d + a] += xj * Siy[a];
        }
    }
    std::vector<double> HXXinv;
    if (pd > 0) {
        std::vector<double> Rx;
        if (!la::cholesky_upper(HXX, (int)pd, Rx))
            fail(CS_ERR_NUMERIC, "MvLmmEngine: H_XX is not positive definite");
        const std::vector<double> Ri = la::upper_inverse(Rx, (int)pd);
        HXXinv.assign(pd * pd, 0.0);  // (R'R)^-1 = R^-1 R^-T
        for (int64_t a = 0; a < pd; ++a)
            for (int64_t b = 0; b < pd; ++b) {
                double acc = 0.0;
                for (int64_t l = std::max(a, b); l < pd; ++l) acc += Ri[a + l * pd] * Ri[b + l * pd];
                HXXinv[a + b * pd] = acc;
            }
    }
    // ---- device: weights [W | W o Y~ | x_j o W] (r x nc) and the eigenbasis (n x r, row-major)
    const int64_t nc = d * (2 + p);
    std::vector<double> wm(r * nc);
    for (int64_t i = 0; i < r; ++i)
        for (int64_t l = 0; l < d; ++l) {
            wm[i + l * r] = w[i + l * r];
            wm[i + (d + l) * r] = w[i + l * r] * yt[i + l * r];
            for (int64_t j = 0; j < p; ++j) wm[i + ((2 + j) * d + l) * r] = UtX[i + j * r] * w[i + l * r];
        }
    DeviceBuffer<double> dWrow, dwm;
    const double* dWp_ptr = dW;
    if (w_colmajor) {
        dWrow.resize(n * r);
        colmajor_to_rowmajor(dW, n, n, r, dWrow.get(), r, s);
        dWp_ptr = dWrow.get();
    }
    dwm.resize(r * nc);
    CS_CUDA(cudaMemcpyAsync(dwm.get(), wm.data(), 8 * r * nc, cudaMemcpyHostToDevice, s));
    // ---- packed view of the kept samples over the window (repacked when keep is not the
    // identity), per-SNP means over observed kept samples (src/mvlmm_engine.cpp:862-887)
    const int64_t M = snp_end - snp_begin;
    bool identity = n == g->n_samples;
    for (int64_t i = 0; identity && i < n; ++i) identity = keep[i] == i;
    const uint8_t* first_row = g->packed.get() + snp_begin * g->stride;
    cs_packed_view view{first_row, M, g->n_samples, g->stride};
    DeviceBuffer<uint8_t> own;
    if (!identity) {
        const int64_t stride = round_up((n + 3) / 4, kRowAlign);
        own.resize(std::max<int64_t>(1, M * stride));
        DeviceBuffer<int32_t> dk;
        dk.resize(n);
        CS_CUDA(cudaMemcpyAsync(dk.get(), keep, 4 * n, cudaMemcpyHostToDevice, s));
        repack(first_row, g->stride, nullptr, M, dk.get(), n, own.get(), stride, s);
        view = cs_packed_view{own.get(), M, n, stride};
    }
    std::vector<int32_t> counts(4 * std::max<int64_t>(M, 1), 0);
    DeviceBuffer<int32_t> dcounts;
    dcounts.resize(std::max<int64_t>(1, 4 * M));
    if (M > 0) {
        row_code_counts(view, dcounts.get(), s);
        CS_CUDA(cudaMemcpyAsync(counts.data(), dcounts.get(), 16 * M, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaStreamSynchronize(s));
    }
    std::vector<double> mean(std::max<int64_t>(M, 1), 0.0), lut(4 * std::max<int64_t>(M, 1), 0.0);
    for (int64_t t = 0; t < M; ++t) {
        const int64_t c00 = counts[4 * t], c10 = counts[4 * t + 2], c11 = counts[4 * t + 3];
        const int64_t obs = c00 + c10 + c11;
        const double mu = obs > 0 ? (double)(2 * c00 + c10) / (double)obs : 0.0;
        mean[t] = mu;
        lut[4 * t] = 2.0 - mu;
        lut[4 * t + 1] = 0.0;
        lut[4 * t + 2] = 1.0 - mu;
        lut[4 * t + 3] = -mu;
    }
    DeviceBuffer<double> dlut;
    dlut.resize(std::max<int64_t>(1, 4 * M));
    if (M > 0) CS_CUDA(cudaMemcpyAsync(dlut.get(), lut.data(), 32 * M, cudaMemcpyHostToDevice, s));
    // ---- blocks of SNPs
    const int64_t mb_max = std::max<int64_t>(1, std::min<int64_t>(2048, (int64_t)(3e8 / (8.0 * r))));
    DeviceBuffer<double> dS, dS2, dH, dRest;
    dS.resize(mb_max * r);
    dS2.resize(mb_max * r);
    dH.resize(mb_max * d);
    dRest.resize(mb_max * (nc - d));
    Workspace ws;
    std::vector<double> hH(mb_max * d), hR(mb_max * (nc - d));
    for (int64_t b0 = 0; b0 < M; b0 += mb_max) {
        const int64_t mb = std::min(mb_max, M - b0);
        // S_rot^T (mb x r, row-major): the block's centred, mean-imputed genotypes rotated by W
        cs_packed_view bv{view.rows + b0 * view.stride, mb, view.n_samples, view.stride};
        if (precision == CS_PRECISION_MIXED) {
            MixedScan* mixed = mixed_scan_create(bv, mean.data() + b0, counts.data() + 4 * b0);
            try {
                mixed_scan_project(mixed, dWp_ptr, r, r, dS.get(), r, s);
            } catch (...) {
                mixed_scan_destroy(mixed);
                throw;
            }
            mixed_scan_destroy(mixed);
        } else {
            decode_gemm_rows_fp64(bv, dlut.get() + 4 * b0, dWp_ptr, r, r, dS.get(), r, ws, s);
        }
        k_square<<<grid_for(mb * r), 256, 0, s>>>(dS.get(), mb * r, dS2.get());
        CS_LAUNCH("mvlmm_square");
        {
            const double one = 1.0, zero = 0.0;
            CS_BLAS(cublasSetStream(blas, s));
            // H (mb x d) = S2 (mb x r) W (r x d): S2 row-major = (r x mb) column-major
            CS_BLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)mb, (int)d, (int)r, &one,
                                dS2.get(), (int)r, dwm.get(), (int)r, &zero, dH.get(), (int)mb));
            CS_BLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)mb, (int)(nc - d), (int)r, &one,
                                dS.get(), (int)r, dwm.get() + d * r, (int)r, &zero, dRest.get(),
                                (int)mb));
        }
        CS_CUDA(cudaMemcpyAsync(hH.data(), dH.get(), 8 * mb * d, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaMemcpyAsync(hR.data(), dRest.get(), 8 * mb * (nc - d), cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaStreamSynchronize(s));
        // ---- per SNP (src/mvlmm_engine.cpp:286-394)
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t k = 0; k < mb; ++k) {
            const int64_t o = b0 + k;
            std::vector<double> HSS(d * d, 0.0), RHSS(d, 0.0), HXS(pd * d, 0.0);
            for (int64_t a = 0; a < d; ++a)
                for (int64_t b = 0; b < d; ++b) {
                    double acc = 0.0;
                    for (int64_t l = 0; l < d; ++l) acc += T[a + l * d] * hH[k + l * mb] * T[b + l * d];
                    HSS[a + b * d] = acc;
                }
            for (int64_t a = 0; a < d; ++a) {
                double acc = 0.0;
                for (int64_t l = 0; l < d; ++l) acc += T[a + l * d] * hR[k + l * mb];
                RHSS[a] = acc;
            }
            for (int64_t j = 0; j < p; ++j)
                for (int64_t a = 0; a < d; ++a)
                    for (int64_t b = 0; b < d; ++b) {
                        double acc = 0.0;
                        for (int64_t l = 0; l < d; ++l)
                            acc += T[a + l * d] * hR[k + ((1 + j) * d + l) * mb] * T[b + l * d];
                        HXS[(j * d + a) + b * pd] = acc;
                    }
            std::vector<double> schur(HSS), adj(RHSS);
            if (p > 0) {
                // Schur = H_SS - H_XS' H_XX^-1 H_XS; adj = RHS_S - H_XS' H_XX^-1 RHS_X
                std::vector<double> Z(pd * d, 0.0), zr(pd, 0.0);
                for (int64_t a = 0; a < pd; ++a) {
                    for (int64_t b = 0; b < d; ++b) {
                        double acc = 0.0;
                        for (int64_t l = 0; l < pd; ++l) acc += HXXinv[a + l * pd] * HXS[l + b * pd];
                        Z[a + b * pd] = acc;
                    }
                    double acc = 0.0;
                    for (int64_t l = 0; l < pd; ++l) acc += HXXinv[a + l * pd] * RHSX[l];
                    zr[a] = acc;
                }
                for (int64_t a = 0; a < d; ++a) {
                    for (int64_t b = 0; b < d; ++b) {
                        double acc = 0.0;
                        for (int64_t l = 0; l < pd; ++l) acc += HXS[l + a * pd] * Z[l + b * pd];
                        schur[a + b * d] -= acc;
                    }
                    double acc = 0.0;
                    for (int64_t l = 0; l < pd; ++l) acc += HXS[l + a * pd] * zr[l];
                    adj[a] -= acc;
                }
            }
            const double nan = std::numeric_limits<double>::quiet_NaN();
            freq[o] = mean[o] / 2.0;
            auto reject = [&](int code) {
                status[o] = code;
                wald[o] = pvalue[o] = nan;
                for (int64_t a = 0; a < d; ++a) beta[o * d + a] = nan;
                if (cov)
                    for (int64_t a = 0; a < d * d; ++a) cov[o * d * d + a] = nan;
            };
            std::vector<double> sinv;
            if (invert_information(schur, (int)d, sinv) != 0) {
                reject(3);
                continue;
            }
            for (int64_t a = 0; a < d; ++a)
                for (int64_t b = a + 1; b < d; ++b) {
                    const double m = 0.5 * (schur[a + b * d] + schur[b + a * d]);
                    schur[a + b * d] = schur[b + a * d] = m;
                }
            std::vector<double> bta(d, 0.0);
            bool finite = true;
            for (int64_t a = 0; a < d; ++a) {
                for (int64_t b = 0; b < d; ++b) bta[a] += sinv[a + b * d] * adj[b];
                finite &= std::isfinite(bta[a]);
            }
            if (!finite) {
                reject(3);
                continue;
            }
            double ws2 = 0.0;
            for (int64_t a = 0; a < d; ++a)
                for (int64_t b = 0; b < d; ++b) ws2 += bta[a] * schur[a + b * d] * bta[b];
            if (!std::isfinite(ws2) || ws2 < 0.0) {
                reject(3);
                continue;
            }
            const double pv = chisq_prob(ws2, (int)d);
            const int cst = condition_covariance(sinv, (int)d);
            if (cst == 3) {
                reject(3);
                continue;
            }
            status[o] = cst;  // 0 OK, 1 roundoff (clipped), 2 boundary
            wald[o] = ws2;
            pvalue[o] = pv;
            for (int64_t a = 0; a < d; ++a) beta[o * d + a] = bta[a];
            if (cov)
                for (int64_t a = 0; a < d * d; ++a) cov[o * d * d + a] = sinv[a];
        }
    }
}

void mvlmm_scan(const cs_genotypes* g, const int32_t* keep, int64_t n, const double* Wp, int64_t r,
                const double* Dv, const double* Uty, int64_t d, const double* UtX, int64_t p,
                const double* Vg, const double* Ve, int64_t snp_begin, int64_t snp_end,
                int precision, double* beta, double* cov, double* wald, double* pvalue,
                double* freq, int32_t* status) {
    if (!Wp || n <= 0 || r <= 0) fail(CS_ERR_INVALID_ARGUMENT, "MvLmmEngine::scan: bad arguments");
    // host W (column-major) -> device, row-major
    DeviceBuffer<double> dWp;
    dWp.resize(n * r);
    {
        std::vector<double> wr(n * r);
        for (int64_t i = 0; i < n; ++i)
            for (int64_t c = 0; c < r; ++c) wr[i * r + c] = Wp[i + c * n];
        CS_CUDA(cudaMemcpy(dWp.get(), wr.data(), 8 * n * r, cudaMemcpyHostToDevice));
    }
    mvlmm_scan_device(g, keep, n, dWp.get(), false, r, Dv, Uty, d, UtX, p, Vg, Ve, snp_begin,
                      snp_end, precision, beta, cov, wald, pvalue, freq, status);
}

}  // namespace cs
