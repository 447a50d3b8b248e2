// Multi-trait matrix-free REML: the multivariate null model of `--model multivariate`
// (MvEigenVce, libCosmicCore/src/eigen_vce.cpp:496-911) without the dense N x N eigenbasis.
//
// Model: vec(Y) ~ N((I_d (x) X) b, V), V = Vg (x) K + Ve (x) I_n for d traits, K = Z Z^T / divisor.
// The reference's EM update (MvEigenVce::updateEM, :551-604), written for a general K instead
// of its eigenbasis, is
//     Vg <- Vg + Vg (Qg - Tg) Vg / (n - p),   Ve <- Ve + Ve (Qe - Te) Ve / (n - p),
//     Qg = (PY)' K (PY),  Qe = (PY)' (PY),  Tg[a][b] = tr(P (E_ab (x) K)),  Te[a][b] = tr(P (E_ab (x) I))
// with P the REML projection.  Here every quantity comes from kinship applies:
//   * P = Q (Q V Q)^+ Q with Q = I_d (x) (I - X (X'X)^-1 X') (an identity of REML), so P v is Q x
//     with x from conjugate gradients on Q V Q restricted to the range of Q: no V^-1 X columns;
//   * the traces are Hutchinson estimates, tr(P A) ~ mean_s z_s' P A z_s over S Rademacher
//     probes of n x d, redrawn each iteration from one mt19937_64 stream (probe s, trait a takes
//     column s d + a), as STCG_VCE draws its probes (libCosmicCore/src/stcg_vce.cpp:215-263);
//   * one CG block carries [Y | Z_1 .. Z_S]: (1 + S) d right-hand sides (264 for 8 traits and 32
//     probes) in every kinship apply, each group of d columns one vector of length n d with its
//     own CG recurrence; the preconditioner is the trait-block Jacobi Q (I_n (x) (Vg + Ve)^-1) Q
//     (the diagonal of K is about 1);
//   * one more apply K [PY | Z_1 .. Z_S] gives Qg and the Tg estimates.
// Starting values Vg = Ve = Cov(Y) / 2 over n - p - 1 (:536-548); the reference's stopping rule
// (|dVg|^2 + |dVe|^2) / max(1, 2 d^2) < tol.
#include <cublas_v2.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "linalg_host.h"
#include "vce_internal.h"

namespace cs {

namespace {

constexpr int kMaxTraits = 16;

unsigned grid_1d(int64_t total) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 16LL * num_sms()));
}

// out[i, j d + a] = f sum_b A[i, j d + b] M1[b][a] + sum_b B[i, j d + b] M2[b][a] over the
// row-major n x (g d) blocks (B and M2 optional); M1, M2 row-major d x d in constant order.
__global__ void k_mix_groups(const double* __restrict__ A, const double* __restrict__ B,
                             int64_t ld, int64_t n, int d, int64_t g,
                             const double* __restrict__ M1, const double* __restrict__ M2,
                             double f, double* __restrict__ out) {
    __shared__ double m1[kMaxTraits * kMaxTraits], m2[kMaxTraits * kMaxTraits];
    for (int t = threadIdx.x; t < d * d; t += blockDim.x) {
        m1[t] = M1[t];
        m2[t] = M2 ? M2[t] : 0.0;
    }
    __syncthreads();
    const int64_t total = n * g * d;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / (g * d), rest = e - i * (g * d);
        const int64_t j = rest / d;
        const int a = (int)(rest - j * d);
        const double* ar = A + i * ld + j * d;
        double acc = 0.0;
        for (int b = 0; b < d; ++b) acc += ar[b] * m1[b * d + a];
        acc *= f;
        if (B) {
            const double* br = B + i * ld + j * d;
            for (int b = 0; b < d; ++b) acc += br[b] * m2[b * d + a];
        }
        out[i * ld + rest] = acc;
    }
}

// X[:, c] += alpha[c] P[:, c];  R[:, c] -= alpha[c] AP[:, c]
__global__ void k_cg_step(double* __restrict__ X, double* __restrict__ R,
                          const double* __restrict__ P, const double* __restrict__ AP, int64_t ld,
                          int64_t n, int64_t k, const double* __restrict__ alpha) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / k, c = e - i * k;
        const double a = alpha[c];
        X[i * ld + c] += a * P[i * ld + c];
        R[i * ld + c] -= a * AP[i * ld + c];
    }
}

// P[:, c] = Zb[:, c] + beta[c] P[:, c]
__global__ void k_cg_dir(double* __restrict__ P, const double* __restrict__ Zb, int64_t ld,
                         int64_t n, int64_t k, const double* __restrict__ beta) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / k, c = e - i * k;
        P[i * ld + c] = Zb[i * ld + c] + beta[c] * P[i * ld + c];
    }
}

struct MvState {
    cs_kinship* op = nullptr;
    double fac = 1.0;  // num_variants / divisor: K = fac x (the operator's Z Z^T / num_variants)
    int precision = CS_PRECISION_FP64;
    int64_t n = 0, p = 0, C = 0;
    int d = 0;
    cublasHandle_t blas = nullptr;
    DeviceBuffer<double> Xd, G;         // X (row-major n x p), (X'X)^-1 (p x p)
    DeviceBuffer<double> T1, T2;        // projection work (C x p)
    DeviceBuffer<double> KW, mats;      // apply work; Vg, Ve, Minv (row-major d x d each)
    int64_t applies = 0, apply_cols = 0;

    // B (row-major n x C) <- Q B
    void project(double* B, int64_t k, cudaStream_t s) {
        if (p == 0 || k == 0) return;
        const double one = 1.0, zero = 0.0, mone = -1.0;
        CS_BLAS(cublasSetStream(blas, s));
        T1.resize(k * p);
        T2.resize(k * p);
        // column-major views: B^T (k x n, ld C), X^T (p x n, ld p)
        CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)k, (int)p, (int)n, &one, B, (int)C,
                            Xd.get(), (int)p, &zero, T1.get(), (int)k));  // (X'B)^T
        CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)k, (int)p, (int)p, &one, T1.get(),
                            (int)k, G.get(), (int)p, &zero, T2.get(), (int)k));  // (G X'B)^T
        CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)k, (int)n, (int)p, &mone, T2.get(),
                            (int)k, Xd.get(), (int)p, &one, B, (int)C));
    }
    // Out = Q (Vg (x) K + Ve (x) I) W over the first k columns (whole groups)
    void apply(const double* W, int64_t k, double* Out, cudaStream_t s) {
        KW.resize(n * C);
        kinship_apply_rowmajor(op, W, C, k, KW.get(), C, precision, s);
        ++applies;
        apply_cols += k;
        prof::Scope ps("mv_kron_combine", s, 4.0 * (double)n * k * d, 24.0 * (double)n * k);
        k_mix_groups<<<grid_1d(n * k), 256, 0, s>>>(KW.get(), W, C, n, d, k / d, mats.get(),
                                                    mats.get() + d * d, fac, Out);
        CS_LAUNCH("mv_kron_combine");
        project(Out, k, s);
    }
    // Zb = Q (R (Vg + Ve)^-1) over the first k columns
    void precondition(const double* R, int64_t k, double* Zb, cudaStream_t s) {
        k_mix_groups<<<grid_1d(n * k), 256, 0, s>>>(R, nullptr, C, n, d, k / d,
                                                    mats.get() + 2 * d * d, nullptr, 1.0, Zb);
        CS_LAUNCH("mv_precondition");
        project(Zb, k, s);
    }
};

// Grouped CG on Q V Q (range of Q) for the k = g d columns of B (already projected), every
// group of d columns one system; stops per group on ||r|| < tol ||b|| (relative) or
// ||r|| < tol, or at max_iter.  Returns CG iterations summed over groups.
int64_t solve_groups(MvState& st, const double* B, double* Xs, int64_t k, double tol,
                     bool relative, int max_iter, PcgWorkspace& ws, cudaStream_t s) {
    const int64_t n = st.n, C = st.C;
    const int d = st.d;
    const int64_t g = k / d;
    ws.R.resize(n * C);
    ws.P.resize(n * C);
    ws.AP.resize(n * C);
    ws.Zp.resize(n * C);
    ws.alpha.resize(C);
    ws.beta.resize(C);
    CS_CUDA(cudaMemsetAsync(Xs, 0, 8 * n * C, s));
    CS_CUDA(cudaMemcpyAsync(ws.R.get(), B, 8 * n * C, cudaMemcpyDeviceToDevice, s));
    st.precondition(ws.R.get(), k, ws.Zp.get(), s);
    CS_CUDA(cudaMemcpyAsync(ws.P.get(), ws.Zp.get(), 8 * n * C, cudaMemcpyDeviceToDevice, s));
    auto group_dots = [&](const double* A, const double* Bm) {
        std::vector<double> col(k), grp(g, 0.0);
        column_dots(A, C, Bm, C, n, k, col.data(), ws, s);
        for (int64_t c = 0; c < k; ++c) grp[c / d] += col[c];
        return grp;
    };
    std::vector<double> bb = group_dots(ws.R.get(), ws.R.get());
    std::vector<double> rz = group_dots(ws.R.get(), ws.Zp.get());
    std::vector<double> thr(g);
    std::vector<char> live(g);
    for (int64_t j = 0; j < g; ++j) {
        thr[j] = relative ? tol * std::sqrt(bb[j]) : tol;
        live[j] = std::sqrt(bb[j]) >= 1e-20 && !(std::sqrt(bb[j]) < thr[j]);
    }
    int64_t iters = 0;
    std::vector<double> alpha(C, 0.0), beta(C, 0.0);
    for (int it = 0; it < max_iter; ++it) {
        bool any = false;
        for (int64_t j = 0; j < g; ++j) any = any || live[j];
        if (!any) break;
        st.apply(ws.P.get(), k, ws.AP.get(), s);
        const std::vector<double> pap = group_dots(ws.P.get(), ws.AP.get());
        for (int64_t j = 0; j < g; ++j) {
            const double a = live[j] && pap[j] != 0.0 ? rz[j] / pap[j] : 0.0;
            for (int t = 0; t < d; ++t) alpha[j * d + t] = a;
            if (live[j]) ++iters;
        }
        CS_CUDA(cudaMemcpyAsync(ws.alpha.get(), alpha.data(), 8 * k, cudaMemcpyHostToDevice, s));
        k_cg_step<<<grid_1d(n * k), 256, 0, s>>>(Xs, ws.R.get(), ws.P.get(), ws.AP.get(), C, n, k,
                                                 ws.alpha.get());
        CS_LAUNCH("mv_cg_step");
        const std::vector<double> rr = group_dots(ws.R.get(), ws.R.get());
        for (int64_t j = 0; j < g; ++j)
            if (live[j] && std::sqrt(rr[j]) < thr[j]) live[j] = 0;
        st.precondition(ws.R.get(), k, ws.Zp.get(), s);
        const std::vector<double> rz_new = group_dots(ws.R.get(), ws.Zp.get());
        for (int64_t j = 0; j < g; ++j) {
            const double b = live[j] && rz[j] != 0.0 ? rz_new[j] / rz[j] : 0.0;
            for (int t = 0; t < d; ++t) beta[j * d + t] = b;
            rz[j] = rz_new[j];
        }
        CS_CUDA(cudaMemcpyAsync(ws.beta.get(), beta.data(), 8 * k, cudaMemcpyHostToDevice, s));
        // frozen groups: beta 0 and Zb of a converged residual keep their direction small; their
        // alpha is 0 from here on, so x and r no longer change
        k_cg_dir<<<grid_1d(n * k), 256, 0, s>>>(ws.P.get(), ws.Zp.get(), C, n, k, ws.beta.get());
        CS_LAUNCH("mv_cg_dir");
    }
    CS_CUDA(cudaStreamSynchronize(s));
    return iters;
}

}  // namespace

void mv_stcg_default_options(cs_mv_stcg_options* o) {
    o->max_iter = 100;
    o->tol = 1e-8;
    o->mc_samples = 32;
    o->pcg_tol = 1e-8;
    o->pcg_relative = 1;
    o->pcg_max_iter = 2000;
    o->probe_seed = 20250101ull;
    o->precision = CS_PRECISION_FP64;
}

void mv_stcg_solve(cs_kinship* op, double divisor, const double* Y, int32_t d, const double* X,
                   int64_t p, const cs_mv_stcg_options* opt_in, double* Vg_out, double* Ve_out,
                   cs_mv_stcg_result* res) {
    const auto t_start = std::chrono::steady_clock::now();
    cs_mv_stcg_options opt;
    if (opt_in) opt = *opt_in;
    else mv_stcg_default_options(&opt);
    const int64_t n = op->rows;
    if (d < 1 || d > kMaxTraits || p < 0 || (p > 0 && !X) || !Y || n <= p + 1)
        fail(CS_ERR_INVALID_ARGUMENT, "multi-trait REML: bad dimensions (1 <= traits <= 16)");
    if (opt.mc_samples < 1 || opt.max_iter < 0 || opt.pcg_max_iter < 1)
        fail(CS_ERR_INVALID_ARGUMENT, "multi-trait REML: bad options");
    if (!(divisor > 0.0)) divisor = (double)op->num_variants;
    cudaStream_t s = 0;
    MvState st;
    st.op = op;
    st.fac = (double)op->num_variants / divisor;
    st.precision = opt.precision;
    st.n = n;
    st.p = p;
    st.d = d;
    const int64_t S = opt.mc_samples, k = (1 + S) * d;
    st.C = k;
    st.blas = shared_blas();
    // covariates: X row-major and (X'X)^-1
    std::vector<double> Xr(std::max<int64_t>(1, n * p)), G(std::max<int64_t>(1, p * p), 0.0);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t a = 0; a < p; ++a) Xr[i * p + a] = X[i + a * n];
    if (p > 0) {
        std::vector<double> xtx(p * p, 0.0);
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b) {
                double acc = 0.0;
                for (int64_t i = 0; i < n; ++i) acc += X[i + a * n] * X[i + b * n];
                xtx[a + b * p] = acc;
            }
        std::vector<double> L, Dd;
        if (!la::ldlt(xtx, (int)p, L, Dd)) fail(CS_ERR_NUMERIC, "multi-trait REML: X'X is singular");
        G = la::ldlt_inverse(L, Dd, (int)p);
    }
    st.Xd.resize(std::max<int64_t>(1, n * p));
    st.G.resize(std::max<int64_t>(1, p * p));
    CS_CUDA(cudaMemcpy(st.Xd.get(), Xr.data(), 8 * n * p, cudaMemcpyHostToDevice));
    CS_CUDA(cudaMemcpy(st.G.get(), G.data(), 8 * p * p, cudaMemcpyHostToDevice));
    // starting values (eigen_vce.cpp:536-548)
    std::vector<double> Vg(d * d), Ve(d * d), mean(d, 0.0);
    for (int a = 0; a < d; ++a) {
        for (int64_t i = 0; i < n; ++i) mean[a] += Y[i + a * n];
        mean[a] /= (double)n;
    }
    for (int a = 0; a < d; ++a)
        for (int b = 0; b < d; ++b) {
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) acc += (Y[i + a * n] - mean[a]) * (Y[i + b * n] - mean[b]);
            Vg[a * d + b] = Ve[a * d + b] = 0.5 * acc / (double)(n - p - 1);
        }
    // blocks: RHS [Y | Z_1 .. Z_S] (projected), solutions, the extra apply
    DeviceBuffer<double> Bk, Xs, KP;
    Bk.resize(n * k);
    Xs.resize(n * k);
    KP.resize(n * k);
    st.mats.resize(3 * d * d);
    {
        std::vector<double> h(n * d);
        for (int64_t i = 0; i < n; ++i)
            for (int a = 0; a < d; ++a) h[i * d + a] = Y[i + a * n];
        CS_CUDA(cudaMemcpy2DAsync(Bk.get(), 8 * k, h.data(), 8 * d, 8 * d, n, cudaMemcpyHostToDevice, s));
        CS_CUDA(cudaStreamSynchronize(s));
    }
    RademacherStream probes;
    probes.seed(opt.probe_seed, s);
    PcgWorkspace ws;
    DeviceBuffer<double> cross;
    cross.resize(k * k);
    int64_t pcg_total = 0;
    res->converged = 0;
    res->iterations = 0;
    const double one = 1.0, zero = 0.0;
    for (int iter = 0; iter < opt.max_iter; ++iter) {
        // mats = [Vg | Ve | (Vg + Ve)^-1]
        std::vector<double> Minv(d * d);
        {
            std::vector<double> M(d * d), L, Dd;
            for (int t = 0; t < d * d; ++t) M[t] = Vg[t] + Ve[t];
            if (!la::ldlt(M, d, L, Dd)) fail(CS_ERR_NUMERIC, "multi-trait REML: Vg + Ve is not positive definite");
            Minv = la::ldlt_inverse(L, Dd, d);
            std::vector<double> all(3 * d * d);
            std::copy(Vg.begin(), Vg.end(), all.begin());
            std::copy(Ve.begin(), Ve.end(), all.begin() + d * d);
            std::copy(Minv.begin(), Minv.end(), all.begin() + 2 * d * d);
            CS_CUDA(cudaMemcpyAsync(st.mats.get(), all.data(), 8 * 3 * d * d, cudaMemcpyHostToDevice, s));
            CS_CUDA(cudaStreamSynchronize(s));
        }
        // probes Z_s (column s d + a), the RHS block projected
        probes.draw(n, S * d, Bk.get() + d, k, s);
        DeviceBuffer<double> rhs;
        rhs.resize(n * k);
        CS_CUDA(cudaMemcpyAsync(rhs.get(), Bk.get(), 8 * n * k, cudaMemcpyDeviceToDevice, s));
        st.project(rhs.get(), k, s);
        pcg_total += solve_groups(st, rhs.get(), Xs.get(), k, opt.pcg_tol, opt.pcg_relative != 0,
                                  opt.pcg_max_iter, ws, s);
        // P [Y | Z] = Q x (the iterates stay in the range of Q; project once more against drift)
        st.project(Xs.get(), k, s);
        // K [PY | Z]: PY in the first d columns, the raw probes after them
        CS_CUDA(cudaMemcpy2DAsync(KP.get(), 8 * k, Xs.get(), 8 * k, 8 * d, n, cudaMemcpyDeviceToDevice, s));
        CS_CUDA(cudaMemcpy2DAsync(KP.get() + d, 8 * k, Bk.get() + d, 8 * k, 8 * S * d, n,
                                  cudaMemcpyDeviceToDevice, s));
        st.KW.resize(n * k);
        kinship_apply_rowmajor(op, KP.get(), k, k, st.KW.get(), k, opt.precision, s);
        ++st.applies;
        st.apply_cols += k;
        // cross products: [P Y | P Z]^T [fac K PY | fac K Z] and [P Y | P Z]^T [PY | Z]
        CS_BLAS(cublasSetStream(st.blas, s));
        std::vector<double> ck(k * k), ci(k * k);
        CS_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)k, (int)k, (int)n, &st.fac,
                            Xs.get(), (int)k, st.KW.get(), (int)k, &zero, cross.get(), (int)k));
        CS_CUDA(cudaMemcpyAsync(ck.data(), cross.get(), 8 * k * k, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaStreamSynchronize(s));
        CS_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)k, (int)k, (int)n, &one,
                            Xs.get(), (int)k, KP.get(), (int)k, &zero, cross.get(), (int)k));
        CS_CUDA(cudaMemcpyAsync(ci.data(), cross.get(), 8 * k * k, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaStreamSynchronize(s));
        // column-major k x k: entry (r, c) = sum_i A[i, r] B[i, c]
        std::vector<double> Qg(d * d), Qe(d * d), Tg(d * d, 0.0), Te(d * d, 0.0);
        for (int a = 0; a < d; ++a)
            for (int b = 0; b < d; ++b) {
                Qg[a * d + b] = ck[a + b * k];
                Qe[a * d + b] = ci[a + b * k];
                for (int64_t q = 1; q <= S; ++q) {
                    Tg[a * d + b] += ck[(q * d + a) + (q * d + b) * k];
                    Te[a * d + b] += ci[(q * d + a) + (q * d + b) * k];
                }
            }
        for (int t = 0; t < d * d; ++t) {
            Tg[t] /= (double)S;
            Te[t] /= (double)S;
        }
        auto sym = [&](std::vector<double>& M) {
            for (int a = 0; a < d; ++a)
                for (int b = a + 1; b < d; ++b) {
                    const double v = 0.5 * (M[a * d + b] + M[b * d + a]);
                    M[a * d + b] = M[b * d + a] = v;
                }
        };
        sym(Qg);
        sym(Qe);
        sym(Tg);
        sym(Te);
        // EM update (eigen_vce.cpp:551-604 in the general form)
        auto update = [&](const std::vector<double>& V0, const std::vector<double>& Qm,
                          const std::vector<double>& Tm) {
            std::vector<double> Dm(d * d), t1(d * d, 0.0), out(d * d);
            for (int t = 0; t < d * d; ++t) Dm[t] = Qm[t] - Tm[t];
            for (int a = 0; a < d; ++a)
                for (int b = 0; b < d; ++b)
                    for (int c = 0; c < d; ++c) t1[a * d + b] += V0[a * d + c] * Dm[c * d + b];
            for (int a = 0; a < d; ++a)
                for (int b = 0; b < d; ++b) {
                    double acc = 0.0;
                    for (int c = 0; c < d; ++c) acc += t1[a * d + c] * V0[c * d + b];
                    out[a * d + b] = V0[a * d + b] + acc / (double)(n - p);
                }
            sym(out);
            return out;
        };
        const std::vector<double> Vg_new = update(Vg, Qg, Tg), Ve_new = update(Ve, Qe, Te);
        double err = 0.0;
        for (int t = 0; t < d * d; ++t)
            err += (Vg_new[t] - Vg[t]) * (Vg_new[t] - Vg[t]) + (Ve_new[t] - Ve[t]) * (Ve_new[t] - Ve[t]);
        err /= std::max(1.0, 2.0 * d * d);
        Vg = Vg_new;
        Ve = Ve_new;
        res->iterations = iter + 1;
        if (err < opt.tol) {
            res->converged = 1;
            break;
        }
    }
    // column-major d x d outputs (symmetric)
    for (int a = 0; a < d; ++a)
        for (int b = 0; b < d; ++b) {
            if (Vg_out) Vg_out[a + b * d] = Vg[a * d + b];
            if (Ve_out) Ve_out[a + b * d] = Ve[a * d + b];
        }
    res->pcg_iterations = pcg_total;
    res->operator_applies = st.applies;
    res->operator_columns = st.apply_cols;
    res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
}

}  // namespace cs
