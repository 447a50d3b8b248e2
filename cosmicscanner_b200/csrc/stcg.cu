// Matrix-free AI-REML on the GPU: the STCG variance-component estimator
// (libCosmicCore/src/stcg_vce.cpp:157-407, declared in libCosmicCore/src/stcg_vce.h:7-54).
//
// theta = (sigma2_g, sigma2_pe, sigma2_e) for V = sg2 Zr K Zr^T + spe2 Zr Zr^T + se2 I over
// records; without the permanent-environment component (every record its own genotype row)
// it is the single-trait LMM's two-component AI-REML.  Per iteration the reference runs
// 1 + p + 3 + mc_samples separate CG solves and mc_samples + 1 separate kinship applies,
// each streaming the packed genotypes for one vector.  Here the solves that share V run as
// two multi-right-hand-side CG blocks:
//   A: [y | X | z_1 .. z_S]         -> V^-1 y, V^-1 X, V^-1 z_t  (P z_t by projection)
//   B: [dVg Py | dVpe Py | Py]      -> q_k = P s_k
// with one kinship apply for [Py | z_1 .. z_S] in between, so every genotype pass carries
// the whole block.  Scores, the 3x3 average-information matrix, the damped AI / EM update
// with its clamps, the SLQ log-likelihood and the stopping rule follow the reference.
#include <cublas_v2.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <limits>
#include <vector>

#include "linalg_host.h"
#include "vce_internal.h"

struct cs_vce {
    cublasHandle_t blas = nullptr;
    cs::RecordMap rm;
    cs::VOperator V;
    cs::PcgWorkspace pw;
    cs::RademacherStream probes, slq_rng;
    cs::DeviceBuffer<double> rhsA, solA, W, IN, DG, DP, rhsB, solB, Q, small, cm;
    cs::DeviceBuffer<double> lz, lw;  // Lanczos blocks
    cs::LowRankPreconditioner precond;
    std::vector<double> beta, a_rows, pe_rows, hist;
    int64_t p = 0, n_rows = 0;
    bool solved = false;
};

namespace cs {

namespace {

unsigned grid_1d(int64_t total) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 16LL * num_sms()));
}

// dst[:, dc + j] = src[:, idx[j]] for j < k (host index list, small)
__global__ void k_copy_cols(const double* __restrict__ src, int64_t lds, int64_t n, int64_t s0,
                            int64_t k, double* __restrict__ dst, int64_t ldd, int64_t d0) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        dst[r * ldd + d0 + c] = src[r * lds + s0 + c];
    }
}

// W[:, c] -= coef[c] * V[:, c]
__global__ void k_axpy_cols(double* __restrict__ Wm, const double* __restrict__ Vm, int64_t ld,
                            int64_t n, int64_t k, const double* __restrict__ coef) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        Wm[r * ld + c] -= coef[c] * Vm[r * ld + c];
    }
}

// Vn[:, c] = W[:, c] * inv[c]
__global__ void k_scale_cols(double* __restrict__ Vn, const double* __restrict__ Wm, int64_t ld,
                             int64_t n, int64_t k, const double* __restrict__ inv, int divide) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k, c = e - r * k;
        Vn[r * ld + c] = divide ? (inv[c] != 0.0 ? Wm[r * ld + c] / inv[c] : 0.0)
                                : Wm[r * ld + c] * inv[c];
    }
}

void copy_cols(const double* src, int64_t lds, int64_t n, int64_t s0, int64_t k, double* dst,
               int64_t ldd, int64_t d0, cudaStream_t s) {
    if (k <= 0) return;
    k_copy_cols<<<grid_1d(n * k), 256, 0, s>>>(src, lds, n, s0, k, dst, ldd, d0);
    CS_LAUNCH("copy_cols");
}

// Host C (a x b, column-major) = A[:, a0 : a0 + a]^T B[:, b0 : b0 + b] for row-major blocks.
std::vector<double> cross(cublasHandle_t blas, const double* A, int64_t lda, int64_t a0, int64_t a,
                          const double* B, int64_t ldb, int64_t b0, int64_t b, int64_t n,
                          DeviceBuffer<double>& tmp, cudaStream_t s) {
    std::vector<double> out(a * b, 0.0);
    if (a == 0 || b == 0) return out;
    tmp.resize(a * b);
    const double one = 1.0, zero = 0.0;
    CS_BLAS(cublasSetStream(blas, s));
    CS_BLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)a, (int)b, (int)n, &one, A + a0,
                        (int)lda, B + b0, (int)ldb, &zero, tmp.get(), (int)a));
    CS_CUDA(cudaMemcpyAsync(out.data(), tmp.get(), 8 * a * b, cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    return out;
}

// Out[:, o0 + j] = Sol[:, s0 + j] - Sol[:, 1 : 1 + p] coef[:, j]   (stcg_vce.cpp:147-154)
void project(cublasHandle_t blas, const double* Sol, int64_t lds, int64_t s0, int64_t k,
             const double* VinvX, int64_t ldv, int64_t p, const std::vector<double>& coef,
             double* Out, int64_t ldo, int64_t o0, int64_t n, DeviceBuffer<double>& tmp,
             cudaStream_t s) {
    copy_cols(Sol, lds, n, s0, k, Out, ldo, o0, s);
    if (p == 0 || k == 0) return;
    tmp.resize(p * k);
    CS_CUDA(cudaMemcpyAsync(tmp.get(), coef.data(), 8 * p * k, cudaMemcpyHostToDevice, s));
    const double mone = -1.0, one = 1.0;
    CS_BLAS(cublasSetStream(blas, s));
    // Out^c (k x n) -= coef^T (k x p) VinvX^c (p x n)
    CS_BLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)k, (int)n, (int)p, &mone, tmp.get(),
                        (int)p, VinvX, (int)ldv, &one, Out + o0, (int)ldo));
}

struct NullFit {
    std::vector<double> XtVinvX, inv, L, D, beta;
    bool ok = false;
};

// XtVinvX = X^T V^-1 X, its inverse, beta  (stcg_vce.cpp:128-145)
NullFit null_fit(const std::vector<double>& xts, int64_t p, int64_t ldc) {
    NullFit f;
    f.XtVinvX.assign(p * p, 0.0);
    for (int64_t a = 0; a < p; ++a)
        for (int64_t b = 0; b < p; ++b) f.XtVinvX[a + b * p] = xts[a + (1 + b) * ldc];
    f.beta.assign(p, 0.0);
    if (p == 0) {
        f.ok = true;
        return f;
    }
    if (!la::ldlt(f.XtVinvX, (int)p, f.L, f.D)) return f;
    f.inv = la::ldlt_inverse(f.L, f.D, (int)p);
    for (int64_t a = 0; a < p; ++a)
        for (int64_t b = 0; b < p; ++b) f.beta[a] += f.inv[a + b * p] * xts[b + 0 * ldc];
    f.ok = true;
    return f;
}

// coef[:, j] = inv * xts[:, c0 + j]
std::vector<double> coefs(const NullFit& f, const std::vector<double>& xts, int64_t p, int64_t ldc,
                          int64_t c0, int64_t k) {
    std::vector<double> c(p * k, 0.0);
    for (int64_t j = 0; j < k; ++j)
        for (int64_t a = 0; a < p; ++a) {
            double acc = 0.0;
            for (int64_t b = 0; b < p; ++b) acc += f.inv[a + b * p] * xts[b + (c0 + j) * ldc];
            c[a + j * p] = acc;
        }
    return c;
}

// Eigen LDLT solve of the 3x3 AI system as the reference uses it: a zero pivot (the absent
// permanent-environment component) contributes a zero step.
bool solve_ai(const double AI[3][3], const double g[3], double out[3]) {
    int idx[3], k = 0;
    for (int i = 0; i < 3; ++i)
        if (AI[i][i] != 0.0) idx[k++] = i;
    out[0] = out[1] = out[2] = 0.0;
    std::vector<double> A(k * k), L, D;
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) A[a + b * k] = AI[idx[a]][idx[b]];
    if (!la::ldlt(A, k, L, D)) return false;
    std::vector<double> r(k);
    for (int a = 0; a < k; ++a) r[a] = g[idx[a]];
    la::ldlt_solve(L, D, k, r.data());
    for (int a = 0; a < k; ++a) out[idx[a]] = r[a];
    return true;
}

}  // namespace

void vce_default_options(cs_vce_options* o) {
    o->max_iter = 50;
    o->tol = 1e-6;
    o->mc_samples = 20;
    o->pcg_tol = 1e-10;
    o->pcg_relative = 0;
    o->pcg_max_iter = 2000;
    o->slq_probes = 30;
    o->slq_steps = 15;
    o->probe_seed = 20250101ull;
    o->precision = CS_PRECISION_FP64;
    o->precond_rank = 0;
}

cs_vce* vce_create() {
    auto* v = new cs_vce();
    try {
        v->blas = shared_blas();
    } catch (...) {
        delete v;
        throw;
    }
    return v;
}

// Stochastic Lanczos quadrature for log|V| (libCosmicCore/src/slq_estimator.cpp:11-106), all
// probes advancing together; the probes come from one mt19937_64(seed) stream, i.e. the
// estimator's schedule with one OpenMP thread.
static double slq_logdet(cs_vce* v, int probes, int steps, uint64_t seed, cudaStream_t s) {
    const int64_t n = v->rm.n_rec;
    const int m = (int)std::min<int64_t>(steps, n);
    const int64_t k = probes;
    v->lz.resize((int64_t)(m + 1) * n * k);
    v->lw.resize(n * k);
    auto Vj = [&](int j) { return v->lz.get() + (int64_t)j * n * k; };
    v->slq_rng.seed(seed, s);
    v->slq_rng.draw(n, k, v->lw.get(), k, s);
    std::vector<double> inv(k, 1.0 / std::sqrt((double)n));
    DeviceBuffer<double> dcoef;
    dcoef.resize(k);
    CS_CUDA(cudaMemcpyAsync(dcoef.get(), inv.data(), 8 * k, cudaMemcpyHostToDevice, s));
    k_scale_cols<<<grid_1d(n * k), 256, 0, s>>>(Vj(0), v->lw.get(), k, n, k, dcoef.get(), 0);
    CS_LAUNCH("scale_cols");
    std::vector<std::vector<double>> alpha(k, std::vector<double>(m, 0.0)), beta(k, std::vector<double>(m, 0.0));
    std::vector<int> actual(k, m);
    std::vector<char> done(k, 0);
    std::vector<double> coef(k), dots(k);
    auto axpy = [&](const double* Vm, const std::vector<double>& c) {
        CS_CUDA(cudaMemcpyAsync(dcoef.get(), c.data(), 8 * k, cudaMemcpyHostToDevice, s));
        k_axpy_cols<<<grid_1d(n * k), 256, 0, s>>>(v->lw.get(), Vm, k, n, k, dcoef.get());
        CS_LAUNCH("axpy_cols");
    };
    for (int j = 0; j < m; ++j) {
        v->V.apply(Vj(j), k, k, v->lw.get(), k, s);
        if (j > 0) {
            for (int64_t c = 0; c < k; ++c) coef[c] = done[c] ? 0.0 : beta[c][j - 1];
            axpy(Vj(j - 1), coef);
        }
        column_dots(v->lw.get(), k, Vj(j), k, n, k, dots.data(), v->pw, s);
        for (int64_t c = 0; c < k; ++c) {
            if (!done[c]) alpha[c][j] = dots[c];
            coef[c] = done[c] ? 0.0 : dots[c];
        }
        axpy(Vj(j), coef);
        // full reorthogonalisation
        for (int q = 0; q <= j; ++q) {
            column_dots(v->lw.get(), k, Vj(q), k, n, k, dots.data(), v->pw, s);
            for (int64_t c = 0; c < k; ++c) coef[c] = done[c] ? 0.0 : dots[c];
            axpy(Vj(q), coef);
        }
        column_dots(v->lw.get(), k, v->lw.get(), k, n, k, dots.data(), v->pw, s);
        for (int64_t c = 0; c < k; ++c) {
            if (done[c]) {
                coef[c] = 0.0;
                continue;
            }
            beta[c][j] = std::sqrt(dots[c]);
            if (beta[c][j] < 1e-12) {
                actual[c] = j + 1;
                done[c] = 1;
                coef[c] = 0.0;
            } else {
                coef[c] = beta[c][j];
            }
        }
        if (j + 1 <= m) {
            CS_CUDA(cudaMemcpyAsync(dcoef.get(), coef.data(), 8 * k, cudaMemcpyHostToDevice, s));
            k_scale_cols<<<grid_1d(n * k), 256, 0, s>>>(Vj(j + 1), v->lw.get(), k, n, k, dcoef.get(), 1);
            CS_LAUNCH("scale_cols");
        }
    }
    CS_CUDA(cudaStreamSynchronize(s));
    double total = 0.0;
    for (int64_t c = 0; c < k; ++c) {
        const int a = actual[c];
        std::vector<double> T(a * a, 0.0), ev, vec;
        for (int j = 0; j < a; ++j) {
            T[j + j * a] = alpha[c][j];
            if (j + 1 < a) T[(j + 1) + j * a] = T[j + (j + 1) * a] = beta[c][j];
        }
        if (!la::eigh(T, a, ev, vec)) fail(CS_ERR_NUMERIC, "SLQ tridiagonal eigensolver failed");
        double ss = 0.0;
        for (int i = 0; i < a; ++i) ss += vec[0 + i * a] * vec[0 + i * a] * std::log(std::max(ev[i], 1e-12));
        total += (double)n * ss;
    }
    return total / (double)probes;
}

void vce_solve_stcg(cs_vce* v, cs_kinship* op, double divisor, const int32_t* rec_to_row,
                    int64_t n_rec, int with_pe, const double* y, const double* X, int64_t p,
                    const cs_vce_options* opt_in, cs_vce_result* res) {
    const auto t_start = std::chrono::steady_clock::now();
    v->blas = shared_blas();  // the calling thread's handle
    cs_vce_options opt;
    if (opt_in) opt = *opt_in;
    else vce_default_options(&opt);
    if (n_rec <= 0 || p < 0 || (p > 0 && X == nullptr) || y == nullptr)
        fail(CS_ERR_INVALID_ARGUMENT, "STCG_VCE: bad dimensions");
    if (opt.mc_samples < 1 || opt.max_iter < 0 || opt.pcg_max_iter < 1)
        fail(CS_ERR_INVALID_ARGUMENT, "STCG_VCE: bad options");
    if (!(divisor > 0.0)) divisor = (double)op->num_variants;
    if (op->num_variants <= 0) fail(CS_ERR_INVALID_ARGUMENT, "STCG_VCE requires a genotype matrix component.");
    cudaStream_t s = 0;
    v->solved = false;
    v->p = p;
    v->n_rows = op->rows;
    v->rm.build(rec_to_row, n_rec, op->rows);
    v->hist.clear();
    cs::VOperator& V = v->V;
    V.op = op;
    V.rm = &v->rm;
    V.fac = (double)op->num_variants / divisor;
    V.with_pe = with_pe != 0;
    V.precision = opt.precision;
    V.applies = V.apply_cols = 0;
    const int64_t n = n_rec, S = opt.mc_samples;
    const int64_t kA = 1 + p + S;
    // ---- moment-based starting values (stcg_vce.cpp:157-214)
    int64_t n_ind = 0;
    for (int64_t i = 0; i < n; ++i) n_ind = std::max<int64_t>(n_ind, (rec_to_row ? rec_to_row[i] : i) + 1);
    double mean_y = 0.0;
    for (int64_t i = 0; i < n; ++i) mean_y += y[i];
    mean_y /= (double)n;
    double var_y = 0.0;
    for (int64_t i = 0; i < n; ++i) var_y += (y[i] - mean_y) * (y[i] - mean_y);
    var_y /= (double)std::max<int64_t>(1, n - 1);
    const double var_floor = std::max(1e-10, var_y * 1e-6);
    std::vector<double> sum_y(n_ind, 0.0), sumsq_y(n_ind, 0.0);
    std::vector<int> cnt_y(n_ind, 0);
    for (int64_t i = 0; i < n; ++i) {
        const int64_t idx = rec_to_row ? rec_to_row[i] : i;
        if (idx >= 0 && idx < n_ind) {
            sum_y[idx] += y[i];
            sumsq_y[idx] += y[i] * y[i];
            cnt_y[idx] += 1;
        }
    }
    double within_ss = 0.0, avg_n = 0.0;
    int within_df = 0;
    std::vector<double> subj_means;
    for (int64_t i = 0; i < n_ind; ++i) {
        if (cnt_y[i] <= 0) continue;
        const double mi = sum_y[i] / cnt_y[i];
        subj_means.push_back(mi);
        avg_n += cnt_y[i];
        if (cnt_y[i] > 1) {
            within_ss += sumsq_y[i] - cnt_y[i] * mi * mi;
            within_df += cnt_y[i] - 1;
        }
    }
    avg_n = subj_means.empty() ? 1.0 : (avg_n / subj_means.size());
    const double within_var = within_df > 0 ? within_ss / within_df : 0.5 * var_y;
    double subj_mean = 0.0;
    for (double m : subj_means) subj_mean += m;
    subj_mean /= (double)std::max<size_t>(1, subj_means.size());
    double between_var = 0.0;
    for (double m : subj_means) between_var += (m - subj_mean) * (m - subj_mean);
    between_var /= (double)std::max<int>(1, (int)subj_means.size() - 1);
    const double rep_guess = std::max(var_floor, between_var - within_var / std::max(1.0, avg_n));
    double pe_guess = std::max(var_floor, 0.35 * within_var);
    double ve_guess = std::max(var_floor, within_var - pe_guess);
    double vg_guess = std::max(var_floor, rep_guess);
    const double total_guess = vg_guess + pe_guess + ve_guess;
    if (total_guess > 0.0 && var_y > var_floor) {
        const double scale = var_y / total_guess;
        vg_guess *= scale;
        pe_guess *= scale;
        ve_guess *= scale;
    }
    V.ve = ve_guess;
    V.vg = vg_guess;
    V.vpe = V.with_pe ? pe_guess : 0.0;

    // ---- optional low-rank deflation preconditioner (records one-to-one with rows)
    cs::LowRankPreconditioner* M = nullptr;
    if (opt.precond_rank > 0 && v->rm.identity) {
        const int rank = (int)std::min<int64_t>(opt.precond_rank, std::max<int64_t>(1, n - 2));
        prof::HostScope hs("stcg_precond_sketch");
        cs_lmm* l = lmm_create();
        try {
            LowRankTarget t;
            t.rows = n;
            t.trace = op->trace;  // of Z Z^T / num_variants; eigenvalues scaled by fac below
            const int prec = opt.precision;
            t.apply = [op, prec](const double* X_, int64_t ldx, int64_t k, double* Y_, int64_t ldy,
                                 cudaStream_t st2) {
                kinship_apply_rowmajor(op, X_, ldx, k, Y_, ldy, prec, st2);
            };
            std::vector<double> Xc(std::max<int64_t>(1, n * p));
            std::copy(X, X + n * p, Xc.begin());
            lmm_prepare_lowrank_target(l, t, y, p > 0 ? Xc.data() : nullptr, p, rank, 10, 42, 0.0,
                                       rank, nullptr, s);
            cs::LowRankPreconditioner& P = v->precond;
            P.n = n;
            P.r = lmm_rank(l);
            P.U.resize(n * P.r);
            CS_CUDA(cudaMemcpyAsync(P.U.get(), lmm_basis_device(l), 8 * n * P.r,
                                    cudaMemcpyDeviceToDevice, s));
            P.lambda = lmm_eigenvalues(l);
            for (double& x : P.lambda) x *= V.fac;
            P.r0 = lmm_residual_eigenvalue(l) * V.fac;
            CS_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            lmm_destroy(l);
            throw;
        }
        lmm_destroy(l);
        M = &v->precond;
    }
    auto set_precond = [&]() {
        if (M) M->set_components(V.vg, V.ve + (V.with_pe ? V.vpe : 0.0), s);
    };

    // ---- constant columns of the first block: [y | X | probes]
    v->rhsA.resize(n * kA);
    v->solA.resize(n * kA);
    {
        std::vector<double> h(n * (1 + p));
        for (int64_t i = 0; i < n; ++i) {
            h[i * (1 + p)] = y[i];
            for (int64_t a = 0; a < p; ++a) h[i * (1 + p) + 1 + a] = X[i + a * n];
        }
        CS_CUDA(cudaMemcpy2DAsync(v->rhsA.get(), 8 * kA, h.data(), 8 * (1 + p), 8 * (1 + p), n,
                                  cudaMemcpyHostToDevice, s));
    }
    v->probes.seed(opt.probe_seed, s);
    const int64_t kIn = 1 + S;
    const int64_t kB = V.with_pe ? 3 : 2;
    v->W.resize(n * kIn);
    v->IN.resize(n * kIn);
    v->DG.resize(n * kIn);
    if (V.with_pe) v->DP.resize(n * kIn);
    v->rhsB.resize(n * kB);
    v->solB.resize(n * kB);
    v->Q.resize(n * kB);
    auto diag_of = [&]() {
        double d = std::max(V.ve, 1e-12) + std::max(V.vg, 1e-12);
        if (V.with_pe) d += std::max(V.vpe, 1e-12);
        return d;
    };
    cs::PcgStats st;
    int64_t pcg_total = 0;
    double last[3] = {NAN, NAN, NAN};
    const int em_warmup = 4;
    const double min_f = 0.5, max_f = 2.0, blend = 0.35;
    res->converged = 0;
    res->iterations = 0;
    res->logl = std::numeric_limits<double>::quiet_NaN();
    for (int iter = 0; iter < opt.max_iter; ++iter) {
        const double diag = diag_of();
        set_precond();
        // ---- block A: V^-1 [y | X | z]
        v->probes.draw(n, S, v->rhsA.get() + 1 + p, kA, s);
        pcg_solve_block(V, diag, v->rhsA.get(), kA, kA, v->solA.get(), kA, opt.pcg_tol,
                        opt.pcg_relative != 0, opt.pcg_max_iter, v->pw, st, s, M);
        pcg_total += st.column_iterations;
        // X^T [V^-1 y | V^-1 X | V^-1 z]
        const std::vector<double> xts =
            cross(v->blas, v->rhsA.get(), kA, 1, p, v->solA.get(), kA, 0, kA, n, v->small, s);
        NullFit nf = null_fit(xts, p, p);
        if (!nf.ok) fail(CS_ERR_NUMERIC, "STCG_VCE: X' V^-1 X is not positive definite");
        // W = [Py | P z_1 .. P z_S]
        {
            std::vector<double> cm(p * kIn);
            const std::vector<double> cz = coefs(nf, xts, p, p, 1 + p, S);
            for (int64_t a = 0; a < p; ++a) cm[a] = nf.beta[a];
            std::copy(cz.begin(), cz.end(), cm.begin() + p);
            copy_cols(v->solA.get(), kA, n, 0, 1, v->W.get(), kIn, 0, s);
            copy_cols(v->solA.get(), kA, n, 1 + p, S, v->W.get(), kIn, 1, s);
            if (p > 0) {
                v->cm.resize(p * kIn);
                CS_CUDA(cudaMemcpyAsync(v->cm.get(), cm.data(), 8 * p * kIn, cudaMemcpyHostToDevice, s));
                const double mone = -1.0, one = 1.0;
                CS_BLAS(cublasSetStream(v->blas, s));
                CS_BLAS(cublasDgemm(v->blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)kIn, (int)n, (int)p, &mone,
                                    v->cm.get(), (int)p, v->solA.get() + 1, (int)kA, &one, v->W.get(),
                                    (int)kIn));
            }
        }
        // derivatives on [Py | z]
        copy_cols(v->W.get(), kIn, n, 0, 1, v->IN.get(), kIn, 0, s);
        copy_cols(v->rhsA.get(), kA, n, 1 + p, S, v->IN.get(), kIn, 1, s);
        V.derivatives(v->IN.get(), kIn, kIn, v->DG.get(), kIn, V.with_pe ? v->DP.get() : nullptr,
                      kIn, s);
        // ---- block B: q_k = P s_k, s = [dVg Py | dVpe Py | Py]
        copy_cols(v->DG.get(), kIn, n, 0, 1, v->rhsB.get(), kB, 0, s);
        if (V.with_pe) copy_cols(v->DP.get(), kIn, n, 0, 1, v->rhsB.get(), kB, 1, s);
        copy_cols(v->W.get(), kIn, n, 0, 1, v->rhsB.get(), kB, kB - 1, s);
        pcg_solve_block(V, diag, v->rhsB.get(), kB, kB, v->solB.get(), kB, opt.pcg_tol,
                        opt.pcg_relative != 0, opt.pcg_max_iter, v->pw, st, s, M);
        pcg_total += st.column_iterations;
        {
            const std::vector<double> xtb =
                cross(v->blas, v->rhsA.get(), kA, 1, p, v->solB.get(), kB, 0, kB, n, v->small, s);
            const std::vector<double> cb = p > 0 ? coefs(nf, xtb, p, p, 0, kB) : std::vector<double>();
            project(v->blas, v->solB.get(), kB, 0, kB, v->solA.get() + 1, kA, p, cb, v->Q.get(), kB,
                    0, n, v->cm, s);
        }
        // ---- traces, quadratic forms, AI
        double tr[3] = {0.0, 0.0, 0.0};
        {
            std::vector<double> d(S);
            column_dots(v->W.get() + 1, kIn, v->DG.get() + 1, kIn, n, S, d.data(), v->pw, s);
            for (int64_t t = 0; t < S; ++t) tr[0] += d[t];
            if (V.with_pe) {
                column_dots(v->W.get() + 1, kIn, v->DP.get() + 1, kIn, n, S, d.data(), v->pw, s);
                for (int64_t t = 0; t < S; ++t) tr[1] += d[t];
            }
            column_dots(v->W.get() + 1, kIn, v->rhsA.get() + 1 + p, kA, n, S, d.data(), v->pw, s);
            for (int64_t t = 0; t < S; ++t) tr[2] += d[t];
            for (double& t : tr) t /= (double)S;
        }
        // s^T [Py-row] and s^T q over the B columns (index map: 0 -> g, pe -> 1, Py -> 2)
        const std::vector<double> sq =
            cross(v->blas, v->rhsB.get(), kB, 0, kB, v->Q.get(), kB, 0, kB, n, v->small, s);
        const std::vector<double> spy =
            cross(v->blas, v->rhsB.get(), kB, 0, kB, v->W.get(), kIn, 0, 1, n, v->small, s);
        int comp_col[3] = {0, V.with_pe ? 1 : -1, (int)kB - 1};
        double quad[3], grad[3], AI[3][3];
        for (int a = 0; a < 3; ++a) {
            quad[a] = comp_col[a] >= 0 ? spy[comp_col[a]] : 0.0;
            grad[a] = 0.5 * (quad[a] - tr[a]);
        }
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b) {
                const double val = (comp_col[a] >= 0 && comp_col[b] >= 0)
                                       ? 0.5 * sq[comp_col[a] + comp_col[b] * kB]
                                       : 0.0;
                AI[a][b] = AI[b][a] = val;
            }
        const double theta[3] = {V.vg, V.with_pe ? V.vpe : 0.0, V.ve};
        double next[3] = {theta[0], theta[1], theta[2]};
        bool em = iter < em_warmup;
        if (!em) {
            double delta[3];
            if (solve_ai(AI, grad, delta) && std::isfinite(delta[0]) && std::isfinite(delta[1]) &&
                std::isfinite(delta[2])) {
                for (int k = 0; k < 3; ++k) {
                    const double lo = std::max(var_floor, theta[k] * min_f);
                    const double hi = std::max(lo, theta[k] * max_f);
                    next[k] = std::max(lo, std::min(hi, theta[k] + blend * delta[k]));
                }
            } else {
                em = true;
            }
        }
        if (em) {
            for (int k = 0; k < 3; ++k) {
                const double denom = std::max(tr[k], var_floor);
                double target = quad[k] / denom;
                if (!std::isfinite(target) || target < 0.0) target = theta[k];
                const double lo = std::max(var_floor, theta[k] * min_f);
                const double hi = std::max(lo, theta[k] * max_f);
                next[k] = std::max(lo, std::min(hi, target));
            }
        }
        for (double& x : next) x = std::max(var_floor, x);
        // ---- REML log-likelihood at the current theta (stcg_vce.cpp:330-348)
        double logl = std::numeric_limits<double>::quiet_NaN();
        if (opt.slq_probes > 0) {
            const double logdetV = slq_logdet(v, opt.slq_probes, opt.slq_steps, 42ull + (uint64_t)iter, s);
            double logdetX = 0.0;
            for (int64_t a = 0; a < p; ++a) logdetX += std::log(nf.D[a]);
            const std::vector<double> ypy =
                cross(v->blas, v->rhsA.get(), kA, 0, 1, v->W.get(), kIn, 0, 1, n, v->small, s);
            logl = -0.5 * (logdetV + logdetX + ypy[0] + (double)(n - p) * std::log(2 * M_PI));
            res->logl = logl;
        }
        double rel = 0.0;
        if (iter > 0 && std::isfinite(last[0]) && std::isfinite(last[1]) && std::isfinite(last[2]))
            for (int k = 0; k < 3; ++k)
                rel = std::max(rel, std::abs(next[k] - last[k]) / (std::abs(last[k]) + 1e-12));
        for (int k = 0; k < 3; ++k) last[k] = next[k];
        V.vg = next[0];
        if (V.with_pe) V.vpe = next[1];
        V.ve = next[2];
        v->hist.insert(v->hist.end(), {next[0], V.with_pe ? next[1] : 0.0, next[2], logl, em ? 0.0 : 1.0});
        res->iterations = iter + 1;
        if (iter > 0 && rel < opt.tol) {
            res->converged = 1;
            break;
        }
    }
    // ---- final BLUE / BLUP (stcg_vce.cpp:364-406)
    {
        const double diag = diag_of();
        set_precond();
        const int64_t k0 = 1 + p;
        pcg_solve_block(V, diag, v->rhsA.get(), kA, k0, v->solA.get(), kA, opt.pcg_tol,
                        opt.pcg_relative != 0, opt.pcg_max_iter, v->pw, st, s, M);
        pcg_total += st.column_iterations;
        const std::vector<double> xts =
            cross(v->blas, v->rhsA.get(), kA, 1, p, v->solA.get(), kA, 0, k0, n, v->small, s);
        NullFit nf = null_fit(xts, p, p);
        if (!nf.ok) fail(CS_ERR_NUMERIC, "STCG_VCE: X' V^-1 X is not positive definite");
        project(v->blas, v->solA.get(), kA, 0, 1, v->solA.get() + 1, kA, p, nf.beta, v->W.get(), kIn,
                0, n, v->cm, s);
        const int64_t nr = v->n_rows;
        DeviceBuffer<double> rows, zt;
        rows.resize(nr);
        zt.resize(nr);
        V.genetic_rows(v->W.get(), kIn, 1, rows.get(), 1, zt.get(), 1, s);
        v->a_rows.assign(nr, 0.0);
        v->pe_rows.assign(nr, 0.0);
        std::vector<double> zh(nr);
        CS_CUDA(cudaMemcpyAsync(v->a_rows.data(), rows.get(), 8 * nr, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaMemcpyAsync(zh.data(), zt.get(), 8 * nr, cudaMemcpyDeviceToHost, s));
        CS_CUDA(cudaStreamSynchronize(s));
        for (int64_t i = 0; i < nr; ++i) {
            v->a_rows[i] *= V.vg;
            v->pe_rows[i] = V.with_pe ? V.vpe * zh[i] : 0.0;
        }
        v->beta = nf.beta;
    }
    res->sigma2_g = V.vg;
    res->sigma2_pe = V.with_pe ? V.vpe : 0.0;
    res->sigma2_e = V.ve;
    res->pcg_iterations = pcg_total;
    res->operator_applies = V.applies;
    res->operator_columns = V.apply_cols;
    res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    v->solved = true;
}

void vce_destroy(cs_vce* v) { delete v; }

void vce_solution(const cs_vce* v, double* beta, double* a_rows, double* pe_rows) {
    if (!v->solved) fail(CS_ERR_INVALID_ARGUMENT, "STCG_VCE: solve() has not run");
    if (beta) std::copy(v->beta.begin(), v->beta.end(), beta);
    if (a_rows) std::copy(v->a_rows.begin(), v->a_rows.end(), a_rows);
    if (pe_rows) std::copy(v->pe_rows.begin(), v->pe_rows.end(), pe_rows);
}

void vce_history(const cs_vce* v, double* out, int64_t* n_iter) {
    const int64_t it = (int64_t)v->hist.size() / 5;
    if (n_iter) *n_iter = it;
    if (out) std::copy(v->hist.begin(), v->hist.end(), out);
}

// Public multi-RHS solve of (sg2 K + se2 I) X = B on device column-major blocks.
void pcg_solve_public(cs_kinship* op, double divisor, double sg2, double se2, const double* B,
                      int64_t ldb, int64_t k, double* X, int64_t ldx, double tol, int relative,
                      int max_iter, int precision, int32_t* iterations, cudaStream_t s) {
    if (k < 0 || ldb < op->rows || ldx < op->rows || max_iter < 1)
        fail(CS_ERR_INVALID_ARGUMENT, "MatrixFreePCG: bad dimensions");
    if (k == 0) return;
    if (!(divisor > 0.0)) divisor = (double)op->num_variants;
    const int64_t n = op->rows;
    RecordMap rm;
    rm.build(nullptr, n, n);
    VOperator V;
    V.op = op;
    V.rm = &rm;
    V.fac = (double)op->num_variants / divisor;
    V.vg = sg2;
    V.ve = se2;
    V.precision = precision;
    PcgWorkspace ws;
    PcgStats st;
    DeviceBuffer<double> b, x;
    b.resize(n * k);
    x.resize(n * k);
    colmajor_to_rowmajor(B, ldb, n, k, b.get(), k, s);
    const double diag = std::max(se2, 1e-12) + std::max(sg2, 1e-12);
    pcg_solve_block(V, diag, b.get(), k, k, x.get(), k, tol, relative != 0, max_iter, ws, st, s);
    rowmajor_to_colmajor(x.get(), k, n, k, X, ldx, s);
    CS_CUDA(cudaStreamSynchronize(s));
    if (iterations) std::copy(st.iterations.begin(), st.iterations.end(), iterations);
}

// The record-level covariance of STCG_VCE (stcg_vce.cpp:80-126) behind MatrixFreePCG.
void pcg_solve_records_public(cs_kinship* op, double divisor, const int32_t* rec_to_row,
                              int64_t n_rec, bool with_pe, double sg2, double spe2, double se2,
                              const double* B, int64_t ldb, int64_t k, double* X, int64_t ldx,
                              double tol, int relative, int max_iter, int precision,
                              int32_t* iterations, cudaStream_t s) {
    if (!rec_to_row) n_rec = op->rows;
    if (k < 0 || n_rec <= 0 || ldb < n_rec || ldx < n_rec || max_iter < 1)
        fail(CS_ERR_INVALID_ARGUMENT, "MatrixFreePCG: bad dimensions");
    if (k == 0) return;
    if (!(divisor > 0.0)) divisor = (double)op->num_variants;
    RecordMap rm;
    rm.build(rec_to_row, n_rec, op->rows);
    VOperator V;
    V.op = op;
    V.rm = &rm;
    V.fac = (double)op->num_variants / divisor;
    V.vg = sg2;
    V.vpe = with_pe ? spe2 : 0.0;
    V.ve = se2;
    V.with_pe = with_pe;
    V.precision = precision;
    PcgWorkspace ws;
    PcgStats st;
    DeviceBuffer<double> b, x;
    b.resize(n_rec * k);
    x.resize(n_rec * k);
    colmajor_to_rowmajor(B, ldb, n_rec, k, b.get(), k, s);
    double diag = std::max(se2, 1e-12) + std::max(sg2, 1e-12);
    if (with_pe) diag += std::max(spe2, 1e-12);
    pcg_solve_block(V, diag, b.get(), k, k, x.get(), k, tol, relative != 0, max_iter, ws, st, s);
    rowmajor_to_colmajor(x.get(), k, n_rec, k, X, ldx, s);
    CS_CUDA(cudaStreamSynchronize(s));
    if (iterations) std::copy(st.iterations.begin(), st.iterations.end(), iterations);
}

}  // namespace cs
