// Multi-trait dense null model: MvEigenVce (libCosmicCore/src/eigen_vce.cpp:496-911, 1031-1065)
// on the eigenbasis of dense.cu, and the mvLMM scan from it (MvLmmEngine::prepareFromVce +
// scan, src/mvlmm_engine.cpp:195-207, 756-931).
//
//   prepare        MvEigenVce::prepare (:496-549): eigenbasis of G[keep, keep] (covariate
//                  projection by default), U^T Y, Vg = Ve = Cov(Y) / 2
//   run_null       runNullModel (:1031-1065): EM (updateEM, :551-604) until the mean squared
//                  change falls below tol, or runAireml (:631-911): EM warm-up, positive-
//                  definite clipping, AI-REML steps with step halving on the REML
//                  log-likelihood (:613-629), fall-back to the EM estimate, SEs from the AI
//                  matrix
//
// Device work: the per-sample d x d algebra of every EM iteration and every log-likelihood
// (one thread per eigen-sample, d <= 8: Cholesky of V_i = D_i Vg + Ve, its inverse, the EM
// moment sums), reduced per block and summed on the host in block order.  Host work: the
// d x d updates, the AI-REML score / information (O(n d (d(d+1)/2)^2) per iteration, opt-in).
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <memory>
#include <utility>
#include <vector>

#include "cs_internal.h"
#include "dense_internal.h"
#include "linalg_host.h"
#include "vce_internal.h"

namespace cs {

constexpr int kMvMaxTraits = 8;

struct MvParams {
    int d;
    double Vg[kMvMaxTraits * kMvMaxTraits];
    double Ve[kMvMaxTraits * kMvMaxTraits];
};

namespace {

// Lower Cholesky factor of A (d x d, column-major) in place; false if a pivot is not positive.
__device__ bool chol_lower(double* A, int d) {
    for (int j = 0; j < d; ++j) {
        double s = A[j + j * d];
        for (int k = 0; k < j; ++k) s -= A[j + k * d] * A[j + k * d];
        if (!(s > 0.0)) return false;
        const double l = sqrt(s);
        A[j + j * d] = l;
        for (int i = j + 1; i < d; ++i) {
            double t = A[i + j * d];
            for (int k = 0; k < j; ++k) t -= A[i + k * d] * A[j + k * d];
            A[i + j * d] = t / l;
        }
    }
    return true;
}

// Per eigen-sample work, reduced per block into partial[block * E + e]:
//   mode 0 (EM, updateEM :560-595, no covariates left):  E = 2 d^2,
//       S_g += (u u' / D_i + Vg - W_g Vg) (D_i > 1e-12) else Vg,  W_g = D_i Vg V_i^-1, u = W_g y_i
//       S_e += e e' + Ve - W_e Ve,  W_e = Ve V_i^-1, e = W_e y_i
//   mode 1 (calcLogLikelihood :613-629): E = 2, sum of -0.5 (log|V_i| + y_i' V_i^-1 y_i) with
//       V_i = D_i Vg + Ve + 1e-8 I, and the count of samples whose V_i is not positive definite
__global__ void k_mv_per_sample(const double* __restrict__ D, const double* __restrict__ Y,
                                int64_t n, MvParams P, int mode, double* __restrict__ partial) {
    constexpr int kM = kMvMaxTraits * kMvMaxTraits;
    const int d = P.d, dd = d * d;
    const int E = mode == 0 ? 2 * dd : 2;
    double acc[2 * kM];
    for (int e = 0; e < E; ++e) acc[e] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double di = D[i];
        double L[kM], y[kMvMaxTraits];
        for (int a = 0; a < d; ++a) y[a] = Y[i + a * n];
        for (int e = 0; e < dd; ++e) L[e] = di * P.Vg[e] + P.Ve[e];
        if (mode == 1)
            for (int a = 0; a < d; ++a) L[a + a * d] += 1e-8;
        if (!chol_lower(L, d)) {
            if (mode == 1) {
                acc[1] += 1.0;
            } else {
                acc[0] = nan("");
            }
            continue;
        }
        if (mode == 1) {
            double ldet = 0.0, quad = 0.0, z[kMvMaxTraits];
            for (int a = 0; a < d; ++a) {
                double t = y[a];
                for (int k = 0; k < a; ++k) t -= L[a + k * d] * z[k];
                z[a] = t / L[a + a * d];
                quad += z[a] * z[a];
                ldet += 2.0 * log(L[a + a * d]);
            }
            acc[0] += -0.5 * (ldet + quad);
            continue;
        }
        // V^-1 = L^-T L^-1: Linv (lower) first
        double Li[kM], Pm[kM];
        for (int e = 0; e < dd; ++e) Li[e] = 0.0;
        for (int j = 0; j < d; ++j) {
            Li[j + j * d] = 1.0 / L[j + j * d];
            for (int i2 = j + 1; i2 < d; ++i2) {
                double t = 0.0;
                for (int k = j; k < i2; ++k) t -= L[i2 + k * d] * Li[k + j * d];
                Li[i2 + j * d] = t / L[i2 + i2 * d];
            }
        }
        for (int a = 0; a < d; ++a)
            for (int b = 0; b < d; ++b) {
                double t = 0.0;
                for (int k = max(a, b); k < d; ++k) t += Li[k + a * d] * Li[k + b * d];
                Pm[a + b * d] = t;
            }
        // W_g = D_i Vg P, u = W_g y; W_e = Ve P, e = W_e y (Li reused as W)
        double u[kMvMaxTraits];
        for (int a = 0; a < d; ++a)
            for (int b = 0; b < d; ++b) {
                double t = 0.0;
                for (int k = 0; k < d; ++k) t += P.Vg[a + k * d] * Pm[k + b * d];
                Li[a + b * d] = di * t;
            }
        for (int a = 0; a < d; ++a) {
            double t = 0.0;
            for (int k = 0; k < d; ++k) t += Li[a + k * d] * y[k];
            u[a] = t;
        }
        if (di > 1e-12) {
            for (int a = 0; a < d; ++a)
                for (int b = 0; b < d; ++b) {
                    double wv = 0.0;
                    for (int k = 0; k < d; ++k) wv += Li[a + k * d] * P.Vg[k + b * d];
                    acc[a + b * d] += u[a] * u[b] / di + P.Vg[a + b * d] - wv;
                }
        } else {
            for (int e = 0; e < dd; ++e) acc[e] += P.Vg[e];
        }
        for (int a = 0; a < d; ++a)
            for (int b = 0; b < d; ++b) {
                double t = 0.0;
                for (int k = 0; k < d; ++k) t += P.Ve[a + k * d] * Pm[k + b * d];
                Li[a + b * d] = t;
            }
        for (int a = 0; a < d; ++a) {
            double t = 0.0;
            for (int k = 0; k < d; ++k) t += Li[a + k * d] * y[k];
            u[a] = t;
        }
        for (int a = 0; a < d; ++a)
            for (int b = 0; b < d; ++b) {
                double wv = 0.0;
                for (int k = 0; k < d; ++k) wv += Li[a + k * d] * P.Ve[k + b * d];
                acc[dd + a + b * d] += u[a] * u[b] + P.Ve[a + b * d] - wv;
            }
    }
    __shared__ double red[8][2 * kM];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int e = 0; e < E; ++e) {
        double v = acc[e];
        for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[warp][e] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < E; e += blockDim.x) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][e];
        partial[blockIdx.x * (int64_t)E + e] = t;
    }
}

}  // namespace

}  // namespace cs

namespace cs {

namespace {

// Sums of the per-sample terms for (Vg, Ve): EM moments (2 d^2) or log-likelihood (2).
std::vector<double> mv_sums(cs_mv_eigen_vce* v, const std::vector<double>& Vg,
                            const std::vector<double>& Ve, int mode) {
    const int64_t n = v->d->n_eig, d = v->traits;
    MvParams P{};
    P.d = (int)d;
    std::copy(Vg.begin(), Vg.end(), P.Vg);
    std::copy(Ve.begin(), Ve.end(), P.Ve);
    const int E = mode == 0 ? (int)(2 * d * d) : 2;
    cudaStream_t s = 0;
    {
        prof::Scope ps(mode == 0 ? "mv_em_moments" : "mv_loglik", s, 0.0, 8.0 * n * (d + 1));
        k_mv_per_sample<<<v->blocks, 256, 0, s>>>(v->dD.get(), v->dY.get(), n, P, mode,
                                                  v->partial.get());
        CS_LAUNCH("mv_per_sample");
    }
    std::vector<double> h((size_t)v->blocks * E), out(E, 0.0);
    CS_CUDA(cudaMemcpyAsync(h.data(), v->partial.get(), 8 * h.size(), cudaMemcpyDeviceToHost, s));
    CS_CUDA(cudaStreamSynchronize(s));
    for (int b = 0; b < v->blocks; ++b)
        for (int e = 0; e < E; ++e) out[e] += h[(size_t)b * E + e];
    return out;
}

double mv_loglik(cs_mv_eigen_vce* v, const std::vector<double>& Vg, const std::vector<double>& Ve) {
    const std::vector<double> r = mv_sums(v, Vg, Ve, 1);
    if (r[1] > 0.0) return -std::numeric_limits<double>::infinity();
    return r[0];
}

// One EM update (updateEM): returns the mean squared change.
double mv_em_step(cs_mv_eigen_vce* v) {
    const int64_t n = v->d->n_eig, d = v->traits;
    const std::vector<double> S = mv_sums(v, v->Vg, v->Ve, 0);
    std::vector<double> Vg_new(d * d), Ve_new(d * d);
    for (int64_t e = 0; e < d * d; ++e) {
        Vg_new[e] = S[e] / (double)n;
        Ve_new[e] = S[d * d + e] / (double)n;
    }
    for (double x : S)
        if (!std::isfinite(x))
            fail(CS_ERR_NUMERIC, "MvEigenVce: a sample covariance is not positive definite");
    double err = 0.0;
    for (int64_t e = 0; e < d * d; ++e) {
        err += (Vg_new[e] - v->Vg[e]) * (Vg_new[e] - v->Vg[e]);
        err += (Ve_new[e] - v->Ve[e]) * (Ve_new[e] - v->Ve[e]);
    }
    err /= std::max(1.0, 2.0 * (double)(d * d));
    v->Vg = Vg_new;
    v->Ve = Ve_new;
    return err;
}

// Eigenvalue clipping at 1e-10 when the smallest is not above it (runAireml's nearPD).
void near_pd(std::vector<double>& M, int d) {
    std::vector<double> ev, Q;
    if (!la::eigh(M, d, ev, Q)) fail(CS_ERR_NUMERIC, "MvEigenVce: eigensolver failed");
    if (*std::min_element(ev.begin(), ev.end()) > 1e-10) return;
    for (double& x : ev) x = std::max(x, 1e-10);
    for (int a = 0; a < d; ++a)
        for (int b = 0; b < d; ++b) {
            double t = 0.0;
            for (int k = 0; k < d; ++k) t += Q[a + k * d] * ev[k] * Q[b + k * d];
            M[a + b * d] = t;
        }
}

// Score and AI matrix of runAireml (:688-739) over every eigen-sample, on the host.
bool mv_score_ai(const DenseNull& dn, int64_t d, const std::vector<double>& Vg,
                 const std::vector<double>& Ve, const std::vector<std::pair<int, int>>& pairs,
                 std::vector<double>& score, std::vector<double>& AI) {
    const int64_t n = dn.n_eig, vs = (int64_t)pairs.size(), np = 2 * vs;
    score.assign(np, 0.0);
    AI.assign(np * np, 0.0);
    std::vector<double> V(d * d), L, Dl, Vinv, v(d), w(vs * d);
    for (int64_t i = 0; i < n; ++i) {
        const double di = dn.D[i], d2 = di * di;
        for (int64_t e = 0; e < d * d; ++e) V[e] = di * Vg[e] + Ve[e];
        for (int64_t a = 0; a < d; ++a) V[a + a * d] += 1e-8;
        if (!la::ldlt(V, (int)d, L, Dl)) return false;
        Vinv = la::ldlt_inverse(L, Dl, (int)d);
        for (int64_t a = 0; a < d; ++a) {
            double t = 0.0;
            for (int64_t b = 0; b < d; ++b) t += Vinv[a + b * d] * dn.Uty[i + b * n];
            v[a] = t;
        }
        for (int64_t a = 0; a < vs; ++a) {
            const int p = pairs[a].first, q = pairs[a].second;
            for (int64_t r = 0; r < d; ++r)
                w[a * d + r] = p == q ? v[p] * Vinv[r + p * d]
                                      : v[q] * Vinv[r + p * d] + v[p] * Vinv[r + q * d];
        }
        for (int64_t a = 0; a < vs; ++a) {
            const int j = pairs[a].first, k = pairs[a].second;
            const double vjvk = v[j] * v[k];
            const double tr = j == k ? Vinv[j + j * d] : 2.0 * Vinv[j + k * d];
            const double quad = j == k ? vjvk : 2.0 * vjvk;
            score[a] += 0.5 * di * (quad - tr);
            score[a + vs] += 0.5 * (quad - tr);
        }
        for (int64_t a = 0; a < vs; ++a) {
            const int j = pairs[a].first, k = pairs[a].second;
            for (int64_t b = a; b < vs; ++b) {
                double qv = j == k ? v[j] * w[b * d + j] : v[j] * w[b * d + k] + v[k] * w[b * d + j];
                qv *= 0.5;
                AI[a + b * np] += d2 * qv;
                AI[a + (vs + b) * np] += di * qv;
                AI[(vs + a) + b * np] += di * qv;
                AI[(vs + a) + (vs + b) * np] += qv;
            }
        }
    }
    // symmetrise: the row-major upper-triangle accumulation of the reference, then 0.5 (A + A')
    std::vector<double> S(np * np);
    for (int64_t a = 0; a < np; ++a)
        for (int64_t b = 0; b < np; ++b) S[a + b * np] = 0.5 * (AI[a + b * np] + AI[b + a * np]);
    AI.swap(S);
    return true;
}

}  // namespace

cs_mv_eigen_vce* mv_prepare(const cs_grm* grm, const int32_t* keep, int64_t n_keep,
                            const double* Y, int64_t d, const double* X, int64_t p,
                            bool projection) {
    if (d < 1 || d > kMvMaxTraits)
        fail(CS_ERR_UNSUPPORTED, "MvEigenVce: 1 to 8 traits are supported");
    if (!projection && p > 0)
        fail(CS_ERR_UNSUPPORTED,
             "MvEigenVce: covariates without the covariate projection are not supported");
    auto basis = eigen_basis(grm, keep, n_keep, Y, d, X, p, projection);
    auto* v = new cs_mv_eigen_vce();
    try {
        v->d = std::move(basis);
        v->traits = d;
        const int64_t n = keep ? n_keep : grm->n;
        // Vg = Ve = Cov(Y) / 2 over the analysed samples, divided by (samples after the
        // projection - 1) as the reference does (:543-547)
        const int64_t n_after = v->d->n_eig;
        std::vector<double> mean(d, 0.0), cov(d * d, 0.0);
        for (int64_t a = 0; a < d; ++a) {
            for (int64_t i = 0; i < n; ++i) mean[a] += Y[i + a * n];
            mean[a] /= (double)n;
        }
        for (int64_t a = 0; a < d; ++a)
            for (int64_t b = 0; b < d; ++b) {
                double t = 0.0;
                for (int64_t i = 0; i < n; ++i) t += (Y[i + a * n] - mean[a]) * (Y[i + b * n] - mean[b]);
                cov[a + b * d] = t / (double)(n_after - 1);
            }
        v->Vg.resize(d * d);
        v->Ve.resize(d * d);
        for (int64_t e = 0; e < d * d; ++e) v->Vg[e] = v->Ve[e] = cov[e] * 0.5;
        const int64_t ne = v->d->n_eig;
        v->dD.resize(ne);
        v->dY.resize(ne * d);
        CS_CUDA(cudaMemcpy(v->dD.get(), v->d->D.data(), 8 * ne, cudaMemcpyHostToDevice));
        CS_CUDA(cudaMemcpy(v->dY.get(), v->d->Uty.data(), 8 * ne * d, cudaMemcpyHostToDevice));
        v->blocks = (int)std::max<int64_t>(1, std::min<int64_t>((ne + 255) / 256, 2LL * num_sms()));
        v->partial.resize((int64_t)v->blocks * 2 * kMvMaxTraits * kMvMaxTraits);
    } catch (...) {
        delete v;
        throw;
    }
    return v;
}

bool mv_run_null(cs_mv_eigen_vce* v, const cs_mv_vce_options* opt) {
    if (!v || !v->d) fail(CS_ERR_INVALID_ARGUMENT, "MvEigenVce: not prepared");
    cs_mv_vce_options o;
    cs_mv_vce_default_options(&o);
    if (opt) o = *opt;
    const int64_t d = v->traits;
    v->Vg_se.assign(d * d, 0.0);
    v->Ve_se.assign(d * d, 0.0);
    if (!o.aireml) {
        // runNullModel's EM branch (:1043-1063)
        for (int iter = 0; iter < o.max_iter; ++iter) {
            const double err = mv_em_step(v);
            v->iterations = iter + 1;
            if (err < o.tol) {
                v->converged = true;
                v->logl = mv_loglik(v, v->Vg, v->Ve);
                return true;
            }
        }
        v->converged = false;
        v->logl = mv_loglik(v, v->Vg, v->Ve);
        return false;
    }
    // runAireml (:631-911)
    std::vector<std::pair<int, int>> pairs;
    for (int j = 0; j < d; ++j)
        for (int k = j; k < d; ++k) pairs.emplace_back(j, k);
    const int64_t vs = (int64_t)pairs.size(), np = 2 * vs;
    int em_iter = 0;
    for (; em_iter < o.max_iter; ++em_iter) {
        const double err = mv_em_step(v);
        if (err < o.tol && em_iter >= o.em_min_iter) break;
    }
    v->iterations = std::min(em_iter + 1, o.max_iter);
    near_pd(v->Vg, (int)d);
    near_pd(v->Ve, (int)d);
    double logl_old = mv_loglik(v, v->Vg, v->Ve);
    const double logl_initial = logl_old;
    const std::vector<double> Vg_initial = v->Vg, Ve_initial = v->Ve;
    v->converged = true;
    if (!std::isfinite(logl_old)) {
        v->logl = logl_old;
        return true;  // the EM result stands
    }
    const double reg = 1e-8;
    bool done = false;
    for (int iter = 0; iter < o.ai_max_iter && !done; ++iter) {
        std::vector<double> score, AI;
        if (!mv_score_ai(*v->d, d, v->Vg, v->Ve, pairs, score, AI)) {
            v->converged = false;
            v->logl = logl_old;
            return false;
        }
        for (int64_t a = 0; a < np; ++a) AI[a + a * np] *= (1.0 + reg);
        std::vector<double> L, Dl;
        if (!la::ldlt(AI, (int)np, L, Dl)) break;
        std::vector<double> delta = score;
        la::ldlt_solve(L, Dl, (int)np, delta.data());
        double step = 1.0;
        bool accepted = false;
        std::vector<double> Vg_t, Ve_t;
        for (int h = 0; h < 12; ++h) {
            Vg_t = v->Vg;
            Ve_t = v->Ve;
            for (int64_t a = 0; a < vs; ++a) {
                const int j = pairs[a].first, k = pairs[a].second;
                Vg_t[j + k * d] += step * delta[a];
                Vg_t[k + j * d] = Vg_t[j + k * d];
                Ve_t[j + k * d] += step * delta[a + vs];
                Ve_t[k + j * d] = Ve_t[j + k * d];
            }
            near_pd(Vg_t, (int)d);
            near_pd(Ve_t, (int)d);
            const double logl_new = mv_loglik(v, Vg_t, Ve_t);
            if (std::isfinite(logl_new) && logl_new >= logl_old - 1e-10) {
                accepted = true;
                break;
            }
            step *= 0.5;
        }
        if (!accepted) break;
        v->Vg = Vg_t;
        v->Ve = Ve_t;
        logl_old = mv_loglik(v, v->Vg, v->Ve);
        double nrm = 0.0;
        for (double x : delta) nrm += x * x;
        if (std::sqrt(nrm) / std::sqrt((double)np) < o.ai_tol) {
            v->logl = logl_old;
            return true;  // converged: the reference returns before computing SEs
        }
    }
    if (logl_old < logl_initial + 1e-8) {
        v->Vg = Vg_initial;
        v->Ve = Ve_initial;
        logl_old = logl_initial;
    }
    v->logl = logl_old;
    // SEs from the AI matrix at the final parameters (:850-890)
    std::vector<double> score, AI;
    if (mv_score_ai(*v->d, d, v->Vg, v->Ve, pairs, score, AI)) {
        for (int64_t a = 0; a < np; ++a) AI[a + a * np] *= (1.0 + 1e-8);
        std::vector<double> L, Dl;
        if (la::ldlt(AI, (int)np, L, Dl)) {
            const std::vector<double> inv = la::ldlt_inverse(L, Dl, (int)np);
            for (int64_t a = 0; a < vs; ++a) {
                const int j = pairs[a].first, k = pairs[a].second;
                const double sg = std::sqrt(std::abs(inv[a + a * np]));
                const double se = std::sqrt(std::abs(inv[(vs + a) + (vs + a) * np]));
                v->Vg_se[j + k * d] = v->Vg_se[k + j * d] = sg;
                v->Ve_se[j + k * d] = v->Ve_se[k + j * d] = se;
            }
        }
    }
    return true;
}

void mv_get(const cs_mv_eigen_vce* v, double* Vg, double* Ve, double* Vg_se, double* Ve_se,
            double* D, double* Uty) {
    if (!v || !v->d) fail(CS_ERR_INVALID_ARGUMENT, "MvEigenVce: not prepared");
    if (Vg) std::copy(v->Vg.begin(), v->Vg.end(), Vg);
    if (Ve) std::copy(v->Ve.begin(), v->Ve.end(), Ve);
    if (Vg_se) std::copy(v->Vg_se.begin(), v->Vg_se.end(), Vg_se);
    if (Ve_se) std::copy(v->Ve_se.begin(), v->Ve_se.end(), Ve_se);
    if (D) std::copy(v->d->D.begin(), v->d->D.end(), D);
    if (Uty) std::copy(v->d->Uty.begin(), v->d->Uty.end(), Uty);
}

void mvlmm_scan_device(const cs_genotypes* g, const int32_t* keep, int64_t n, const double* dW,
                       bool w_colmajor, int64_t r, const double* Dv, const double* Uty, int64_t d,
                       const double* UtX, int64_t p, const double* Vg, const double* Ve,
                       int64_t snp_begin, int64_t snp_end, int precision, double* beta,
                       double* cov, double* wald, double* pvalue, double* freq,
                       int32_t* status);

void mv_scan(const cs_genotypes* g, const int32_t* keep, int64_t n_keep, const cs_mv_eigen_vce* v,
             int64_t snp_begin, int64_t snp_end, int precision, double* beta, double* cov,
             double* wald, double* pvalue, double* freq, int32_t* status) {
    if (!v || !v->d) fail(CS_ERR_INVALID_ARGUMENT, "MvEigenVce: not prepared");
    const DenseNull& dn = *v->d;
    if (n_keep != dn.n) fail(CS_ERR_INVALID_ARGUMENT, "MvLmmEngine::scan: sample count mismatch");
    mvlmm_scan_device(g, keep, n_keep, dn.W.get(), true, dn.n_eig, dn.D.data(), dn.Uty.data(),
                      v->traits, dn.UtX.data(), dn.p, v->Vg.data(), v->Ve.data(), snp_begin,
                      snp_end, precision, beta, cov, wald, pvalue, freq, status);
}

}  // namespace cs
