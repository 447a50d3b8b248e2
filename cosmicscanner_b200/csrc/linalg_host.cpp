// Small dense FP64 algebra on the host.  These matrices are at most a few hundred wide
// (sketch width, covariates, variance components), so plain loops are fast enough and
// keep the library free of any host LAPACK dependency.
#include "linalg_host.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace cs {
namespace la {

bool cholesky_upper(const std::vector<double>& G, int n, std::vector<double>& R) {
    R.assign((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i <= j; ++i) {
            double s = G[i + (size_t)j * n];
            for (int k = 0; k < i; ++k) s -= R[k + (size_t)i * n] * R[k + (size_t)j * n];
            if (i == j) {
                if (!(s > 0.0) || !std::isfinite(s)) return false;
                R[j + (size_t)j * n] = std::sqrt(s);
            } else {
                R[i + (size_t)j * n] = s / R[i + (size_t)i * n];
            }
        }
    }
    return true;
}

std::vector<double> upper_inverse(const std::vector<double>& R, int n) {
    std::vector<double> X((size_t)n * n, 0.0);
    // column j of the inverse solves R x = e_j: back substitution in axpy form, which walks
    // the columns of R contiguously; the columns are independent
#pragma omp parallel for schedule(dynamic, 4) if (n > 96)
    for (int j = 0; j < n; ++j) {
        double* x = X.data() + (size_t)j * n;
        x[j] = 1.0;
        for (int k = j; k >= 0; --k) {
            const double* rk = R.data() + (size_t)k * n;
            const double xk = x[k] / rk[k];
            x[k] = xk;
            for (int i = 0; i < k; ++i) x[i] -= xk * rk[i];
        }
    }
    return X;
}

bool tridiag_ql(const std::vector<double>& A_in, int n, std::vector<double>& d,
                std::vector<double>& Q, std::vector<PlaneRotation>& rots) {
    // Householder reduction of the lower triangle to tridiagonal form, updating only the
    // trailing block; the reflectors are kept for the backward accumulation of Q.
    std::vector<double> A((size_t)n * n);
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < n; ++r) {
            const int lo_r = std::max(r, c), lo_c = std::min(r, c);
            A[r + (size_t)c * n] = A_in[lo_r + (size_t)lo_c * n];
        }
    d.assign(n, 0.0);
    std::vector<double> e(n, 0.0);
    std::vector<double> refl((size_t)n * n, 0.0);  // column k: reflector v_k (rows k+1..n-1)
    std::vector<char> has_refl(n, 0);
    std::vector<double> p(n), w(n);
    for (int k = 0; k + 2 < n; ++k) {
        const int m0 = k + 1, len = n - m0;
        const double* col = A.data() + (size_t)k * n;
        double norm2 = 0.0;
        for (int i = m0; i < n; ++i) norm2 += col[i] * col[i];
        const double norm = std::sqrt(norm2);
        const double x0 = col[m0];
        d[k] = col[k];
        if (norm == 0.0) {
            e[k] = 0.0;
            continue;
        }
        const double alpha = x0 > 0 ? -norm : norm;
        double* v = refl.data() + (size_t)k * n;
        for (int i = m0; i < n; ++i) v[i] = col[i];
        v[m0] -= alpha;
        double vn = 0.0;
        for (int i = m0; i < n; ++i) vn += v[i] * v[i];
        vn = std::sqrt(vn);
        e[k] = alpha;
        if (vn == 0.0) continue;
        for (int i = m0; i < n; ++i) v[i] /= vn;
        has_refl[k] = 1;
        // p = A_sub v over the trailing block (symmetric: column dots)
        for (int c = m0; c < n; ++c) {
            const double* __restrict__ ac = A.data() + (size_t)c * n;
            const double* __restrict__ vv = v;
            double sacc = 0.0;
#pragma omp simd reduction(+ : sacc)
            for (int j = m0; j < n; ++j) sacc += ac[j] * vv[j];
            p[c] = sacc;
        }
        double kappa = 0.0;
        for (int i = m0; i < n; ++i) kappa += v[i] * p[i];
        for (int i = m0; i < n; ++i) w[i] = p[i] - kappa * v[i];
        // A_sub -= 2 (v w^T + w v^T)
        for (int c = m0; c < n; ++c) {
            double* __restrict__ ac = A.data() + (size_t)c * n;
            const double* __restrict__ vv = v;
            const double* __restrict__ ww = w.data();
            const double vc = 2.0 * v[c], wc = 2.0 * w[c];
#pragma omp simd
            for (int r = m0; r < n; ++r) ac[r] -= vv[r] * wc + ww[r] * vc;
        }
        (void)len;
    }
    if (n >= 2) {
        d[n - 2] = A[(n - 2) + (size_t)(n - 2) * n];
        e[n - 2] = A[(n - 1) + (size_t)(n - 2) * n];
    }
    d[n - 1] = A[(n - 1) + (size_t)(n - 1) * n];
    // Q = H_0 H_1 ... H_{n-3}, accumulated backwards on the trailing blocks (column-major)
    Q.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Q[i + (size_t)i * n] = 1.0;
    std::vector<double> t(n);
    for (int k = n - 3; k >= 0; --k) {
        if (!has_refl[k]) continue;
        const int m0 = k + 1;
        const double* v = refl.data() + (size_t)k * n;
        for (int c = m0; c < n; ++c) {
            const double* __restrict__ qc = Q.data() + (size_t)c * n;
            double sacc = 0.0;
#pragma omp simd reduction(+ : sacc)
            for (int i = m0; i < n; ++i) sacc += v[i] * qc[i];
            t[c] = 2.0 * sacc;
        }
        for (int c = m0; c < n; ++c) {
            double* __restrict__ qc = Q.data() + (size_t)c * n;
            const double tc = t[c];
#pragma omp simd
            for (int i = m0; i < n; ++i) qc[i] -= v[i] * tc;
        }
    }
    // Implicit QL with shifts on (d, e); the plane rotations are recorded so that they can be
    // applied to the columns of Q afterwards (in order).
    rots.clear();
    rots.reserve((size_t)n * 8);
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        int m;
        do {
            for (m = l; m < n - 1; ++m) {
                const double dd = std::abs(d[m]) + std::abs(d[m + 1]);
                if (std::abs(e[m]) <= 1e-15 * dd) break;
            }
            if (m != l) {
                if (++iter > 200) return false;
                double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                double r = std::sqrt(g * g + 1.0);
                g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
                double s = 1.0, c = 1.0, pp = 0.0;
                int i;
                for (i = m - 1; i >= l; --i) {
                    const double f = s * e[i];
                    const double b = c * e[i];
                    r = std::sqrt(f * f + g * g);
                    e[i + 1] = r;
                    if (r == 0.0) {
                        d[i + 1] -= pp;
                        e[m] = 0.0;
                        break;
                    }
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - pp;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    pp = s * r;
                    d[i + 1] = g + pp;
                    g = c * r - b;
                    rots.push_back(PlaneRotation{i, c, s});
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= pp;
                e[l] = g;
                e[m] = 0.0;
            }
        } while (m != l);
    }
    return true;
}

bool eigh(const std::vector<double>& A_in, int n, std::vector<double>& evals,
          std::vector<double>& V) {
    std::vector<double> d, Q;
    std::vector<PlaneRotation> rots;
    if (!tridiag_ql(A_in, n, d, Q, rots)) return false;
    // rotations on the columns of Q, each thread on its own block of rows
    constexpr int kRowBlock = 64;
    const int blocks = (n + kRowBlock - 1) / kRowBlock;
#pragma omp parallel for schedule(static) if (n > 96)
    for (int bidx = 0; bidx < blocks; ++bidx) {
        const int r0 = bidx * kRowBlock, r1 = std::min(n, r0 + kRowBlock);
        for (const PlaneRotation& rt : rots) {
            double* __restrict__ qa = Q.data() + (size_t)rt.i * n;
            double* __restrict__ qb = qa + n;
#pragma omp simd
            for (int r = r0; r < r1; ++r) {
                const double f = qb[r];
                qb[r] = rt.s * qa[r] + rt.c * f;
                qa[r] = rt.c * qa[r] - rt.s * f;
            }
        }
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
    evals.resize(n);
    V.assign((size_t)n * n, 0.0);
    for (int c = 0; c < n; ++c) {
        evals[c] = d[order[c]];
        std::copy(Q.begin() + (size_t)order[c] * n, Q.begin() + (size_t)(order[c] + 1) * n,
                  V.begin() + (size_t)c * n);
    }
    return true;
}

bool ldlt(const std::vector<double>& A, int n, std::vector<double>& L, std::vector<double>& D) {
    L.assign((size_t)n * n, 0.0);
    D.assign(n, 0.0);
    for (int j = 0; j < n; ++j) {
        double d = A[j + (size_t)j * n];
        for (int s = 0; s < j; ++s) d -= L[j + (size_t)s * n] * L[j + (size_t)s * n] * D[s];
        D[j] = d;
        if (!(d > 0.0) || !std::isfinite(d)) return false;
        L[j + (size_t)j * n] = 1.0;
        for (int i = j + 1; i < n; ++i) {
            double v = A[i + (size_t)j * n];
            for (int s = 0; s < j; ++s) v -= L[i + (size_t)s * n] * L[j + (size_t)s * n] * D[s];
            L[i + (size_t)j * n] = v / d;
        }
    }
    return true;
}

void ldlt_solve(const std::vector<double>& L, const std::vector<double>& D, int n, double* b) {
    for (int i = 0; i < n; ++i)
        for (int s = 0; s < i; ++s) b[i] -= L[i + (size_t)s * n] * b[s];
    for (int i = 0; i < n; ++i) b[i] /= D[i];
    for (int i = n - 1; i >= 0; --i)
        for (int s = i + 1; s < n; ++s) b[i] -= L[s + (size_t)i * n] * b[s];
}

std::vector<double> ldlt_inverse(const std::vector<double>& L, const std::vector<double>& D, int n) {
    std::vector<double> X((size_t)n * n, 0.0);
    for (int c = 0; c < n; ++c) {
        X[c + (size_t)c * n] = 1.0;
        ldlt_solve(L, D, n, X.data() + (size_t)c * n);
    }
    return X;
}

}  // namespace la
}  // namespace cs
