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

bool eigh(const std::vector<double>& A_in, int n, std::vector<double>& evals,
          std::vector<double>& V) {
    // A (row-major == column-major for a symmetric matrix) from the lower triangle
    std::vector<double> A((size_t)n * n);
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < n; ++r) {
            const int lo_r = std::max(r, c), lo_c = std::min(r, c);
            A[r + (size_t)c * n] = A_in[lo_r + (size_t)lo_c * n];
        }
    // Qt: transpose of the accumulated orthogonal factor, row-major: Qt[j][k] = Q[k][j]
    std::vector<double> Qt((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Qt[(size_t)i * n + i] = 1.0;
    std::vector<double> v(n), p(n), w(n), qv(n);
    // Householder reduction to tridiagonal form: A <- H A H, Q <- Q H
    for (int k = 0; k + 2 < n; ++k) {
        double norm2 = 0.0;
        for (int i = k + 1; i < n; ++i) norm2 += A[i + (size_t)k * n] * A[i + (size_t)k * n];
        const double x0 = A[k + 1 + (size_t)k * n];
        const double norm = std::sqrt(norm2);
        if (norm == 0.0) continue;
        const double alpha = x0 > 0 ? -norm : norm;
        std::fill(v.begin(), v.end(), 0.0);
        for (int i = k + 1; i < n; ++i) v[i] = A[i + (size_t)k * n];
        v[k + 1] -= alpha;
        double vn = 0.0;
        for (int i = k + 1; i < n; ++i) vn += v[i] * v[i];
        vn = std::sqrt(vn);
        if (vn == 0.0) continue;
        for (int i = k + 1; i < n; ++i) v[i] /= vn;
        // p = A v (A symmetric: column c of A dotted with v)
#pragma omp parallel for schedule(static) if (n > 96)
        for (int c = 0; c < n; ++c) {
            const double* col = A.data() + (size_t)c * n;
            double s = 0.0;
            for (int j = k + 1; j < n; ++j) s += col[j] * v[j];
            p[c] = s;
        }
        double kappa = 0.0;
        for (int i = k + 1; i < n; ++i) kappa += v[i] * p[i];
        for (int i = 0; i < n; ++i) w[i] = p[i] - kappa * v[i];
        // A' = A - 2 (v w^T + w v^T)
#pragma omp parallel for schedule(static) if (n > 96)
        for (int c = 0; c < n; ++c) {
            double* col = A.data() + (size_t)c * n;
            const double vc = v[c], wc = w[c];
            for (int r = 0; r < n; ++r) col[r] -= 2.0 * (v[r] * wc + w[r] * vc);
        }
        // Q <- Q H: Q[r][j] -= 2 (Q v)_r v_j, i.e. Qt[j][r] -= 2 v_j qv_r
        for (int r = 0; r < n; ++r) qv[r] = 0.0;
        for (int j = k + 1; j < n; ++j) {
            const double vj = v[j];
            const double* row = Qt.data() + (size_t)j * n;
            for (int r = 0; r < n; ++r) qv[r] += row[r] * vj;
        }
#pragma omp parallel for schedule(static) if (n > 96)
        for (int j = k + 1; j < n; ++j) {
            double* row = Qt.data() + (size_t)j * n;
            const double vj = 2.0 * v[j];
            for (int r = 0; r < n; ++r) row[r] -= vj * qv[r];
        }
    }
    std::vector<double> d(n), e(n, 0.0);
    for (int i = 0; i < n; ++i) d[i] = A[i + (size_t)i * n];
    for (int i = 0; i + 1 < n; ++i) e[i] = A[i + 1 + (size_t)i * n];
    // Implicit QL with shifts on (d, e); the plane rotations are recorded and applied to
    // the eigenvector rows afterwards, in parallel (e[i] couples d[i] and d[i+1]).
    struct Rot {
        int i;
        double c, s;
    };
    std::vector<Rot> rots;
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
                double r = std::hypot(g, 1.0);
                g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
                double s = 1.0, c = 1.0, pp = 0.0;
                int i;
                for (i = m - 1; i >= l; --i) {
                    const double f = s * e[i];
                    const double b = c * e[i];
                    r = std::hypot(f, g);
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
                    rots.push_back(Rot{i, c, s});
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= pp;
                e[l] = g;
                e[m] = 0.0;
            }
        } while (m != l);
    }
    // eigenvectors: rows of Q (= columns of Qt) rotated in sequence; each row independently
    std::vector<double> Vr((size_t)n * n);  // row-major: Vr[r][j] = Q[r][j]
    for (int j = 0; j < n; ++j)
        for (int r = 0; r < n; ++r) Vr[(size_t)r * n + j] = Qt[(size_t)j * n + r];
#pragma omp parallel
    {
#ifdef _OPENMP
        const int nt = omp_get_num_threads(), tid = omp_get_thread_num();
#else
        const int nt = 1, tid = 0;
#endif
        const int r0 = (int)((int64_t)n * tid / nt), r1 = (int)((int64_t)n * (tid + 1) / nt);
        for (const Rot& rt : rots)
            for (int r = r0; r < r1; ++r) {
                double* row = Vr.data() + (size_t)r * n;
                const double f = row[rt.i + 1];
                row[rt.i + 1] = rt.s * row[rt.i] + rt.c * f;
                row[rt.i] = rt.c * row[rt.i] - rt.s * f;
            }
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
    evals.resize(n);
    V.assign((size_t)n * n, 0.0);
    for (int c = 0; c < n; ++c) {
        evals[c] = d[order[c]];
        for (int r = 0; r < n; ++r) V[r + (size_t)c * n] = Vr[(size_t)r * n + order[c]];
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
