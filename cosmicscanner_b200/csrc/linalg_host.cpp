// Small dense FP64 algebra on the host.  These matrices are at most a few hundred wide
// (sketch width, covariates, variance components), so plain loops are fast enough and
// keep the library free of any host LAPACK dependency.
#include "linalg_host.h"

#include <algorithm>
#include <cmath>
#include <numeric>

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
    for (int j = 0; j < n; ++j) {
        X[j + (size_t)j * n] = 1.0 / R[j + (size_t)j * n];
        for (int i = j - 1; i >= 0; --i) {
            double s = 0.0;
            for (int k = i + 1; k <= j; ++k) s += R[i + (size_t)k * n] * X[k + (size_t)j * n];
            X[i + (size_t)j * n] = -s / R[i + (size_t)i * n];
        }
    }
    return X;
}

bool eigh(const std::vector<double>& A_in, int n, std::vector<double>& evals,
          std::vector<double>& V) {
    std::vector<double> A((size_t)n * n);
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < n; ++r) {
            const int lo_r = std::max(r, c), lo_c = std::min(r, c);
            A[r + (size_t)c * n] = A_in[lo_r + (size_t)lo_c * n];
        }
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) V[i + (size_t)i * n] = 1.0;
    std::vector<double> v(n), p(n), w(n);
    // Householder reduction to tridiagonal form, accumulating V = H_0 H_1 ...
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
        // A <- H A H with H = I - 2 v v^T: A' = A - 2 (v w^T + w v^T), w = p - (v^T p) v
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int j = k + 1; j < n; ++j) s += A[i + (size_t)j * n] * v[j];
            p[i] = s;
        }
        double kappa = 0.0;
        for (int i = k + 1; i < n; ++i) kappa += v[i] * p[i];
        for (int i = 0; i < n; ++i) w[i] = p[i] - kappa * v[i];
        for (int c = 0; c < n; ++c)
            for (int r = 0; r < n; ++r)
                A[r + (size_t)c * n] -= 2.0 * (v[r] * w[c] + w[r] * v[c]);
        // V <- V H
        for (int r = 0; r < n; ++r) {
            double s = 0.0;
            for (int j = k + 1; j < n; ++j) s += V[r + (size_t)j * n] * v[j];
            for (int j = k + 1; j < n; ++j) V[r + (size_t)j * n] -= 2.0 * s * v[j];
        }
    }
    std::vector<double> d(n), e(n, 0.0);
    for (int i = 0; i < n; ++i) d[i] = A[i + (size_t)i * n];
    for (int i = 0; i + 1 < n; ++i) e[i] = A[i + 1 + (size_t)i * n];
    // Implicit QL with shifts on (d, e); e[i] couples d[i] and d[i+1].
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
                    double f = s * e[i];
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
                    for (int k = 0; k < n; ++k) {
                        f = V[k + (size_t)(i + 1) * n];
                        V[k + (size_t)(i + 1) * n] = s * V[k + (size_t)i * n] + c * f;
                        V[k + (size_t)i * n] = c * V[k + (size_t)i * n] - s * f;
                    }
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= pp;
                e[l] = g;
                e[m] = 0.0;
            }
        } while (m != l);
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
    evals.resize(n);
    std::vector<double> W((size_t)n * n);
    for (int c = 0; c < n; ++c) {
        evals[c] = d[order[c]];
        for (int r = 0; r < n; ++r) W[r + (size_t)c * n] = V[r + (size_t)order[c] * n];
    }
    V.swap(W);
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
