// CPU oracle for the matrix-free mixed-model path — TEST INFRASTRUCTURE ONLY.
// Restates the reference CosmicScanner algorithms in plain FP64 loops (no Eigen,
// which is absent here).  Each function cites the reference file:line it follows.
// Only the tests and bench.py's CPU-baseline leg load this library.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <random>
#include <stdexcept>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// libCosmicCore/src/plink_reader.cpp:18-21 lookup table; kinship_operator.cpp:18-20.
const float kLookup[4] = {2.0f, NAN, 1.0f, 0.0f};
const float kDosage[4] = {2.0f, 0.0f, 1.0f, 0.0f};
const double kObserved[4] = {1.0, 0.0, 1.0, 1.0};

inline int code_at(const uint8_t* row, int64_t sample) {
    return (row[sample >> 2] >> ((sample & 3) * 2)) & 3;
}

struct Selection {
    const uint8_t* bed;
    int64_t n_fam, stride;
    const double* mean;
    const double* inv_std;
    const int32_t* keep;
    int64_t n_keep;
    const int32_t* variants;
    int64_t n_var;
    bool identity;
    int64_t rows() const { return keep ? n_keep : n_fam; }
    int64_t cols() const { return n_var; }
    int64_t snp(int64_t t) const { return variants ? variants[t] : t; }
    int64_t sample(int64_t r) const { return identity ? r : keep[r]; }
    const uint8_t* row(int64_t t) const { return bed + snp(t) * stride; }
};

// kinship_operator.cpp:35-64: an explicit keep equal to 0..n-1 is the identity path.
Selection make_selection(const uint8_t* bed, int64_t n_fam, int64_t stride, const double* mean,
                         const double* inv_std, const int32_t* keep, int64_t n_keep,
                         const int32_t* variants, int64_t n_var) {
    Selection s{bed, n_fam, stride, mean, inv_std, keep, n_keep, variants, n_var, true};
    if (keep) {
        s.identity = (n_keep == n_fam);
        for (int64_t i = 0; s.identity && i < n_fam; ++i) s.identity = keep[i] == i;
    }
    return s;
}

// libgomp static schedule without chunk: the first (m % w) workers take one extra iteration.
void static_range(int64_t m, int workers, int w, int64_t* lo, int64_t* hi) {
    const int64_t q = m / workers, r = m % workers;
    *lo = w * q + std::min<int64_t>(w, r);
    *hi = *lo + q + (w < r ? 1 : 0);
}

// kinship_operator.cpp:74-137 (multiplyZt)
void multiply_zt(const Selection& s, const double* v, double* u) {
    const int64_t n = s.rows();
    for (int64_t t = 0; t < s.cols(); ++t) {
        const int64_t j = s.snp(t);
        const double inv_std = s.inv_std[j];
        u[t] = 0.0;
        if (inv_std == 0.0) continue;
        const double mean = s.mean[j];
        const uint8_t* col = s.row(t);
        double sum_xv = 0.0, sum_v = 0.0;
        if (s.identity) {
            const int64_t full = n >> 2;
            for (int64_t b = 0; b < full; ++b) {
                const uint8_t byte = col[b];
                const int64_t r = b << 2;
                const double v0 = v[r], v1 = v[r + 1], v2 = v[r + 2], v3 = v[r + 3];
                sum_xv += v0 * kDosage[byte & 3] + v1 * kDosage[(byte >> 2) & 3] +
                          v2 * kDosage[(byte >> 4) & 3] + v3 * kDosage[(byte >> 6) & 3];
                sum_v += v0 * kObserved[byte & 3] + v1 * kObserved[(byte >> 2) & 3] +
                         v2 * kObserved[(byte >> 4) & 3] + v3 * kObserved[(byte >> 6) & 3];
            }
            for (int64_t r = full << 2; r < n; ++r) {
                const int code = code_at(col, r);
                if (code == 1) continue;
                sum_xv += static_cast<double>(kDosage[code]) * v[r];
                sum_v += v[r];
            }
        } else {
            for (int64_t r = 0; r < n; ++r) {
                const int code = code_at(col, s.keep[r]);
                if (code == 1) continue;
                sum_xv += static_cast<double>(kDosage[code]) * v[r];
                sum_v += v[r];
            }
        }
        u[t] = (sum_xv - mean * sum_v) * inv_std;
    }
}

// kinship_operator.cpp:139-209 (multiplyZ) with worker-order reduction.
void multiply_z(const Selection& s, const double* u, double* y, int n_threads) {
    const int64_t n = s.rows(), m = s.cols();
    std::fill(y, y + n, 0.0);
    auto accumulate = [&](int64_t t, double* dest) {
        const int64_t j = s.snp(t);
        const double inv_std = s.inv_std[j];
        if (inv_std == 0.0) return;
        const double mean = s.mean[j];
        const double weight = u[t] * inv_std;
        const uint8_t* col = s.row(t);
        if (s.identity) {
            const double vmap[4] = {(2.0 - mean) * weight, 0.0, (1.0 - mean) * weight,
                                    (0.0 - mean) * weight};
            const int64_t full = n >> 2;
            for (int64_t b = 0; b < full; ++b) {
                const uint8_t byte = col[b];
                const int64_t r = b << 2;
                dest[r] += vmap[byte & 3];
                dest[r + 1] += vmap[(byte >> 2) & 3];
                dest[r + 2] += vmap[(byte >> 4) & 3];
                dest[r + 3] += vmap[(byte >> 6) & 3];
            }
            for (int64_t r = full << 2; r < n; ++r) dest[r] += vmap[code_at(col, r)];
        } else {
            for (int64_t r = 0; r < n; ++r) {
                const int code = code_at(col, s.keep[r]);
                if (code == 1) continue;
                dest[r] += (static_cast<double>(kDosage[code]) - mean) * weight;
            }
        }
    };
    const int workers = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(n_threads, m)));
    if (workers == 1) {
        for (int64_t t = 0; t < m; ++t) accumulate(t, y);
        return;
    }
    std::vector<double> local(static_cast<size_t>(n) * workers, 0.0);
#pragma omp parallel for num_threads(workers) schedule(static, 1)
    for (int w = 0; w < workers; ++w) {
        int64_t lo, hi;
        static_range(m, workers, w, &lo, &hi);
        for (int64_t t = lo; t < hi; ++t) accumulate(t, local.data() + static_cast<size_t>(w) * n);
    }
    for (int w = 0; w < workers; ++w)
        for (int64_t r = 0; r < n; ++r) y[r] += local[static_cast<size_t>(w) * n + r];
}

// ---------------------------------------------------------------- small dense algebra
// Column-major helpers, plain loops.

// Householder QR of A (n x k, ld n, n >= k), returns thin Q (n x k) in place of A.
// Follows Eigen's makeHouseholder convention (beta = -sign(c0) * norm).
void householder_thin_q(double* A, int64_t n, int64_t k) {
    std::vector<double> tau(k, 0.0);
    for (int64_t j = 0; j < k; ++j) {
        double* col = A + j * n;
        const double c0 = col[j];
        double tail = 0.0;
        for (int64_t i = j + 1; i < n; ++i) tail += col[i] * col[i];
        if (tail <= std::numeric_limits<double>::min()) {
            tau[j] = 0.0;
            for (int64_t i = j + 1; i < n; ++i) col[i] = 0.0;
            continue;
        }
        double beta = std::sqrt(c0 * c0 + tail);
        if (c0 >= 0.0) beta = -beta;
        const double scale = 1.0 / (c0 - beta);
        for (int64_t i = j + 1; i < n; ++i) col[i] *= scale;
        tau[j] = (beta - c0) / beta;
        col[j] = beta;
        // apply H = I - tau v v^T to the trailing columns (v = [1; col[j+1:]])
#pragma omp parallel for schedule(static)
        for (int64_t c = j + 1; c < k; ++c) {
            double* a = A + c * n;
            double dot = a[j];
            for (int64_t i = j + 1; i < n; ++i) dot += col[i] * a[i];
            dot *= tau[j];
            a[j] -= dot;
            for (int64_t i = j + 1; i < n; ++i) a[i] -= dot * col[i];
        }
    }
    // Form Q = H_0 ... H_{k-1} [I_k; 0] by backward accumulation.
    std::vector<double> Q(static_cast<size_t>(n) * k, 0.0);
    for (int64_t c = 0; c < k; ++c) Q[c * n + c] = 1.0;
    for (int64_t j = k - 1; j >= 0; --j) {
        const double* v = A + j * n;
        if (tau[j] == 0.0) continue;
#pragma omp parallel for schedule(static)
        for (int64_t c = j; c < k; ++c) {
            double* q = Q.data() + c * n;
            double dot = q[j];
            for (int64_t i = j + 1; i < n; ++i) dot += v[i] * q[i];
            dot *= tau[j];
            q[j] -= dot;
            for (int64_t i = j + 1; i < n; ++i) q[i] -= dot * v[i];
        }
    }
    std::memcpy(A, Q.data(), sizeof(double) * Q.size());
}

// Cyclic Jacobi eigensolver for a symmetric k x k matrix (column-major).
// Returns eigenvalues ascending (like Eigen's SelfAdjointEigenSolver) and vectors.
void jacobi_eigh(const double* S, int64_t k, double* evals, double* evecs) {
    std::vector<double> A(S, S + k * k);
    for (int64_t i = 0; i < k; ++i)
        for (int64_t j = 0; j < k; ++j) evecs[i + j * k] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int64_t j = 0; j < k; ++j)
            for (int64_t i = 0; i < k; ++i) {
                if (i != j) off += A[i + j * k] * A[i + j * k];
                else diag += A[i + j * k] * A[i + j * k];
            }
        if (off <= 1e-30 * diag || off == 0.0) break;
        for (int64_t p = 0; p < k - 1; ++p)
            for (int64_t q = p + 1; q < k; ++q) {
                const double apq = A[p + q * k];
                if (std::abs(apq) < 1e-300) continue;
                const double app = A[p + p * k], aqq = A[q + q * k];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) /
                                 (std::abs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int64_t r = 0; r < k; ++r) {
                    const double arp = A[r + p * k], arq = A[r + q * k];
                    A[r + p * k] = c * arp - s * arq;
                    A[r + q * k] = s * arp + c * arq;
                }
                for (int64_t r = 0; r < k; ++r) {
                    const double apr = A[p + r * k], aqr = A[q + r * k];
                    A[p + r * k] = c * apr - s * aqr;
                    A[q + r * k] = s * apr + c * aqr;
                }
                for (int64_t r = 0; r < k; ++r) {
                    const double vrp = evecs[r + p * k], vrq = evecs[r + q * k];
                    evecs[r + p * k] = c * vrp - s * vrq;
                    evecs[r + q * k] = s * vrp + c * vrq;
                }
            }
    }
    std::vector<int64_t> order(k);
    for (int64_t i = 0; i < k; ++i) order[i] = i;
    std::sort(order.begin(), order.end(),
              [&](int64_t a, int64_t b) { return A[a + a * k] < A[b + b * k]; });
    std::vector<double> V(evecs, evecs + k * k);
    for (int64_t c = 0; c < k; ++c) {
        evals[c] = A[order[c] + order[c] * k];
        for (int64_t r = 0; r < k; ++r) evecs[r + c * k] = V[r + order[c] * k];
    }
}

// LDL^T of a small SPD matrix (p x p).  Returns false when a pivot is not positive
// (Eigen LDLT::isPositive() in the reference objective).
bool ldlt(const double* A, int64_t p, std::vector<double>& L, std::vector<double>& D) {
    L.assign(p * p, 0.0);
    D.assign(p, 0.0);
    for (int64_t j = 0; j < p; ++j) {
        double d = A[j + j * p];
        for (int64_t s = 0; s < j; ++s) d -= L[j + s * p] * L[j + s * p] * D[s];
        D[j] = d;
        if (!(d > 0.0)) return false;
        L[j + j * p] = 1.0;
        for (int64_t i = j + 1; i < p; ++i) {
            double v = A[i + j * p];
            for (int64_t s = 0; s < j; ++s) v -= L[i + s * p] * L[j + s * p] * D[s];
            L[i + j * p] = v / d;
        }
    }
    return true;
}

void ldlt_solve(const std::vector<double>& L, const std::vector<double>& D, int64_t p, double* b) {
    for (int64_t i = 0; i < p; ++i)
        for (int64_t s = 0; s < i; ++s) b[i] -= L[i + s * p] * b[s];
    for (int64_t i = 0; i < p; ++i) b[i] /= D[i];
    for (int64_t i = p - 1; i >= 0; --i)
        for (int64_t s = i + 1; s < p; ++s) b[i] -= L[s + i * p] * b[s];
}

// src/lmm_engine.cpp:22-58 (gamma_q): series / continued fraction, 1e-7 tolerance.
double gamma_q(double a, double x) {
    if (x < 0.0 || a <= 0.0) return 1.0;
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

}  // namespace

extern "C" {

void orc_compute_stats(const uint8_t* bed, int64_t n_samples, int64_t n_snps, int64_t stride,
                       double* mean, double* inv_std, int32_t* count_out, double* sum_out) {
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n_snps; ++j) {
        const uint8_t* col = bed + j * stride;
        double sum = 0.0, sum_sq = 0.0;
        int count = 0;
        for (int64_t i = 0; i < n_samples; ++i) {
            const float val = kLookup[(col[i / 4] >> ((i % 4) * 2)) & 3];
            if (!std::isnan(val)) {
                sum += val;
                sum_sq += val * val;
                count++;
            }
        }
        (void)sum_sq;
        if (count_out) count_out[j] = count;
        if (sum_out) sum_out[j] = sum;
        if (count > 0) {
            const double m = sum / count;
            const double p = m / 2.0;
            const double var = 2.0 * p * (1.0 - p);
            mean[j] = m;
            inv_std[j] = (var < 1e-9) ? 0.0 : 1.0 / std::sqrt(var);
        } else {
            mean[j] = 0.0;
            inv_std[j] = 0.0;
        }
    }
}

int orc_kinship_apply_vector(const uint8_t* bed, int64_t n_fam, int64_t stride,
                             const double* mean, const double* inv_std,
                             const int32_t* keep, int64_t n_keep,
                             const int32_t* variants, int64_t n_var,
                             const double* v, double* out, int n_threads) {
    Selection s = make_selection(bed, n_fam, stride, mean, inv_std, keep, n_keep, variants, n_var);
    if (s.cols() == 0) return -1;
    std::vector<double> u(s.cols()), w(s.rows());
    multiply_zt(s, v, u.data());
    multiply_z(s, u.data(), w.data(), std::max(1, n_threads));
    const double scaling = 1.0 / static_cast<double>(s.cols());
    for (int64_t r = 0; r < s.rows(); ++r) out[r] = scaling * w[r];
    return 0;
}

int orc_kinship_apply_block(const uint8_t* bed, int64_t n_fam, int64_t stride,
                            const double* mean, const double* inv_std,
                            const int32_t* keep, int64_t n_keep,
                            const int32_t* variants, int64_t n_var,
                            const double* X, int64_t ldx, int64_t k,
                            double* out, int64_t ldo, int n_threads) {
    Selection s = make_selection(bed, n_fam, stride, mean, inv_std, keep, n_keep, variants, n_var);
    const int64_t n = s.rows(), m = s.cols();
    if (m == 0) return -1;
    std::vector<double> result(static_cast<size_t>(n) * k, 0.0);
    const int64_t block = 512;
    std::vector<double> z, proj;
    for (int64_t first = 0; first < m; first += block) {
        const int64_t count = std::min(block, m - first);
        z.assign(static_cast<size_t>(n) * count, 0.0);
#pragma omp parallel for num_threads(std::max(1, n_threads)) schedule(static)
        for (int64_t j = 0; j < count; ++j) {
            const int64_t snp = s.snp(first + j);
            const double mu = mean[snp], is = inv_std[snp];
            double* dest = z.data() + j * n;
            if (is == 0.0) continue;
            const double values[4] = {(2.0 - mu) * is, 0.0, (1.0 - mu) * is, -mu * is};
            const uint8_t* col = bed + snp * stride;
            for (int64_t r = 0; r < n; ++r) dest[r] = values[code_at(col, s.sample(r))];
        }
        proj.assign(static_cast<size_t>(count) * k, 0.0);  // count x k
#pragma omp parallel for num_threads(std::max(1, n_threads)) schedule(static) collapse(2)
        for (int64_t c = 0; c < k; ++c)
            for (int64_t j = 0; j < count; ++j) {
                const double* zc = z.data() + j * n;
                const double* xc = X + c * ldx;
                double acc = 0.0;
                for (int64_t r = 0; r < n; ++r) acc += zc[r] * xc[r];
                proj[j + c * count] = acc;
            }
#pragma omp parallel for num_threads(std::max(1, n_threads)) schedule(static)
        for (int64_t c = 0; c < k; ++c) {
            double* rc = result.data() + c * n;
            for (int64_t j = 0; j < count; ++j) {
                const double pj = proj[j + c * count];
                const double* zc = z.data() + j * n;
                for (int64_t r = 0; r < n; ++r) rc[r] += zc[r] * pj;
            }
        }
    }
    const double scaling = 1.0 / static_cast<double>(m);
    for (int64_t c = 0; c < k; ++c)
        for (int64_t r = 0; r < n; ++r) out[r + c * ldo] = result[r + c * n] * scaling;
    return 0;
}

double orc_kinship_trace(const uint8_t* bed, int64_t n_fam, int64_t stride,
                         const double* mean, const double* inv_std,
                         const int32_t* keep, int64_t n_keep,
                         const int32_t* variants, int64_t n_var) {
    Selection s = make_selection(bed, n_fam, stride, mean, inv_std, keep, n_keep, variants, n_var);
    double total = 0.0;
    for (int64_t t = 0; t < s.cols(); ++t) {
        const int64_t j = s.snp(t);
        if (inv_std[j] == 0.0) continue;
        const uint8_t* col = s.row(t);
        double sum_sq = 0.0;
        for (int64_t r = 0; r < s.rows(); ++r) {
            const int code = code_at(col, s.sample(r));
            if (code == 1) continue;
            const double z = (static_cast<double>(kDosage[code]) - mean[j]) * inv_std[j];
            sum_sq += z * z;
        }
        total += sum_sq;
    }
    return (1.0 / static_cast<double>(s.cols())) * total;
}

void orc_kinship_diagonal(const uint8_t* bed, int64_t n_fam, int64_t stride,
                          const double* mean, const double* inv_std,
                          const int32_t* keep, int64_t n_keep,
                          const int32_t* variants, int64_t n_var, double* diag) {
    Selection s = make_selection(bed, n_fam, stride, mean, inv_std, keep, n_keep, variants, n_var);
    const double scaling = 1.0 / static_cast<double>(s.cols());
    std::fill(diag, diag + s.rows(), 0.0);
    for (int64_t t = 0; t < s.cols(); ++t) {
        const int64_t j = s.snp(t);
        if (inv_std[j] == 0.0) continue;
        const uint8_t* col = s.row(t);
        for (int64_t r = 0; r < s.rows(); ++r) {
            const int code = code_at(col, keep ? keep[r] : r);
            if (code == 1) continue;
            const double z = (static_cast<double>(kDosage[code]) - mean[j]) * inv_std[j];
            diag[r] += scaling * z * z;
        }
    }
}

void orc_dense_z(const uint8_t* bed, int64_t n_fam, int64_t stride,
                 const double* mean, const double* inv_std,
                 const int32_t* keep, int64_t n_keep,
                 const int32_t* variants, int64_t n_var, double* z, int64_t ldz) {
    Selection s = make_selection(bed, n_fam, stride, mean, inv_std, keep, n_keep, variants, n_var);
    for (int64_t t = 0; t < s.cols(); ++t) {
        const int64_t j = s.snp(t);
        const uint8_t* col = bed + j * stride;
        for (int64_t r = 0; r < s.rows(); ++r) {
            const float dosage = kLookup[code_at(col, keep ? keep[r] : r)];
            z[r + t * ldz] = std::isnan(dosage) ? 0.0 : (dosage - mean[j]) * inv_std[j];
        }
    }
}

void orc_kinship_batch_fixture(int n, int m, uint64_t seed, uint8_t* bed_out,
                               int n_sel, const int32_t* rows, int n_widths,
                               const int32_t* widths, double* omega_out) {
    std::mt19937_64 rng(seed);
    const int stride = (n + 3) / 4;
    bed_out[0] = 0x6c;
    bed_out[1] = 0x1b;
    bed_out[2] = 0x01;
    for (int j = 0; j < m; ++j)
        for (int b = 0; b < stride; ++b) {
            unsigned char byte = 0;
            for (int k = 0; k < 4; ++k) {
                const unsigned char code = j % 31 == 0 ? 3 : j % 37 == 0 ? 1 : rng() % 4;
                byte |= code << (2 * k);
            }
            bed_out[3 + static_cast<size_t>(j) * stride + b] = byte;
        }
    if (!omega_out) return;
    size_t off = 0;
    for (int s = 0; s < n_sel; ++s)
        for (int w = 0; w < n_widths; ++w) {
            std::normal_distribution<double> normal;
            for (int j = 0; j < widths[w]; ++j)
                for (int i = 0; i < rows[s]; ++i) omega_out[off++] = normal(rng);
        }
}

void orc_normal_matrix(uint64_t seed, int64_t n, int64_t cols, double* out) {
    std::mt19937_64 generator(seed);
    std::normal_distribution<double> normal(0.0, 1.0);
    for (int64_t j = 0; j < cols; ++j)
        for (int64_t i = 0; i < n; ++i) out[i + j * n] = normal(generator);
}

int orc_prepare_marker(const double* raw, int64_t n, double min_maf, double* values,
                       double* freq, int32_t* observed_out) {
    double dosage_sum = 0.0;
    int observed = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (std::isnan(raw[i])) continue;
        dosage_sum += raw[i];
        ++observed;
    }
    *observed_out = observed;
    *freq = 0.0;
    if (observed == 0) return 0;
    const double af = dosage_sum / (2.0 * observed);
    *freq = af;
    const int passes = observed >= 3 && std::min(af, 1.0 - af) >= min_maf;
    double encoded_sum = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        values[i] = raw[i];
        if (std::isfinite(values[i])) encoded_sum += values[i];
    }
    const double encoded_mean = encoded_sum / observed;
    for (int64_t i = 0; i < n; ++i) {
        if (!std::isfinite(values[i])) values[i] = encoded_mean;
        values[i] -= encoded_mean;
    }
    return passes;
}

double orc_chisq_prob(double stat, int df) {
    if (stat <= 0) return 1.0;
    return gamma_q(df / 2.0, stat / 2.0);
}

int orc_lowrank_reml(const double* U, const double* lam, int64_t n, int64_t rank, double r0,
                     const double* y, const double* X, int64_t p, orc_lowrank_result* res) {
    const int64_t df = n - p;
    if (df <= 0) return -1;
    // apply_ratio_inverse(eta, rhs) = base*rhs + U diag(1/(1+eta*lambda) - base) U^T rhs
    auto ratio_inverse = [&](double eta, const double* rhs, int64_t cols, double* out) {
        const double base = 1.0 / (1.0 + eta * r0);
        std::vector<double> utr(rank * cols, 0.0);
        for (int64_t c = 0; c < cols; ++c)
            for (int64_t j = 0; j < rank; ++j) {
                double acc = 0.0;
                for (int64_t i = 0; i < n; ++i) acc += U[i + j * n] * rhs[i + c * n];
                utr[j + c * rank] = acc * (1.0 / (1.0 + eta * lam[j]) - base);
            }
        for (int64_t c = 0; c < cols; ++c)
            for (int64_t i = 0; i < n; ++i) {
                double acc = 0.0;
                for (int64_t j = 0; j < rank; ++j) acc += U[i + j * n] * utr[j + c * rank];
                out[i + c * n] = base * rhs[i + c * n] + acc;
            }
    };
    auto objective = [&](double log_eta, double* quadratic) {
        const double eta = std::exp(log_eta);
        std::vector<double> rx(n * p), info(p * p), ry(n), beta(p), resid(n), rr(n);
        ratio_inverse(eta, X, p, rx.data());
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b) {
                double acc = 0.0;
                for (int64_t i = 0; i < n; ++i) acc += X[i + a * n] * rx[i + b * n];
                info[a + b * p] = acc;
            }
        std::vector<double> L, D;
        if (!ldlt(info.data(), p, L, D)) return std::numeric_limits<double>::infinity();
        ratio_inverse(eta, y, 1, ry.data());
        for (int64_t a = 0; a < p; ++a) {
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) acc += X[i + a * n] * ry[i];
            beta[a] = acc;
        }
        ldlt_solve(L, D, p, beta.data());
        for (int64_t i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int64_t a = 0; a < p; ++a) acc += X[i + a * n] * beta[a];
            resid[i] = y[i] - acc;
        }
        ratio_inverse(eta, resid.data(), 1, rr.data());
        double qf = 0.0;
        for (int64_t i = 0; i < n; ++i) qf += resid[i] * rr[i];
        if (!(qf > 0.0) || !std::isfinite(qf)) return std::numeric_limits<double>::infinity();
        if (quadratic) *quadratic = qf;
        double logdet_r = (n - rank) * std::log1p(eta * r0);
        for (int64_t j = 0; j < rank; ++j) logdet_r += std::log(1.0 + eta * lam[j]);
        double logdet_x = 0.0;
        for (int64_t a = 0; a < p; ++a) logdet_x += std::log(std::max(std::abs(D[a]), 1e-300));
        return logdet_r + logdet_x + df * std::log(qf / static_cast<double>(df));
    };
    const int grid = 81;
    int best_index = 0;
    double best_log_eta = -12.0;
    double best_obj = objective(best_log_eta, nullptr);
    for (int i = 1; i < grid; ++i) {
        const double cand = -12.0 + 24.0 * i / static_cast<double>(grid - 1);
        const double v = objective(cand, nullptr);
        if (v < best_obj) {
            best_obj = v;
            best_log_eta = cand;
            best_index = i;
        }
    }
    double left = -12.0 + 24.0 * std::max(0, best_index - 1) / static_cast<double>(grid - 1);
    double right = -12.0 + 24.0 * std::min(grid - 1, best_index + 1) / static_cast<double>(grid - 1);
    const double golden = (std::sqrt(5.0) - 1.0) / 2.0;
    double c = right - golden * (right - left), d = left + golden * (right - left);
    double fc = objective(c, nullptr), fd = objective(d, nullptr);
    for (int it = 0; it < 80 && right - left > 1e-8; ++it) {
        if (fc < fd) {
            right = d; d = c; fd = fc; c = right - golden * (right - left);
            fc = objective(c, nullptr);
        } else {
            left = c; c = d; fc = fd; d = left + golden * (right - left);
            fd = objective(d, nullptr);
        }
    }
    best_log_eta = 0.5 * (left + right);
    double quadratic = 0.0;
    best_obj = objective(best_log_eta, &quadratic);
    if (!std::isfinite(best_obj)) return -2;
    res->best_log_eta = best_log_eta;
    res->best_objective = best_obj;
    res->delta = std::exp(-best_log_eta);
    res->sigma2_e = quadratic / static_cast<double>(df);
    res->sigma2_g = std::exp(best_log_eta) * res->sigma2_e;
    return 0;
}

int orc_lowrank_prepare(const uint8_t* bed, int64_t n_fam, int64_t stride,
                        const double* mean, const double* inv_std,
                        const int32_t* keep, int64_t n_keep,
                        const int32_t* variants, int64_t n_var,
                        const double* y, const double* X, int64_t p,
                        int rank, int oversample, uint64_t seed,
                        double trace_threshold, int min_rank, int n_threads,
                        double* U_out, double* lambda_out, orc_lowrank_result* res) {
    Selection s = make_selection(bed, n_fam, stride, mean, inv_std, keep, n_keep, variants, n_var);
    const int64_t n = s.rows();
    if (rank <= 0 || rank >= n) return -1;
    const int64_t sk = std::min<int64_t>(n, rank + std::max(0, oversample));
    std::vector<double> omega(n * sk), sample(n * sk), q(n * sk);
    orc_normal_matrix(seed, n, sk, omega.data());
    auto apply = [&](const double* in, double* out) {
        orc_kinship_apply_block(bed, n_fam, stride, mean, inv_std, keep, n_keep, variants, n_var,
                                in, n, sk, out, n, n_threads);
    };
    apply(omega.data(), sample.data());
    for (int it = 0; it < 2; ++it) {
        q = sample;
        householder_thin_q(q.data(), n, sk);
        apply(q.data(), sample.data());
    }
    q = sample;
    householder_thin_q(q.data(), n, sk);
    std::vector<double> kq(n * sk), small(sk * sk);
    apply(q.data(), kq.data());
#pragma omp parallel for schedule(static) collapse(2)
    for (int64_t b = 0; b < sk; ++b)
        for (int64_t a = 0; a < sk; ++a) {
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) acc += q[i + a * n] * kq[i + b * n];
            small[a + b * sk] = acc;
        }
    std::vector<double> evals(sk), evecs(sk * sk);
    jacobi_eigh(small.data(), sk, evals.data(), evecs.data());
    std::vector<double> lead(rank);
    for (int j = 0; j < rank; ++j) lead[j] = std::max(0.0, evals[sk - 1 - j]);
    const double total_trace = orc_kinship_trace(bed, n_fam, stride, mean, inv_std, keep, n_keep,
                                                 variants, n_var);
    int selected = rank;
    bool met = trace_threshold <= 0.0;
    if (trace_threshold > 0.0 && total_trace > 0.0) {
        double retained = 0.0;
        const int first_allowed = std::min(rank, std::max(1, min_rank));
        for (int j = 0; j < rank; ++j) {
            retained += lead[j];
            if (j + 1 >= first_allowed && retained / total_trace >= trace_threshold) {
                selected = j + 1;
                met = true;
                break;
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (int j = 0; j < selected; ++j) {
        const int64_t src = sk - 1 - j;
        for (int64_t i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int64_t a = 0; a < sk; ++a) acc += q[i + a * n] * evecs[a + src * sk];
            U_out[i + j * n] = acc;
        }
    }
    double lam_sum = 0.0, lam_sq = 0.0;
    for (int j = 0; j < selected; ++j) {
        lambda_out[j] = lead[j];
        lam_sum += lead[j];
        lam_sq += lead[j] * lead[j];
    }
    const double r0 = std::max(0.0, (total_trace - lam_sum) / static_cast<double>(n - selected));
    const double approx_sq = lam_sq + (n - selected) * r0 * r0;
    double cross = r0 * total_trace;
    for (int j = 0; j < selected; ++j) cross += (lead[j] - r0) * lead[j];
    const double resid_sq = std::max(0.0, total_trace * total_trace + approx_sq - 2.0 * cross);
    res->rank = selected;
    res->sketch_size = static_cast<int32_t>(sk);
    res->residual_eigenvalue = r0;
    res->relative_frobenius_error =
        std::sqrt(resid_sq) / std::max(total_trace, std::numeric_limits<double>::min());
    res->trace = total_trace;
    res->trace_fraction = total_trace > 0.0 ? lam_sum / total_trace : 0.0;
    res->trace_threshold_met = met;
    return orc_lowrank_reml(U_out, lambda_out, n, selected, r0, y, X, p, res);
}

int orc_scan_lowrank(const uint8_t* bed, int64_t n_fam, int64_t stride, int64_t n_snps,
                     const int32_t* keep, int64_t n,
                     const double* U, const double* lam, int64_t rank, double r0,
                     double sg2, double se2,
                     const double* y, const double* X, int64_t p, double min_maf,
                     double* beta_out, double* se_out, double* pval_out, double* log10p_out,
                     double* freq_out, int32_t* tested) {
    (void)n_fam;
    // applyLowRankVinv, src/lmm_engine.cpp:1097-1105
    const double base = 1.0 / std::max(1e-12, sg2 * r0 + se2);
    std::vector<double> corr(rank);
    for (int64_t j = 0; j < rank; ++j) corr[j] = 1.0 / (sg2 * lam[j] + se2) - base;
    auto vinv = [&](const double* rhs, double* out) {
        std::vector<double> t(rank);
        for (int64_t j = 0; j < rank; ++j) {
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) acc += U[i + j * n] * rhs[i];
            t[j] = acc * corr[j];
        }
        for (int64_t i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int64_t j = 0; j < rank; ++j) acc += U[i + j * n] * t[j];
            out[i] = base * rhs[i] + acc;
        }
    };
    // :1273-1285 null quantities
    std::vector<double> vx(n * p), info(p * p), info_inv(p * p), vy(n), beta(p), resid(n), py(n);
    for (int64_t a = 0; a < p; ++a) vinv(X + a * n, vx.data() + a * n);
    for (int64_t a = 0; a < p; ++a)
        for (int64_t b = 0; b < p; ++b) {
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) acc += X[i + a * n] * vx[i + b * n];
            info[a + b * p] = acc;
        }
    std::vector<double> L, D;
    if (!ldlt(info.data(), p, L, D)) return -1;
    for (int64_t c = 0; c < p; ++c) {
        std::vector<double> e(p, 0.0);
        e[c] = 1.0;
        ldlt_solve(L, D, p, e.data());
        for (int64_t r = 0; r < p; ++r) info_inv[r + c * p] = e[r];
    }
    vinv(y, vy.data());
    for (int64_t a = 0; a < p; ++a) {
        double acc = 0.0;
        for (int64_t b = 0; b < p; ++b) {
            double xb = 0.0;
            for (int64_t i = 0; i < n; ++i) xb += X[i + b * n] * vy[i];
            acc += info_inv[a + b * p] * xb;
        }
        beta[a] = acc;
    }
    for (int64_t i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int64_t a = 0; a < p; ++a) acc += X[i + a * n] * beta[a];
        resid[i] = y[i] - acc;
    }
    vinv(resid.data(), py.data());
    // per-marker (:1337-1358), then the block formulas of :1309-1320
    std::vector<double> raw(n), g(n), vg(n), xvg(p), mid(p);
#pragma omp parallel for schedule(dynamic, 16) firstprivate(raw, g, vg, xvg, mid)
    for (int64_t j = 0; j < n_snps; ++j) {
        tested[j] = 0;
        const uint8_t* row = bed + j * stride;
        for (int64_t i = 0; i < n; ++i) {
            const int code = code_at(row, keep[i]);
            raw[i] = code == 1 ? std::numeric_limits<double>::quiet_NaN()
                               : (code == 0 ? 2.0 : (code == 2 ? 1.0 : 0.0));
        }
        double f = 0.0;
        int32_t obs = 0;
        if (!orc_prepare_marker(raw.data(), n, min_maf, g.data(), &f, &obs)) continue;
        vinv(g.data(), vg.data());
        double score = 0.0, var = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            score += g[i] * py[i];
            var += g[i] * vg[i];
        }
        for (int64_t a = 0; a < p; ++a) {
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) acc += X[i + a * n] * vg[i];
            xvg[a] = acc;
        }
        for (int64_t a = 0; a < p; ++a) {
            double acc = 0.0;
            for (int64_t b = 0; b < p; ++b) acc += info_inv[a + b * p] * xvg[b];
            mid[a] = acc;
        }
        for (int64_t a = 0; a < p; ++a) var -= xvg[a] * mid[a];
        if (!(var > 1e-12) || !std::isfinite(var)) continue;
        const double stat = score / std::sqrt(var);
        const double pv = orc_chisq_prob(stat * stat, 1);
        tested[j] = 1;
        freq_out[j] = f;
        beta_out[j] = score / var;
        se_out[j] = 1.0 / std::sqrt(var);
        pval_out[j] = pv;
        log10p_out[j] = pv > 0.0 ? -std::log10(pv) : 300.0;
    }
    return 0;
}

int orc_pcg_solve(const uint8_t* bed, int64_t n_fam, int64_t stride,
                  const double* mean, const double* inv_std,
                  const int32_t* keep, int64_t n_keep,
                  const int32_t* variants, int64_t n_var,
                  double sg2, double se2, const double* b, double tol, int max_iter,
                  double* x) {
    Selection s = make_selection(bed, n_fam, stride, mean, inv_std, keep, n_keep, variants, n_var);
    const int64_t n = s.rows();
    auto mult = [&](const double* v, double* out) {
        std::vector<double> kv(n);
        orc_kinship_apply_vector(bed, n_fam, stride, mean, inv_std, keep, n_keep, variants, n_var,
                                 v, kv.data(), 1);
        for (int64_t i = 0; i < n; ++i) out[i] = sg2 * kv[i] + se2 * v[i];
    };
    const double diag = sg2 + se2;
    std::vector<double> r(n), z(n), pdir(n), ap(n);
    std::fill(x, x + n, 0.0);
    mult(x, ap.data());
    double rn = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        r[i] = b[i] - ap[i];
        rn += r[i] * r[i];
    }
    if (std::sqrt(rn) < 1e-20) return 0;
    double rsold = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        z[i] = r[i] / diag;
        pdir[i] = z[i];
        rsold += r[i] * z[i];
    }
    for (int it = 0; it < max_iter; ++it) {
        mult(pdir.data(), ap.data());
        double pap = 0.0;
        for (int64_t i = 0; i < n; ++i) pap += pdir[i] * ap[i];
        const double alpha = rsold / pap;
        rn = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * pdir[i];
            r[i] -= alpha * ap[i];
            rn += r[i] * r[i];
        }
        if (std::sqrt(rn) < tol) return it + 1;
        double rsnew = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            z[i] = r[i] / diag;
            rsnew += r[i] * z[i];
        }
        for (int64_t i = 0; i < n; ++i) pdir[i] = z[i] + (rsnew / rsold) * pdir[i];
        rsold = rsnew;
    }
    return max_iter;
}

}  // extern "C"

// ---------------------------------------------------------------- STCG_VCE
namespace {

// libCosmicCore/src/plink_reader.cpp:355-402 (multiply_Zt_v) and :241-308 (multiply_Z_v)
// over every SNP of the reader, one worker; then apply_G's division by the SNP count
// (libCosmicCore/src/stcg_vce.cpp:80-87).
struct GenoMatrix {
    const uint8_t* bed;
    int64_t n, m, stride;
    const double* mean;
    const double* inv_std;
    // Optional precomputed dense K = Z Z^T / m (n x n, column-major): the same operator applied
    // as one matrix-vector product (rows summed in a fixed order), for sizes where the two
    // genotype passes per CG step would make the restatement too slow to serve as a checker.
    const double* dense_k = nullptr;
    void apply_G(const double* u, double* out) const {
        if (dense_k) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                double acc = 0.0;
                for (int64_t j = 0; j < n; ++j) acc += dense_k[j + i * n] * u[j];
                out[i] = acc;
            }
            return;
        }
        std::vector<double> t(m);
        for (int64_t j = 0; j < m; ++j) {
            const double is = inv_std[j];
            if (is == 0.0) { t[j] = 0.0; continue; }
            const double mu = mean[j];
            const uint8_t* col = bed + j * stride;
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) {
                const int code = code_at(col, i);
                if (code != 1) acc += (static_cast<double>(kLookup[code]) - mu) * u[i];
            }
            t[j] = acc * is;
        }
        std::fill(out, out + n, 0.0);
        for (int64_t j = 0; j < m; ++j) {
            const double is = inv_std[j];
            if (is == 0.0) continue;
            const double mu = mean[j];
            const double w = t[j] * is;
            const double vmap[4] = {(static_cast<double>(kLookup[0]) - mu) * w, 0.0,
                                    (static_cast<double>(kLookup[2]) - mu) * w,
                                    (static_cast<double>(kLookup[3]) - mu) * w};
            const uint8_t* col = bed + j * stride;
            for (int64_t i = 0; i < n; ++i) out[i] += vmap[code_at(col, i)];
        }
        const double denom = (double)std::max<int64_t>(1, m);
        for (int64_t i = 0; i < n; ++i) out[i] /= denom;
    }
};

double dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

// Eigen::LDLT solve of the 3x3 AI system as the reference uses it: a zero pivot (the
// absent permanent-environment component) contributes a zero step.
bool solve_ai(const double AI[3][3], const double g[3], double out[3]) {
    int idx[3], k = 0;
    for (int i = 0; i < 3; ++i)
        if (AI[i][i] != 0.0) idx[k++] = i;
    out[0] = out[1] = out[2] = 0.0;
    std::vector<double> A(k * k), L, D;
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) A[a + b * k] = AI[idx[a]][idx[b]];
    if (!ldlt(A.data(), k, L, D)) return false;
    std::vector<double> r(k);
    for (int a = 0; a < k; ++a) r[a] = g[idx[a]];
    ldlt_solve(L, D, k, r.data());
    for (int a = 0; a < k; ++a) out[idx[a]] = r[a];
    return true;
}

// Symmetric tridiagonal eigen-decomposition (implicit QL); returns eigenvalues and the
// first components of the eigenvectors (all the SLQ quadrature needs).
void tridiag_eig_first(std::vector<double> d, std::vector<double> e, std::vector<double>& evals,
                       std::vector<double>& first) {
    const int n = (int)d.size();
    std::vector<double> Z(n * n, 0.0);
    for (int i = 0; i < n; ++i) Z[i + i * n] = 1.0;
    e.push_back(0.0);
    for (int l = 0; l < n; ++l) {
        int iter = 0, m;
        do {
            for (m = l; m < n - 1; ++m) {
                const double dd = std::abs(d[m]) + std::abs(d[m + 1]);
                if (std::abs(e[m]) <= 1e-15 * dd) break;
            }
            if (m != l) {
                if (++iter > 200) break;
                double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                double r = std::hypot(g, 1.0);
                g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
                double s = 1.0, c = 1.0, p = 0.0;
                int i;
                for (i = m - 1; i >= l; --i) {
                    double f = s * e[i], b = c * e[i];
                    r = std::hypot(f, g);
                    e[i + 1] = r;
                    if (r == 0.0) { d[i + 1] -= p; e[m] = 0.0; break; }
                    s = f / r; c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                    for (int k = 0; k < n; ++k) {
                        f = Z[k + (i + 1) * n];
                        Z[k + (i + 1) * n] = s * Z[k + i * n] + c * f;
                        Z[k + i * n] = c * Z[k + i * n] - s * f;
                    }
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= p; e[l] = g; e[m] = 0.0;
            }
        } while (m != l);
    }
    evals = d;
    first.resize(n);
    for (int i = 0; i < n; ++i) first[i] = Z[0 + i * n];
}

struct Stcg {
    GenoMatrix geno;
    const int32_t* rec_to_ind;  // NULL: record i is genotype row i
    int64_t n_rec, p;
    bool with_pe;
    const double* y;
    const double* X;  // n_rec x p column-major
    double vg = 0.0, vpe = 0.0, ve = 0.0;
    double pcg_tol;
    int pcg_max_iter;
    int64_t pcg_iterations = 0;

    int ind(int64_t i) const { return rec_to_ind ? rec_to_ind[i] : (int)i; }
    // stcg_vce.cpp:64-78
    void gather(const double* v, std::vector<double>& u) const {
        u.assign(geno.n, 0.0);
        for (int64_t i = 0; i < n_rec; ++i)
            if (ind(i) >= 0) u[ind(i)] += v[i];
    }
    void scatter(const std::vector<double>& u, double* out) const {
        for (int64_t i = 0; i < n_rec; ++i) out[i] = ind(i) >= 0 ? u[ind(i)] : 0.0;
    }
    // stcg_vce.cpp:89-101
    void dV_genetic(const double* v, double* out) const {
        std::vector<double> u, gu(geno.n);
        gather(v, u);
        geno.apply_G(u.data(), gu.data());
        scatter(gu, out);
    }
    void dV_pe(const double* v, double* out) const {
        std::vector<double> u;
        gather(v, u);
        scatter(u, out);
    }
    // stcg_vce.cpp:103-115
    void apply_V(const double* v, double* out) const {
        std::vector<double> tmp(n_rec);
        std::fill(out, out + n_rec, 0.0);
        dV_genetic(v, tmp.data());
        for (int64_t i = 0; i < n_rec; ++i) out[i] += vg * tmp[i];
        if (with_pe) {
            dV_pe(v, tmp.data());
            for (int64_t i = 0; i < n_rec; ++i) out[i] += vpe * tmp[i];
        }
        for (int64_t i = 0; i < n_rec; ++i) out[i] += ve * v[i];
    }
    // stcg_vce.cpp:117-126 + matrix_free_pcg.h:20-68 (x0 = 0)
    std::vector<double> solve_V(const std::vector<double>& b) {
        const int64_t n = n_rec;
        std::vector<double> x(n, 0.0), r(b), z(n), pd(n), ap(n);
        if (std::sqrt(dot(r, r)) < 1e-20) return x;
        double diag = std::max(ve, 1e-12) + std::max(vg, 1e-12);
        if (with_pe) diag += std::max(vpe, 1e-12);
        for (int64_t i = 0; i < n; ++i) z[i] = r[i] / diag;
        pd = z;
        double rsold = dot(r, z);
        for (int it = 0; it < pcg_max_iter; ++it) {
            ++pcg_iterations;
            apply_V(pd.data(), ap.data());
            const double alpha = rsold / dot(pd, ap);
            for (int64_t i = 0; i < n; ++i) {
                x[i] += alpha * pd[i];
                r[i] -= alpha * ap[i];
            }
            if (std::sqrt(dot(r, r)) < pcg_tol) return x;
            for (int64_t i = 0; i < n; ++i) z[i] = r[i] / diag;
            const double rsnew = dot(r, z);
            for (int64_t i = 0; i < n; ++i) pd[i] = z[i] + (rsnew / rsold) * pd[i];
            rsold = rsnew;
        }
        return x;
    }
    // stcg_vce.cpp:128-145
    struct Null {
        std::vector<double> Vinv_y, Vinv_X, XtVinvX, XtVinvX_inv, beta;
    };
    bool compute_null(Null& nl) {
        nl.Vinv_y = solve_V(std::vector<double>(y, y + n_rec));
        nl.Vinv_X.assign(n_rec * p, 0.0);
        for (int64_t j = 0; j < p; ++j) {
            std::vector<double> xs = solve_V(std::vector<double>(X + j * n_rec, X + (j + 1) * n_rec));
            std::copy(xs.begin(), xs.end(), nl.Vinv_X.begin() + j * n_rec);
        }
        nl.XtVinvX.assign(p * p, 0.0);
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b) {
                double acc = 0.0;
                for (int64_t i = 0; i < n_rec; ++i) acc += X[i + a * n_rec] * nl.Vinv_X[i + b * n_rec];
                nl.XtVinvX[a + b * p] = acc;
            }
        std::vector<double> L, D;
        nl.XtVinvX_inv.assign(p * p, 0.0);
        nl.beta.assign(p, 0.0);
        if (p == 0) return true;
        if (!ldlt(nl.XtVinvX.data(), p, L, D)) return false;
        for (int64_t c = 0; c < p; ++c) {
            std::vector<double> e(p, 0.0);
            e[c] = 1.0;
            ldlt_solve(L, D, p, e.data());
            for (int64_t r = 0; r < p; ++r) nl.XtVinvX_inv[r + c * p] = e[r];
        }
        std::vector<double> xty(p, 0.0);
        for (int64_t a = 0; a < p; ++a)
            for (int64_t i = 0; i < n_rec; ++i) xty[a] += X[i + a * n_rec] * nl.Vinv_y[i];
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b) nl.beta[a] += nl.XtVinvX_inv[a + b * p] * xty[b];
        return true;
    }
    // stcg_vce.cpp:147-154: P v = V^-1 v - V^-1 X (XtVinvX)^-1 X^T V^-1 v
    std::vector<double> project(const std::vector<double>& vinv_v, const Null& nl) const {
        std::vector<double> xtv(p, 0.0), coef(p, 0.0), out(vinv_v);
        for (int64_t a = 0; a < p; ++a)
            for (int64_t i = 0; i < n_rec; ++i) xtv[a] += X[i + a * n_rec] * vinv_v[i];
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b) coef[a] += nl.XtVinvX_inv[a + b * p] * xtv[b];
        for (int64_t i = 0; i < n_rec; ++i) {
            double acc = 0.0;
            for (int64_t a = 0; a < p; ++a) acc += nl.Vinv_X[i + a * n_rec] * coef[a];
            out[i] -= acc;
        }
        return out;
    }
    std::vector<double> apply_P(const std::vector<double>& v, const Null& nl) {
        return project(solve_V(v), nl);
    }
};

}  // namespace

extern "C" {

static int stcg_vce_impl(const GenoMatrix& geno, const int32_t* rec_to_ind, int64_t n_rec,
                         int with_pe, const double* y, const double* X, int64_t p,
                         const orc_stcg_options* opt, orc_stcg_result* res, double* beta_out,
                         double* a_ind_out, double* pe_ind_out) {
    const int64_t n_fam = geno.n;
    Stcg st{geno, rec_to_ind, n_rec, p, with_pe != 0, y, X};
    st.pcg_tol = opt->pcg_tol;
    st.pcg_max_iter = opt->pcg_max_iter;
    const int64_t n = n_rec;
    // stcg_vce.cpp:157-214: moment-based starting values
    int64_t n_ind = 0;
    for (int64_t i = 0; i < n; ++i) n_ind = std::max<int64_t>(n_ind, st.ind(i) + 1);
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
        const int idx = st.ind(i);
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
    st.ve = ve_guess;
    st.vg = vg_guess;
    st.vpe = st.with_pe ? pe_guess : 0.0;

    std::mt19937_64 rng(opt->probe_seed);
    std::uniform_int_distribution<int> bit(0, 1);
    double last[3] = {NAN, NAN, NAN};
    const int em_warmup = 4;
    const double min_f = 0.5, max_f = 2.0, blend = 0.35;
    res->converged = 0;
    res->iterations = 0;
    res->logl = NAN;
    for (int iter = 0; iter < opt->max_iter; ++iter) {
        Stcg::Null nl;
        if (!st.compute_null(nl)) return -1;
        std::vector<double> Py(n);
        for (int64_t i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int64_t a = 0; a < p; ++a) acc += nl.Vinv_X[i + a * n] * nl.beta[a];
            Py[i] = nl.Vinv_y[i] - acc;
        }
        std::vector<double> s[3], q[3];
        s[0].assign(n, 0.0);
        s[1].assign(n, 0.0);
        s[2] = Py;
        st.dV_genetic(Py.data(), s[0].data());
        if (st.with_pe) st.dV_pe(Py.data(), s[1].data());
        for (int k = 0; k < 3; ++k) q[k] = st.apply_P(s[k], nl);
        double tr[3] = {0, 0, 0};
        for (int t = 0; t < opt->mc_samples; ++t) {
            std::vector<double> z(n);
            for (int64_t i = 0; i < n; ++i) z[i] = bit(rng) ? 1.0 : -1.0;
            std::vector<double> Pz = st.apply_P(z, nl);
            std::vector<double> dg(n), dp(n, 0.0);
            st.dV_genetic(z.data(), dg.data());
            if (st.with_pe) st.dV_pe(z.data(), dp.data());
            tr[0] += dot(Pz, dg);
            tr[1] += dot(Pz, dp);
            tr[2] += dot(Pz, z);
        }
        for (double& t : tr) t /= (double)opt->mc_samples;
        double quad[3], grad[3];
        for (int k = 0; k < 3; ++k) {
            quad[k] = dot(Py, s[k]);
            grad[k] = 0.5 * (quad[k] - tr[k]);
        }
        double AI[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b) AI[a][b] = AI[b][a] = 0.5 * dot(s[a], q[b]);
        const double theta[3] = {st.vg, st.with_pe ? st.vpe : 0.0, st.ve};
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
        for (double& v : next) v = std::max(var_floor, v);
        // stcg_vce.cpp:330-348: REML log-likelihood with the SLQ log-determinant (at the
        // current theta, before the update); the estimator's probes come from one
        // mt19937_64(42 + iter) stream, i.e. its one-thread schedule.
        if (opt->slq_probes > 0) {
            const int m = (int)std::min<int64_t>(opt->slq_steps, n);
            std::mt19937_64 srng(42ull + (uint64_t)iter);
            std::uniform_int_distribution<int> sbit(0, 1);
            double total = 0.0;
            for (int sp = 0; sp < opt->slq_probes; ++sp) {
                std::vector<double> z(n);
                for (int64_t i = 0; i < n; ++i) z[i] = sbit(srng) ? 1.0 : -1.0;
                std::vector<std::vector<double>> V(m + 1, std::vector<double>(n, 0.0));
                const double nz = std::sqrt((double)n);
                for (int64_t i = 0; i < n; ++i) V[0][i] = z[i] / nz;
                std::vector<double> alpha(m, 0.0), beta(m, 0.0);
                int actual = m;
                for (int j = 0; j < m; ++j) {
                    std::vector<double> w(n);
                    st.apply_V(V[j].data(), w.data());
                    if (j > 0)
                        for (int64_t i = 0; i < n; ++i) w[i] -= beta[j - 1] * V[j - 1][i];
                    alpha[j] = dot(w, V[j]);
                    for (int64_t i = 0; i < n; ++i) w[i] -= alpha[j] * V[j][i];
                    for (int k = 0; k <= j; ++k) {
                        const double pr = dot(w, V[k]);
                        for (int64_t i = 0; i < n; ++i) w[i] -= pr * V[k][i];
                    }
                    beta[j] = std::sqrt(dot(w, w));
                    if (beta[j] < 1e-12) {
                        actual = j + 1;
                        break;
                    }
                    for (int64_t i = 0; i < n; ++i) V[j + 1][i] = w[i] / beta[j];
                }
                std::vector<double> d(alpha.begin(), alpha.begin() + actual);
                std::vector<double> e(beta.begin(), beta.begin() + std::max(0, actual - 1));
                std::vector<double> ev, first;
                tridiag_eig_first(d, e, ev, first);
                double ss = 0.0;
                for (int i = 0; i < actual; ++i)
                    ss += first[i] * first[i] * std::log(std::max(ev[i], 1e-12));
                total += (double)n * ss;
            }
            const double logdetV = total / opt->slq_probes;
            std::vector<double> L, D;
            double logdetX = 0.0;
            if (p > 0 && ldlt(nl.XtVinvX.data(), p, L, D))
                for (int64_t a = 0; a < p; ++a) logdetX += std::log(D[a]);
            const double yPy = dot(std::vector<double>(y, y + n), Py);
            res->logl = -0.5 * (logdetV + logdetX + yPy + (double)(n - p) * std::log(2 * M_PI));
        }
        double rel = 0.0;
        if (iter > 0 && std::isfinite(last[0]) && std::isfinite(last[1]) && std::isfinite(last[2]))
            for (int k = 0; k < 3; ++k)
                rel = std::max(rel, std::abs(next[k] - last[k]) / (std::abs(last[k]) + 1e-12));
        for (int k = 0; k < 3; ++k) last[k] = next[k];
        st.vg = next[0];
        if (st.with_pe) st.vpe = next[1];
        st.ve = next[2];
        res->iterations = iter + 1;
        if (iter > 0 && rel < opt->tol) {
            res->converged = 1;
            break;
        }
    }
    // stcg_vce.cpp:371-406: final BLUE / BLUP
    Stcg::Null nl;
    if (!st.compute_null(nl)) return -1;
    std::vector<double> Py(n);
    for (int64_t i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int64_t a = 0; a < p; ++a) acc += nl.Vinv_X[i + a * n] * nl.beta[a];
        Py[i] = nl.Vinv_y[i] - acc;
    }
    std::vector<double> zi, ai(n_fam);
    st.gather(Py.data(), zi);
    st.geno.apply_G(zi.data(), ai.data());
    if (beta_out) std::copy(nl.beta.begin(), nl.beta.end(), beta_out);
    for (int64_t i = 0; i < n_fam; ++i) {
        if (a_ind_out) a_ind_out[i] = ai[i] * st.vg;
        if (pe_ind_out) pe_ind_out[i] = st.with_pe ? st.vpe * zi[i] : 0.0;
    }
    res->sigma2_g = st.vg;
    res->sigma2_pe = st.with_pe ? st.vpe : 0.0;
    res->sigma2_e = st.ve;
    res->pcg_iterations = st.pcg_iterations;
    return 0;
}

int orc_stcg_vce(const uint8_t* bed, int64_t n_fam, int64_t stride, int64_t n_snps,
                 const double* mean, const double* inv_std, const int32_t* rec_to_ind,
                 int64_t n_rec, int with_pe, const double* y, const double* X, int64_t p,
                 const orc_stcg_options* opt, orc_stcg_result* res, double* beta_out,
                 double* a_ind_out, double* pe_ind_out) {
    return stcg_vce_impl(GenoMatrix{bed, n_fam, n_snps, stride, mean, inv_std}, rec_to_ind, n_rec,
                         with_pe, y, X, p, opt, res, beta_out, a_ind_out, pe_ind_out);
}

int orc_stcg_vce_dense(const double* K, int64_t n_fam, const int32_t* rec_to_ind, int64_t n_rec,
                       int with_pe, const double* y, const double* X, int64_t p,
                       const orc_stcg_options* opt, orc_stcg_result* res, double* beta_out,
                       double* a_ind_out, double* pe_ind_out) {
    GenoMatrix geno{nullptr, n_fam, 0, 0, nullptr, nullptr};
    geno.dense_k = K;
    return stcg_vce_impl(geno, rec_to_ind, n_rec, with_pe, y, X, p, opt, res, beta_out, a_ind_out,
                         pe_ind_out);
}

}  // extern "C"

// ---------------------------------------------------------------- scanSTCG
extern "C" {

// src/models/repeatability_scan_stcg.cpp:42-140 (scan_stcg_with_grm) over SNPs
// [snp_begin, snp_end) of the packed rows; dense FP64, one LDLT solve per SNP as written.
int orc_stcg_scan(const uint8_t* bed, int64_t n_fam, int64_t stride, const double* G, int64_t q,
                  const int32_t* subject_rows, const int32_t* obs_to_subject, int64_t n_obs,
                  const double* y, const double* X, int64_t p, double vg, double vpe, double ve,
                  double min_maf, int64_t snp_begin, int64_t snp_end, double* beta, double* se,
                  double* pval, double* log10p, double* maf_out, int32_t* tested) {
    (void)n_fam;
    std::vector<double> D(q, 0.0), K(q * q);
    for (int64_t i = 0; i < n_obs; ++i) D[obs_to_subject[i]] += 1.0;
    for (int64_t c = 0; c < q; ++c)
        for (int64_t r = 0; r < q; ++r) K[r + c * q] = vg * G[r + c * q] + (r == c ? vpe : 0.0);
    std::vector<double> L, Dl;
    if (!ldlt(K.data(), q, L, Dl)) return -1;
    std::vector<double> M(q * q, 0.0);
    for (int64_t c = 0; c < q; ++c) {
        M[c + c * q] = 1.0;
        ldlt_solve(L, Dl, q, M.data() + c * q);
    }
    for (int64_t s2 = 0; s2 < q; ++s2) M[s2 + s2 * q] += D[s2] / ve;
    std::vector<double> LM, DM;
    if (!ldlt(M.data(), q, LM, DM)) return -2;
    auto woodbury = [&](const double* v, double* out) {
        std::vector<double> z(q, 0.0);
        for (int64_t i = 0; i < n_obs; ++i) z[obs_to_subject[i]] += v[i];
        ldlt_solve(LM, DM, q, z.data());
        for (int64_t i = 0; i < n_obs; ++i) out[i] = v[i] / ve - z[obs_to_subject[i]] / (ve * ve);
    };
    std::vector<double> Vy(n_obs), VX(n_obs * p);
    woodbury(y, Vy.data());
    for (int64_t a = 0; a < p; ++a) woodbury(X + a * n_obs, VX.data() + a * n_obs);
    std::vector<double> XtVX(p * p, 0.0), Xty(p, 0.0);
    for (int64_t a = 0; a < p; ++a) {
        for (int64_t b = 0; b < p; ++b)
            for (int64_t i = 0; i < n_obs; ++i) XtVX[a + b * p] += X[i + a * n_obs] * VX[i + b * n_obs];
        for (int64_t i = 0; i < n_obs; ++i) Xty[a] += X[i + a * n_obs] * Vy[i];
    }
    std::vector<double> LX, DX;
    if (p > 0 && !ldlt(XtVX.data(), p, LX, DX)) return -3;
    std::vector<double> bh(Xty);
    if (p > 0) ldlt_solve(LX, DX, p, bh.data());
    std::vector<double> resid(n_obs), Py(n_obs);
    for (int64_t i = 0; i < n_obs; ++i) {
        double fit = 0.0;
        for (int64_t a = 0; a < p; ++a) fit += X[i + a * n_obs] * bh[a];
        resid[i] = y[i] - fit;
    }
    woodbury(resid.data(), Py.data());
    std::vector<double> g(n_obs), Vg(n_obs), t(p);
    for (int64_t j = snp_begin; j < snp_end; ++j) {
        const int64_t o = j - snp_begin;
        const uint8_t* row = bed + j * stride;
        double sum_g = 0.0;
        int valid_n = 0;
        for (int64_t i = 0; i < n_obs; ++i) {
            const int code = code_at(row, subject_rows[obs_to_subject[i]]);
            const float val = kLookup[code];
            g[i] = val;
            if (!std::isnan(val)) {
                sum_g += val;
                ++valid_n;
            } else {
                g[i] = 0.0;
            }
        }
        tested[o] = 0;
        beta[o] = se[o] = pval[o] = log10p[o] = NAN;
        double maf = valid_n > 0 ? sum_g / (2.0 * valid_n) : 0.0;
        if (maf > 0.5) maf = 1.0 - maf;
        maf_out[o] = maf;
        if (valid_n < 10) continue;
        if (maf < min_maf) continue;
        const double gm = sum_g / valid_n;
        for (int64_t i = 0; i < n_obs; ++i) g[i] -= gm;
        double score = 0.0;
        for (int64_t i = 0; i < n_obs; ++i) score += g[i] * Py[i];
        woodbury(g.data(), Vg.data());
        for (int64_t a = 0; a < p; ++a) {
            t[a] = 0.0;
            for (int64_t i = 0; i < n_obs; ++i) t[a] += X[i + a * n_obs] * Vg[i];
        }
        if (p > 0) ldlt_solve(LX, DX, p, t.data());
        double var = 0.0;
        for (int64_t i = 0; i < n_obs; ++i) {
            double pg = Vg[i];
            for (int64_t a = 0; a < p; ++a) pg -= VX[i + a * n_obs] * t[a];
            var += g[i] * pg;
        }
        if (var < 1e-15) continue;
        const double z = score / std::sqrt(var);
        const double pv = std::erfc(std::abs(z) / std::sqrt(2.0));
        tested[o] = 1;
        beta[o] = score / var;
        se[o] = 1.0 / std::sqrt(var);
        pval[o] = pv;
        log10p[o] = (pv > 0.0 && pv <= 1.0) ? -std::log10(pv) : (pv > 1.0 ? 0.0 : 300.0);
    }
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------- MvLMM scan
namespace {

// mvlmm_numerics.h:27-45 / :47-69 with the Jacobi eigensolver: 0 OK, 1 roundoff,
// 2 boundary, 3 singular.
int mv_invert(const std::vector<double>& info, int64_t d, std::vector<double>& cov) {
    for (double v : info)
        if (!std::isfinite(v)) return 3;
    std::vector<double> sym(d * d), ev(d), V(d * d);
    for (int64_t a = 0; a < d; ++a)
        for (int64_t b = 0; b < d; ++b) sym[a + b * d] = 0.5 * (info[a + b * d] + info[b + a * d]);
    jacobi_eigh(sym.data(), d, ev.data(), V.data());
    double mn = ev[0], mx = 0.0;
    for (double v : ev) {
        mn = std::min(mn, v);
        mx = std::max(mx, std::abs(v));
    }
    const double tol = 128.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, mx) * d;
    if (!(mn > tol)) return 3;
    cov.assign(d * d, 0.0);
    for (int64_t a = 0; a < d; ++a)
        for (int64_t b = 0; b < d; ++b)
            for (int64_t l = 0; l < d; ++l) cov[a + b * d] += V[a + l * d] * V[b + l * d] / ev[l];
    for (int64_t a = 0; a < d; ++a)
        for (int64_t b = a + 1; b < d; ++b) cov[a + b * d] = cov[b + a * d] = 0.5 * (cov[a + b * d] + cov[b + a * d]);
    return 0;
}

int mv_condition(std::vector<double>& cov, int64_t d) {
    for (int64_t a = 0; a < d; ++a)
        for (int64_t b = a + 1; b < d; ++b) cov[a + b * d] = cov[b + a * d] = 0.5 * (cov[a + b * d] + cov[b + a * d]);
    std::vector<double> ev(d), V(d * d);
    jacobi_eigh(cov.data(), d, ev.data(), V.data());
    double mn = ev[0], mx = 0.0;
    for (double v : ev) {
        mn = std::min(mn, v);
        mx = std::max(mx, std::abs(v));
    }
    const double tol = 128.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, mx) * d;
    if (mn < -tol) return 3;
    if (mn < 0.0) {
        std::fill(cov.begin(), cov.end(), 0.0);
        for (int64_t a = 0; a < d; ++a)
            for (int64_t b = 0; b < d; ++b)
                for (int64_t l = 0; l < d; ++l) cov[a + b * d] += V[a + l * d] * V[b + l * d] * std::max(ev[l], 0.0);
        for (int64_t a = 0; a < d; ++a)
            for (int64_t b = a + 1; b < d; ++b) cov[a + b * d] = cov[b + a * d] = 0.5 * (cov[a + b * d] + cov[b + a * d]);
        return 1;
    }
    return mn <= tol ? 2 : 0;
}

// (d x d) inverse of an SPD matrix through LDL^T (Sigma.llt().solve(I) in the reference)
std::vector<double> spd_inv(const std::vector<double>& A, int64_t d) {
    std::vector<double> L, D, X(d * d, 0.0);
    ldlt(A.data(), d, L, D);
    for (int64_t c = 0; c < d; ++c) {
        X[c + c * d] = 1.0;
        ldlt_solve(L, D, d, X.data() + c * d);
    }
    return X;
}

}  // namespace

extern "C" {

// src/mvlmm_engine.cpp:756-931 + processBlock :210-396, default options
int orc_mvlmm_scan(const uint8_t* bed, int64_t n_fam, int64_t stride, const int32_t* keep,
                   int64_t n, const double* W, int64_t r, const double* Dv, const double* Uty,
                   int64_t d, const double* UtX, int64_t p, const double* Vg, const double* Ve,
                   int64_t snp_begin, int64_t snp_end, double* beta, double* cov, double* wald,
                   double* pvalue, double* freq, int32_t* status) {
    (void)n_fam;
    std::vector<std::vector<double>> Si(r);
    for (int64_t i = 0; i < r; ++i) {
        std::vector<double> S(d * d);
        for (int64_t a = 0; a < d * d; ++a) S[a] = Dv[i] * Vg[a] + Ve[a];
        Si[i] = spd_inv(S, d);
    }
    const int64_t pd = p * d;
    std::vector<double> HXX(pd * pd, 0.0), RHSX(pd, 0.0);
    for (int64_t i = 0; i < r; ++i) {
        std::vector<double> siy(d, 0.0);
        for (int64_t a = 0; a < d; ++a)
            for (int64_t b = 0; b < d; ++b) siy[a] += Si[i][a + b * d] * Uty[i + b * r];
        for (int64_t j = 0; j < p; ++j) {
            for (int64_t k = 0; k < p; ++k)
                for (int64_t a = 0; a < d; ++a)
                    for (int64_t b = 0; b < d; ++b)
                        HXX[(j * d + a) + (k * d + b) * pd] += UtX[i + j * r] * UtX[i + k * r] * Si[i][a + b * d];
            for (int64_t a = 0; a < d; ++a) RHSX[j * d + a] += UtX[i + j * r] * siy[a];
        }
    }
    std::vector<double> HXXi = pd > 0 ? spd_inv(HXX, pd) : std::vector<double>();
    std::vector<double> s(n), srot(r);
    for (int64_t snp = snp_begin; snp < snp_end; ++snp) {
        const int64_t o = snp - snp_begin;
        const uint8_t* row = bed + snp * stride;
        double sum = 0.0;
        int count = 0;
        for (int64_t i = 0; i < n; ++i) {
            const float v = kLookup[code_at(row, keep[i])];
            s[i] = v;
            if (!std::isnan(v)) {
                sum += v;
                ++count;
            }
        }
        const double mean = count > 0 ? sum / count : 0.0;
        for (int64_t i = 0; i < n; ++i) s[i] = std::isnan(s[i]) ? 0.0 : s[i] - mean;
        for (int64_t c = 0; c < r; ++c) {
            double acc = 0.0;
            for (int64_t i = 0; i < n; ++i) acc += W[i + c * n] * s[i];
            srot[c] = acc;
        }
        std::vector<double> HSS(d * d, 0.0), RHSS(d, 0.0), HXS(pd * d, 0.0);
        for (int64_t i = 0; i < r; ++i) {
            const double si = srot[i];
            std::vector<double> siy(d, 0.0);
            for (int64_t a = 0; a < d; ++a)
                for (int64_t b = 0; b < d; ++b) siy[a] += Si[i][a + b * d] * Uty[i + b * r];
            for (int64_t a = 0; a < d * d; ++a) HSS[a] += si * si * Si[i][a];
            for (int64_t a = 0; a < d; ++a) RHSS[a] += si * siy[a];
            for (int64_t j = 0; j < p; ++j)
                for (int64_t a = 0; a < d; ++a)
                    for (int64_t b = 0; b < d; ++b)
                        HXS[(j * d + a) + b * pd] += UtX[i + j * r] * si * Si[i][a + b * d];
        }
        std::vector<double> schur(HSS), adj(RHSS);
        for (int64_t a = 0; a < d; ++a) {
            for (int64_t b = 0; b < d; ++b) {
                double acc = 0.0;
                for (int64_t u = 0; u < pd; ++u)
                    for (int64_t v = 0; v < pd; ++v) acc += HXS[u + a * pd] * HXXi[u + v * pd] * HXS[v + b * pd];
                schur[a + b * d] -= acc;
            }
            double acc = 0.0;
            for (int64_t u = 0; u < pd; ++u)
                for (int64_t v = 0; v < pd; ++v) acc += HXS[u + a * pd] * HXXi[u + v * pd] * RHSX[v];
            adj[a] -= acc;
        }
        freq[o] = mean / 2.0;
        wald[o] = pvalue[o] = NAN;
        status[o] = 3;
        std::vector<double> sinv;
        if (mv_invert(schur, d, sinv) != 0) continue;
        for (int64_t a = 0; a < d; ++a)
            for (int64_t b = a + 1; b < d; ++b) schur[a + b * d] = schur[b + a * d] = 0.5 * (schur[a + b * d] + schur[b + a * d]);
        std::vector<double> bt(d, 0.0);
        for (int64_t a = 0; a < d; ++a)
            for (int64_t b = 0; b < d; ++b) bt[a] += sinv[a + b * d] * adj[b];
        double w2 = 0.0;
        for (int64_t a = 0; a < d; ++a)
            for (int64_t b = 0; b < d; ++b) w2 += bt[a] * schur[a + b * d] * bt[b];
        if (!std::isfinite(w2) || w2 < 0.0) continue;
        const int cst = mv_condition(sinv, d);
        if (cst == 3) continue;
        status[o] = cst;
        wald[o] = w2;
        pvalue[o] = orc_chisq_prob(w2, (int)d);
        for (int64_t a = 0; a < d; ++a) beta[o * d + a] = bt[a];
        for (int64_t a = 0; a < d * d; ++a) cov[o * d * d + a] = sinv[a];
    }
    return 0;
}


// ---------------------------------------------------------------- timed CPU restatement helpers
// Byte-at-a-time table decode of SNP columns snps[0..count) (every sample), as the reference's
// apply_block does per 512-SNP block (kinship_operator.cpp:265-285).
void orc_decode_z_cols(const uint8_t* bed, int64_t stride, const double* mean,
                       const double* inv_std, const int32_t* snps, int64_t count, int64_t n,
                       double* z, int64_t ldz, int n_threads) {
#pragma omp parallel for num_threads(std::max(1, n_threads)) schedule(static)
    for (int64_t j = 0; j < count; ++j) {
        const int64_t snp = snps[j];
        const double mu = mean[snp], is = inv_std[snp];
        double* dest = z + j * ldz;
        if (is == 0.0) {
            std::fill(dest, dest + n, 0.0);
            continue;
        }
        const double values[4] = {(2.0 - mu) * is, 0.0, (1.0 - mu) * is, -mu * is};
        double quad[256][4];
        for (int b = 0; b < 256; ++b)
            for (int q = 0; q < 4; ++q) quad[b][q] = values[(b >> (2 * q)) & 3];
        const uint8_t* col = bed + snp * stride;
        const int64_t full = n >> 2;
        for (int64_t b = 0; b < full; ++b) std::memcpy(dest + 4 * b, quad[col[b]], 32);
        for (int64_t r = full << 2; r < n; ++r) dest[r] = values[code_at(col, r)];
    }
}

// genotype_encoding.h:33-81 for every sample: raw dosage 2/1/0 (NaN for code 01), observed
// count, A1 frequency = sum / (2 obs), pass = obs >= 3 and MAF >= min_maf; the encoded
// column is raw - mean with missing calls at the mean (so 0 after centring); gsq = its
// sum of squares.
void orc_scan_encode_cols(const uint8_t* bed, int64_t stride, int64_t first, int64_t count,
                          int64_t n, double min_maf, double* g, int64_t ldg, double* freq,
                          int32_t* pass, double* gsq, int n_threads) {
#pragma omp parallel for num_threads(std::max(1, n_threads)) schedule(static)
    for (int64_t j = 0; j < count; ++j) {
        const uint8_t* col = bed + (first + j) * stride;
        double* dest = g + j * ldg;
        double sum = 0.0;
        int observed = 0;
        for (int64_t i = 0; i < n; ++i) {
            const int code = code_at(col, i);
            if (code == 1) continue;
            sum += code == 0 ? 2.0 : (code == 2 ? 1.0 : 0.0);
            ++observed;
        }
        freq[j] = 0.0;
        pass[j] = 0;
        gsq[j] = 0.0;
        if (observed == 0) {
            std::fill(dest, dest + n, 0.0);
            continue;
        }
        const double af = sum / (2.0 * observed);
        freq[j] = af;
        pass[j] = observed >= 3 && std::min(af, 1.0 - af) >= min_maf;
        const double m = sum / observed;
        const double values[4] = {2.0 - m, 0.0, 1.0 - m, 0.0 - m};
        double sq = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            dest[i] = values[code_at(col, i)];
            sq += dest[i] * dest[i];
        }
        gsq[j] = sq;
    }
}

void orc_chisq_prob_vec(const double* stat, int64_t count, int df, double* out, int n_threads) {
#pragma omp parallel for num_threads(std::max(1, n_threads)) schedule(static)
    for (int64_t j = 0; j < count; ++j) out[j] = orc_chisq_prob(stat[j], df);
}


// A Rademacher block from std::mt19937_64(seed) through std::uniform_int_distribution<int>(0, 1)
// (libCosmicCore/src/stcg_vce.cpp:215-216, 249-251): after `skip` draws, column c (c < cols) of
// the n x cols column-major output takes the next draws c*n .. c*n + n - 1, mapped 1 -> +1,
// 0 -> -1.  The multi-trait matrix-free REML's probes follow this stream.
void orc_rademacher(uint64_t seed, int64_t skip, int64_t n, int64_t cols, double* out) {
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> bit(0, 1);
    for (int64_t i = 0; i < skip; ++i) (void)bit(rng);
    for (int64_t c = 0; c < cols; ++c)
        for (int64_t i = 0; i < n; ++i) out[i + c * n] = bit(rng) ? 1.0 : -1.0;
}
}  // extern "C"
