// Small dense FP64 algebra on the host (k x k with k <= a few hundred; p x p; 3 x 3).
// Column-major storage, a[r + c * n].
#pragma once
#include <cstdint>
#include <vector>

namespace cs {
namespace la {

// G = R^T R (R upper triangular, positive diagonal).  Returns false if G is not
// numerically positive definite.
bool cholesky_upper(const std::vector<double>& G, int n, std::vector<double>& R);
// Inverse of an upper-triangular matrix.
std::vector<double> upper_inverse(const std::vector<double>& R, int n);
// Symmetric eigendecomposition (Householder tridiagonalisation + implicit QL).  Reads
// the lower triangle of A.  Eigenvalues ascending; column j of V is the j-th vector.
bool eigh(const std::vector<double>& A, int n, std::vector<double>& evals, std::vector<double>& V);
// The same up to the eigenvectors: eigenvalues d (unsorted), the tridiagonalising Q
// (column-major) and the QL plane rotations; applying every rotation in order to columns
// (i, i+1) of Q as (q_i, q_{i+1}) <- (c q_i - s q_{i+1}, s q_i + c q_{i+1}) turns column j
// of Q into the eigenvector of d[j].
struct PlaneRotation {
    int32_t i;
    double c, s;
};
bool tridiag_ql(const std::vector<double>& A, int n, std::vector<double>& d,
                std::vector<double>& Q, std::vector<PlaneRotation>& rots);
// LDL^T without pivoting of a small symmetric matrix; false when a pivot is not > 0
// (the reference rejects non-positive LDLT factorisations).
bool ldlt(const std::vector<double>& A, int n, std::vector<double>& L, std::vector<double>& D);
void ldlt_solve(const std::vector<double>& L, const std::vector<double>& D, int n, double* b);
std::vector<double> ldlt_inverse(const std::vector<double>& L, const std::vector<double>& D, int n);

}  // namespace la
}  // namespace cs
