// Small dense linear algebra on the host (projected Krylov matrices, p x p block factors).
#pragma once

#include <cstdint>
#include <vector>

namespace hsg {

// Symmetric eigendecomposition of the n x n column-major matrix a (lower triangle read):
// eigenvalues ascending into w, orthonormal eigenvectors overwrite a (column j <-> w[j]).
// Householder tridiagonalization followed by implicit QL with Wilkinson shifts.
void sym_eig(int n, std::vector<double>& a, std::vector<double>& w);

// Lower Cholesky of the p x p SPD matrix g (column-major); returns false if not positive definite
// (or the smallest pivot is below rel_tol * largest diagonal entry).
bool cholesky(int p, const std::vector<double>& g, std::vector<double>& l, double rel_tol = 0.0);

// Inverse of a lower-triangular p x p matrix.
std::vector<double> lower_inverse(int p, const std::vector<double>& l);

// c = a * b (column-major, a: m x k, b: k x n)
std::vector<double> matmul(int m, int k, int n, const std::vector<double>& a, const std::vector<double>& b);

}  // namespace hsg
