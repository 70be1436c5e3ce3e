// Small dense linear algebra on the host (projected Krylov matrices, p x p block factors).
#pragma once

#include <complex>
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

// Complex Schur form of the real n x n column-major matrix a: a = U T U^H with T upper triangular
// and U unitary (both column-major, complex). Throws std::runtime_error if the QR iteration fails.
void complex_schur(int n, const std::vector<double>& a, std::vector<std::complex<double>>& T,
                   std::vector<std::complex<double>>& U);

// Reorders a complex Schur form so that the diagonal entries appear by ascending key (key[i] belongs
// to the entry at position i on entry), by adjacent swaps (unitary, T stays triangular).
void schur_sort(int n, std::vector<std::complex<double>>& T, std::vector<std::complex<double>>& U,
                const std::vector<double>& key);

// Eigenvectors y_k (k < count, unit 2-norm, in Schur coordinates: x_k = U y_k) of the upper
// triangular T. Diagonal entries within cluster_rtol of T(k, k) just above k form one block whose
// members keep their own coordinates, so a multiple eigenvalue gets independent vectors.
std::vector<std::complex<double>> schur_eigenvectors(int n, const std::vector<std::complex<double>>& T, int count,
                                                     double cluster_rtol);

// Greedy orthonormal basis (m x r, column-major, r <= want returned) drawn from the `count` pool
// vectors (m x count, column-major; parts of unit vectors, so norms are comparable): each step takes
// the pool vector with the largest remainder norm after projection on the basis so far (two passes),
// and the basis stops when that largest remainder falls below min_norm. A direction that is only
// rounding noise (a tiny part, such as the imaginary part of a nearly real vector) is therefore never
// taken while a genuine one is left.
std::vector<double> pivoted_basis(int m, int count, const std::vector<double>& pool, int want, double min_norm, int& r);

}  // namespace hsg
