// Test harness: plain C entry points over the host dense routines of hsolve_b200/csrc/dense_host.cpp,
// built by tests/test_dense_host.py into a temporary shared object and called through ctypes.
#include <complex>
#include <cstring>
#include <vector>

#include "dense_host.hpp"

extern "C" {

int t_sym_eig(int n, const double* a_in, double* w_out, double* v_out) {
  std::vector<double> a(a_in, a_in + static_cast<std::size_t>(n) * n), w;
  try {
    hsg::sym_eig(n, a, w);
  } catch (...) {
    return 1;
  }
  std::memcpy(w_out, w.data(), sizeof(double) * n);
  std::memcpy(v_out, a.data(), sizeof(double) * static_cast<std::size_t>(n) * n);
  return 0;
}

int t_cholesky(int p, const double* g_in, double rel_tol, double* l_out) {
  std::vector<double> g(g_in, g_in + static_cast<std::size_t>(p) * p), l;
  const bool ok = hsg::cholesky(p, g, l, rel_tol);
  if (ok) std::memcpy(l_out, l.data(), sizeof(double) * static_cast<std::size_t>(p) * p);
  return ok ? 1 : 0;
}

void t_lower_inverse(int p, const double* l_in, double* out) {
  std::vector<double> l(l_in, l_in + static_cast<std::size_t>(p) * p);
  const std::vector<double> inv = hsg::lower_inverse(p, l);
  std::memcpy(out, inv.data(), sizeof(double) * static_cast<std::size_t>(p) * p);
}

void t_matmul(int m, int k, int n, const double* a_in, const double* b_in, double* c_out) {
  std::vector<double> a(a_in, a_in + static_cast<std::size_t>(m) * k), b(b_in, b_in + static_cast<std::size_t>(k) * n);
  const std::vector<double> c = hsg::matmul(m, k, n, a, b);
  std::memcpy(c_out, c.data(), sizeof(double) * static_cast<std::size_t>(m) * n);
}

}  // extern "C"

// complex Schur form, sorted by key, and the first `count` eigenvectors (interleaved re/im)
extern "C" int t_schur(int n, const double* a_in, const double* key, int count, double cluster_rtol, double* t_out, double* u_out,
            double* y_out) {
  std::vector<double> a(a_in, a_in + static_cast<std::size_t>(n) * n);
  std::vector<std::complex<double>> T, U;
  try {
    hsg::complex_schur(n, a, T, U);
    if (key) {
      // keys computed by the caller for the eigenvalues as the unsorted form lists them are not
      // available; the harness sorts by -|t_ii| (largest magnitude first)
      std::vector<double> k(n);
      for (int i = 0; i < n; ++i) k[i] = -std::abs(T[static_cast<std::size_t>(i) * (n + 1)]);
      hsg::schur_sort(n, T, U, k);
    }
    const std::vector<std::complex<double>> Y = hsg::schur_eigenvectors(n, T, count, cluster_rtol);
    std::memcpy(t_out, T.data(), sizeof(double) * 2 * T.size());
    std::memcpy(u_out, U.data(), sizeof(double) * 2 * U.size());
    std::memcpy(y_out, Y.data(), sizeof(double) * 2 * Y.size());
  } catch (...) {
    return 1;
  }
  return 0;
}

// greedy orthonormal basis of a pool of vectors; returns its column count
extern "C" int t_pivoted_basis(int m, int count, const double* pool_in, int want, double min_norm, double* q_out) {
  std::vector<double> pool(pool_in, pool_in + static_cast<std::size_t>(m) * count);
  int r = 0;
  const std::vector<double> q = hsg::pivoted_basis(m, count, pool, want, min_norm, r);
  std::memcpy(q_out, q.data(), sizeof(double) * q.size());
  return r;
}
