// Test harness: plain C entry points over the host dense routines of hsolve_b200/csrc/dense_host.cpp,
// built by tests/test_dense_host.py into a temporary shared object and called through ctypes.
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
