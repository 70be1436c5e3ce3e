// Small dense linear algebra (see dense_host.hpp): the textbook Householder reduction to
// tridiagonal form and the implicit QL iteration with Wilkinson shifts, written for this project.
#include "dense_host.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <stdexcept>

namespace hsg {

namespace {

// Reduce symmetric a (n x n, col-major, full) to tridiagonal T = Q^T a Q; a is overwritten by Q,
// d = diag(T), e[i] = T(i+1, i) for i < n-1, e[n-1] = 0.
void tridiagonalize(int n, std::vector<double>& a, std::vector<double>& d, std::vector<double>& e) {
  auto A = [&](int i, int j) -> double& { return a[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * n]; };
  // symmetrize from the lower triangle
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < j; ++i) A(i, j) = A(j, i);
  std::vector<double> q(static_cast<std::size_t>(n) * n, 0.0);
  auto Q = [&](int i, int j) -> double& { return q[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * n]; };
  for (int i = 0; i < n; ++i) Q(i, i) = 1.0;
  std::vector<double> v(n), pv(n), wv(n), uq(n);
  d.assign(n, 0.0);
  e.assign(n, 0.0);
  for (int k = 0; k + 2 < n; ++k) {
    // Householder vector for x = A(k+1:n, k)
    double alpha = 0.0;
    for (int i = k + 1; i < n; ++i) alpha += A(i, k) * A(i, k);
    alpha = std::sqrt(alpha);
    if (alpha == 0.0) continue;
    const double x0 = A(k + 1, k);
    const double s = x0 >= 0 ? -alpha : alpha;  // target value of the first entry
    double vnorm2 = 0.0;
    for (int i = k + 1; i < n; ++i) { v[i] = A(i, k); }
    v[k + 1] = x0 - s;
    for (int i = k + 1; i < n; ++i) vnorm2 += v[i] * v[i];
    if (vnorm2 == 0.0) continue;
    const double beta = 2.0 / vnorm2;
    // p = beta * A v (trailing block; A symmetric, so column i gives row i contiguously),
    // K = beta/2 v^T p, w = p - K v
    for (int i = k + 1; i < n; ++i) {
      const double* ai = &A(0, i);
      double sum = 0.0;
      for (int j = k + 1; j < n; ++j) sum += ai[j] * v[j];
      pv[i] = beta * sum;
    }
    double kk = 0.0;
    for (int i = k + 1; i < n; ++i) kk += v[i] * pv[i];
    kk *= 0.5 * beta;
    for (int i = k + 1; i < n; ++i) wv[i] = pv[i] - kk * v[i];
    for (int j = k + 1; j < n; ++j)
      for (int i = k + 1; i < n; ++i) A(i, j) -= v[i] * wv[j] + wv[i] * v[j];
    A(k + 1, k) = s;
    A(k, k + 1) = s;
    for (int i = k + 2; i < n; ++i) { A(i, k) = 0.0; A(k, i) = 0.0; }
    // Q = Q H, H = I - beta v v^T: u = Q v by columns, then Q -= beta u v^T by columns
    std::fill(uq.begin(), uq.end(), 0.0);
    for (int j = k + 1; j < n; ++j) {
      const double vj = v[j];
      const double* qj = &Q(0, j);
      for (int i = 0; i < n; ++i) uq[i] += qj[i] * vj;
    }
    for (int j = k + 1; j < n; ++j) {
      const double c = beta * v[j];
      double* qj = &Q(0, j);
      for (int i = 0; i < n; ++i) qj[i] -= uq[i] * c;
    }
  }
  for (int i = 0; i < n; ++i) d[i] = A(i, i);
  for (int i = 0; i + 1 < n; ++i) e[i] = A(i + 1, i);
  a.swap(q);
}

// Implicit QL with Wilkinson shifts on (d, e); z accumulates the rotations (n x n, col-major).
void tridiagonal_ql(int n, std::vector<double>& d, std::vector<double>& e, std::vector<double>& z) {
  auto Z = [&](int i, int j) -> double& { return z[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * n]; };
  const double eps = std::numeric_limits<double>::epsilon();
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    while (true) {
      int m = l;
      for (; m < n - 1; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= eps * dd) break;
      }
      if (m == l) break;
      if (++iter > 60) throw std::runtime_error("tridiagonal QL did not converge");
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool deflated = false;
      for (; i >= l; --i) {
        double f = s * e[i];
        const double b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        for (int k = 0; k < n; ++k) {
          f = Z(k, i + 1);
          Z(k, i + 1) = s * Z(k, i) + c * f;
          Z(k, i) = c * Z(k, i) - s * f;
        }
      }
      if (deflated) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
}

}  // namespace

void sym_eig(int n, std::vector<double>& a, std::vector<double>& w) {
  if (n == 0) { w.clear(); return; }
  if (n == 1) { w.assign(1, a[0]); a[0] = 1.0; return; }
  std::vector<double> d, e;
  tridiagonalize(n, a, d, e);
  tridiagonal_ql(n, d, e, a);
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](int x, int y) { return d[x] < d[y]; });
  std::vector<double> z(a.size());
  w.resize(n);
  for (int j = 0; j < n; ++j) {
    w[j] = d[idx[j]];
    std::copy(a.begin() + static_cast<std::ptrdiff_t>(idx[j]) * n, a.begin() + static_cast<std::ptrdiff_t>(idx[j] + 1) * n,
              z.begin() + static_cast<std::ptrdiff_t>(j) * n);
  }
  a.swap(z);
}

bool cholesky(int p, const std::vector<double>& g, std::vector<double>& l, double rel_tol) {
  l.assign(static_cast<std::size_t>(p) * p, 0.0);
  double dmax = 0.0;
  for (int i = 0; i < p; ++i) dmax = std::max(dmax, g[i + i * p]);
  if (!(dmax > 0.0)) return false;
  for (int j = 0; j < p; ++j) {
    double s = g[j + j * p];
    for (int k = 0; k < j; ++k) s -= l[j + k * p] * l[j + k * p];
    if (!(s > rel_tol * dmax) || !std::isfinite(s)) return false;
    const double ljj = std::sqrt(s);
    l[j + j * p] = ljj;
    for (int i = j + 1; i < p; ++i) {
      double t = g[i + j * p];
      for (int k = 0; k < j; ++k) t -= l[i + k * p] * l[j + k * p];
      l[i + j * p] = t / ljj;
    }
  }
  return true;
}

std::vector<double> lower_inverse(int p, const std::vector<double>& l) {
  std::vector<double> inv(static_cast<std::size_t>(p) * p, 0.0);
  for (int j = 0; j < p; ++j) {
    inv[j + j * p] = 1.0 / l[j + j * p];
    for (int i = j + 1; i < p; ++i) {
      double s = 0.0;
      for (int k = j; k < i; ++k) s += l[i + k * p] * inv[k + j * p];
      inv[i + j * p] = -s / l[i + i * p];
    }
  }
  return inv;
}

std::vector<double> matmul(int m, int k, int n, const std::vector<double>& a, const std::vector<double>& b) {
  std::vector<double> c(static_cast<std::size_t>(m) * n, 0.0);
  for (int j = 0; j < n; ++j)
    for (int q = 0; q < k; ++q) {
      const double bv = b[q + static_cast<std::size_t>(j) * k];
      if (bv == 0.0) continue;
      for (int i = 0; i < m; ++i) c[i + static_cast<std::size_t>(j) * m] += a[i + static_cast<std::size_t>(q) * m] * bv;
    }
  return c;
}

}  // namespace hsg
