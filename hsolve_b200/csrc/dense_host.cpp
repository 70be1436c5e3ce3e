// Small dense linear algebra (see dense_host.hpp): the textbook Householder reduction to
// tridiagonal form and the implicit QL iteration with Wilkinson shifts, written for this project.
#include "dense_host.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
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


// ------------------------------------------------------------- general (non-symmetric) matrices
//
// Complex Schur form T = U^H A U of a real matrix, written for this project from the standard
// algorithm: Householder reduction to upper Hessenberg form, then the shifted QR iteration with
// Wilkinson shifts in complex arithmetic (Givens rotations, one shift per step; a 2 x 2 window is
// resolved the same way), deflation when a subdiagonal entry falls below eps times its neighbours.

namespace {

using cplx = std::complex<double>;

// rotation G = [c s; -conj(s) c] (c real) with G [x; y] = [r; 0]
void givens(cplx x, cplx y, double& c, cplx& s) {
  const double ax = std::abs(x), ay = std::abs(y);
  if (ay == 0.0) { c = 1.0; s = 0.0; return; }
  if (ax == 0.0) { c = 0.0; s = std::conj(y) / ay; return; }
  const double r = std::hypot(ax, ay);
  c = ax / r;
  s = (x / ax) * std::conj(y) / r;
}

}  // namespace

void complex_schur(int n, const std::vector<double>& a, std::vector<cplx>& T, std::vector<cplx>& U) {
  // Householder reduction to Hessenberg form (real), Q accumulated
  std::vector<double> h(a), q(static_cast<std::size_t>(n) * n, 0.0);
  auto H = [&](int i, int j) -> double& { return h[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * n]; };
  auto Q = [&](int i, int j) -> double& { return q[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * n]; };
  for (int i = 0; i < n; ++i) Q(i, i) = 1.0;
  std::vector<double> v(n);
  for (int k = 0; k + 2 < n; ++k) {
    double alpha = 0.0;
    for (int i = k + 1; i < n; ++i) alpha += H(i, k) * H(i, k);
    alpha = std::sqrt(alpha);
    if (alpha == 0.0) continue;
    const double x0 = H(k + 1, k);
    const double s = x0 >= 0 ? -alpha : alpha;
    for (int i = k + 1; i < n; ++i) v[i] = H(i, k);
    v[k + 1] = x0 - s;
    double vn = 0.0;
    for (int i = k + 1; i < n; ++i) vn += v[i] * v[i];
    if (vn == 0.0) continue;
    const double beta = 2.0 / vn;
    for (int j = 0; j < n; ++j) {  // H = (I - beta v v^T) H
      double t = 0.0;
      for (int i = k + 1; i < n; ++i) t += v[i] * H(i, j);
      t *= beta;
      for (int i = k + 1; i < n; ++i) H(i, j) -= t * v[i];
    }
    for (int i = 0; i < n; ++i) {  // H = H (I - beta v v^T), Q = Q (I - beta v v^T)
      double t = 0.0, u = 0.0;
      for (int j = k + 1; j < n; ++j) { t += H(i, j) * v[j]; u += Q(i, j) * v[j]; }
      t *= beta;
      u *= beta;
      for (int j = k + 1; j < n; ++j) { H(i, j) -= t * v[j]; Q(i, j) -= u * v[j]; }
    }
    for (int i = k + 2; i < n; ++i) H(i, k) = 0.0;
  }
  T.assign(h.begin(), h.end());
  U.assign(q.begin(), q.end());
  auto t = [&](int i, int j) -> cplx& { return T[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * n]; };
  auto u = [&](int i, int j) -> cplx& { return U[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * n]; };
  const double eps = std::numeric_limits<double>::epsilon();
  double anorm = 0.0;
  for (std::size_t e = 0; e < T.size(); ++e) anorm = std::max(anorm, std::abs(T[e]));
  int hi = n - 1, iter = 0, total = 0;
  while (hi > 0) {
    int l = hi;
    while (l > 0) {
      const double sub = std::abs(t(l, l - 1));
      const double nb = std::abs(t(l, l)) + std::abs(t(l - 1, l - 1));
      if (sub <= eps * (nb > 0.0 ? nb : anorm)) { t(l, l - 1) = 0.0; break; }
      --l;
    }
    if (l == hi) { --hi; iter = 0; continue; }
    if (++total > 100 * n) throw std::runtime_error("complex_schur: QR iteration did not converge");
    ++iter;
    // Wilkinson shift from the trailing 2 x 2 of the window (an exceptional shift now and then)
    const cplx a11 = t(hi - 1, hi - 1), a12 = t(hi - 1, hi), a21 = t(hi, hi - 1), a22 = t(hi, hi);
    cplx mu;
    if (iter % 11 == 10) {
      mu = a22 + cplx(std::abs(a21), 0.0) * 0.75;
    } else {
      const cplx half = 0.5 * (a11 - a22);
      const cplx disc = std::sqrt(half * half + a12 * a21);
      const cplx m1 = a22 + half + disc, m2 = a22 + half - disc;
      mu = std::abs(m1 - a22) <= std::abs(m2 - a22) ? m1 : m2;
    }
    cplx x = t(l, l) - mu, y = t(l + 1, l);
    for (int k = l; k < hi; ++k) {
      double c;
      cplx s;
      givens(x, y, c, s);
      // rows k, k+1 (columns from k-1, or l at the first step, to the right end)
      for (int j = (k > l ? k - 1 : l); j < n; ++j) {
        const cplx r0 = t(k, j), r1 = t(k + 1, j);
        t(k, j) = c * r0 + s * r1;
        t(k + 1, j) = -std::conj(s) * r0 + c * r1;
      }
      // columns k, k+1 (rows up to k+2) and the Schur vectors
      const int rmax = std::min(k + 2, hi);
      for (int i = 0; i <= rmax; ++i) {
        const cplx c0 = t(i, k), c1 = t(i, k + 1);
        t(i, k) = c * c0 + std::conj(s) * c1;
        t(i, k + 1) = -s * c0 + c * c1;
      }
      for (int i = 0; i < n; ++i) {
        const cplx c0 = u(i, k), c1 = u(i, k + 1);
        u(i, k) = c * c0 + std::conj(s) * c1;
        u(i, k + 1) = -s * c0 + c * c1;
      }
      if (k + 1 < hi) {
        x = t(k + 1, k);
        y = t(k + 2, k);
      }
    }
  }
  for (int j = 0; j < n; ++j)
    for (int i = j + 1; i < n; ++i) t(i, j) = 0.0;
}

void schur_sort(int n, std::vector<cplx>& T, std::vector<cplx>& U, const std::vector<double>& key) {
  auto t = [&](int i, int j) -> cplx& { return T[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * n]; };
  auto u = [&](int i, int j) -> cplx& { return U[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * n]; };
  // keys travel with the diagonal entries they were computed for
  std::vector<double> kk(key);
  for (int pos = 0; pos < n; ++pos) {
    int best = pos;
    for (int i = pos + 1; i < n; ++i)
      if (kk[i] < kk[best]) best = i;
    for (int k = best - 1; k >= pos; --k) {
      // swap diagonal entries k and k+1: G's first column is the eigenvector of the 2 x 2 block for
      // its second eigenvalue
      const cplx a = t(k, k), b = t(k, k + 1), d = t(k + 1, k + 1);
      cplx g1 = b, g2 = d - a;
      const double nr = std::hypot(std::abs(g1), std::abs(g2));
      if (nr == 0.0) { std::swap(kk[k], kk[k + 1]); continue; }
      g1 /= nr;
      g2 /= nr;
      // G = [g1 -conj(g2); g2 conj(g1)]; T = G^H T G, U = U G
      for (int j = k; j < n; ++j) {
        const cplx r0 = t(k, j), r1 = t(k + 1, j);
        t(k, j) = std::conj(g1) * r0 + std::conj(g2) * r1;
        t(k + 1, j) = -g2 * r0 + g1 * r1;
      }
      for (int i = 0; i <= k + 1; ++i) {
        const cplx c0 = t(i, k), c1 = t(i, k + 1);
        t(i, k) = c0 * g1 + c1 * g2;
        t(i, k + 1) = -c0 * std::conj(g2) + c1 * std::conj(g1);
      }
      for (int i = 0; i < n; ++i) {
        const cplx c0 = u(i, k), c1 = u(i, k + 1);
        u(i, k) = c0 * g1 + c1 * g2;
        u(i, k + 1) = -c0 * std::conj(g2) + c1 * std::conj(g1);
      }
      t(k + 1, k) = 0.0;
      std::swap(kk[k], kk[k + 1]);
    }
  }
}

std::vector<cplx> schur_eigenvectors(int n, const std::vector<cplx>& T, int count, double cluster_rtol) {
  auto t = [&](int i, int j) { return T[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * n]; };
  double tnorm = 0.0;
  for (const cplx& z : T) tnorm = std::max(tnorm, std::abs(z));
  const double smin = std::max(tnorm * std::numeric_limits<double>::epsilon(), 1e-300);
  std::vector<cplx> Y(static_cast<std::size_t>(n) * count, cplx(0.0));
  for (int k = 0; k < count; ++k) {
    const cplx lam = t(k, k);
    // the cluster of entries equal to lam just above k is treated as one block: its members' own
    // coordinates are set (unit vector), only the entries above the cluster are solved for
    int a = k;
    while (a > 0 && std::abs(t(a - 1, a - 1) - lam) <= cluster_rtol * std::max(std::abs(lam), smin)) --a;
    cplx* y = &Y[static_cast<std::size_t>(k) * n];
    y[k] = 1.0;
    for (int i = a - 1; i >= 0; --i) {
      cplx s = 0.0;
      for (int j = i + 1; j <= k; ++j) s += t(i, j) * y[j];
      cplx den = t(i, i) - lam;
      if (std::abs(den) < smin) den = smin;
      y[i] = -s / den;
    }
    double nr = 0.0;
    for (int i = 0; i <= k; ++i) nr += std::norm(y[i]);
    nr = std::sqrt(nr);
    for (int i = 0; i <= k; ++i) y[i] /= nr;
  }
  return Y;
}

std::vector<double> pivoted_basis(int m, int count, const std::vector<double>& pool, int want, double min_norm, int& r) {
  std::vector<double> q;
  r = 0;
  std::vector<double> v(m), best(m);
  for (; r < want; ++r) {
    double best_norm = -1.0;
    for (int j = 0; j < count; ++j) {
      std::copy(pool.begin() + static_cast<std::ptrdiff_t>(j) * m, pool.begin() + static_cast<std::ptrdiff_t>(j + 1) * m,
                v.begin());
      for (int pass = 0; pass < 2; ++pass)
        for (int t = 0; t < r; ++t) {
          const double* qt = &q[static_cast<std::size_t>(t) * m];
          double d = 0.0;
          for (int i = 0; i < m; ++i) d += qt[i] * v[i];
          for (int i = 0; i < m; ++i) v[i] -= d * qt[i];
        }
      double nr = 0.0;
      for (double x : v) nr += x * x;
      nr = std::sqrt(nr);
      if (nr > best_norm) {
        best_norm = nr;
        best = v;
      }
    }
    if (!(best_norm >= min_norm)) break;
    for (double& x : best) x /= best_norm;
    q.insert(q.end(), best.begin(), best.end());
  }
  return q;
}

}  // namespace hsg
