// Block Krylov-Schur (see eigen.hpp).
#include "eigen.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <limits>
#include <numeric>
#include <random>

#include "blas_kernels.cuh"
#include "dense_host.hpp"

namespace hsg {

namespace {

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

struct Basis {
  std::int64_t n;
  int cols;
  bool bid;
  DevBuf<double> V, BV, tmp, tmpB, g, part, small;
  std::int64_t part_cap = 0;
  double* v(int j) { return V.p + static_cast<std::int64_t>(j) * n; }
  double* bv(int j) { return bid ? v(j) : BV.p + static_cast<std::int64_t>(j) * n; }
};

void to_host(std::vector<double>& h, const double* d, std::size_t count, cudaStream_t s) {
  h.resize(count);
  cuda_check(cudaMemcpyAsync(h.data(), d, count * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H");
  cuda_check(cudaStreamSynchronize(s), "sync");
}

void to_dev(double* d, const std::vector<double>& h, cudaStream_t s) {
  cuda_check(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s), "H2D");
}

// Orthogonalize columns [j, j+p) of the basis against columns [0, j) (CGS2, B inner product),
// returning the accumulated coefficients H (j x p) on the host. Both passes' coefficients stay on the
// device (pass q's at q j p in B.g) and are read in one transfer at the end.
std::vector<double> orthogonalize(Basis& B, int j, int p, cudaStream_t s) {
  std::vector<double> Htot(static_cast<std::size_t>(j) * p, 0.0), H;
  if (j == 0) return Htot;
  const std::size_t jp = static_cast<std::size_t>(j) * p;
  for (int pass = 0; pass < 2; ++pass) {
    double* G = B.g.p + pass * jp;
    gram(B.n, j, p, B.bid ? B.v(0) : B.bv(0), B.n, B.v(j), B.n, G, B.part.p, B.part_cap, s);
    gemm_tall(B.n, j, p, B.v(0), B.n, G, j, B.v(j), B.n, -1.0, 1.0, s);
  }
  to_host(H, B.g.p, 2 * jp, s);
  for (std::size_t t = 0; t < jp; ++t) Htot[t] = H[t] + H[jp + t];
  return Htot;
}

// Thresholds of the block orthonormalization (the contract of hsolve's BlockOrthonormalizer,
// src/eigen/block_ortho.hpp:28-64, with this project's values): Cholesky-QR is trusted while the
// column-scaled condition number of the first pass's R stays below kMaxCholQrCond and the second
// pass's Gram matrix stays within kMaxSecondPassDeviation of I; a column whose B-norm falls to
// kDeficientRatio of its input norm is dependent on the basis to working precision.
constexpr double kMaxCholQrCond = 1e5;
constexpr double kMaxSecondPassDeviation = 0.5;
constexpr double kDeficientRatio = 1e-10;

// B-orthonormalize columns [j, j+p) in place (CholQR2) when the block is well conditioned:
// returns R (p x p, upper in the sense W_old = W_new R, column-major), or an empty vector with the
// block unchanged when the fast path must not be taken: a column of B-norm <= kDeficientRatio *
// before[c] (its norm before the projection on the basis), G not numerically positive definite,
// the scaled condition number of R1 above kMaxCholQrCond, or the second pass's G far from I.
// before[c] is computed here from hn2[c] (the squared projections of the input column on the basis)
// and the first pass's G: ||w_c||^2 = ||h_c||^2 + G_cc, the basis being B-orthonormal.
std::vector<double> normalize(Basis& B, KrylovOperator& op, int j, int p, const std::vector<double>& hn2,
                              std::vector<double>& before, cudaStream_t s) {
  std::vector<double> Rtot(static_cast<std::size_t>(p) * p, 0.0);
  for (int i = 0; i < p; ++i) Rtot[i + i * p] = 1.0;
  std::vector<double> G, L;
  for (int pass = 0; pass < 2; ++pass) {
    if (!B.bid) op.bprod(B.v(j), B.n, B.bv(j), B.n, p);
    gram(B.n, p, p, B.v(j), B.n, B.bv(j), B.n, B.g.p, B.part.p, B.part_cap, s);
    to_host(G, B.g.p, static_cast<std::size_t>(p) * p, s);
    for (int a = 0; a < p; ++a)
      for (int b = 0; b < a; ++b) { const double m = 0.5 * (G[a + b * p] + G[b + a * p]); G[a + b * p] = m; G[b + a * p] = m; }
    bool ok = true;
    if (pass == 0) {
      before.resize(p);
      for (int a = 0; a < p; ++a) before[a] = std::sqrt(std::max(0.0, hn2[a] + G[a + a * p]));
      // every column keeps more than its deficiency share, and the column-scaled G is well enough
      // conditioned for Cholesky-QR: cond(R1) = sqrt(cond(D^-1/2 G D^-1/2))
      std::vector<double> Gs(G);
      for (int a = 0; a < p && ok; ++a) ok = G[a + a * p] > kDeficientRatio * kDeficientRatio * before[a] * before[a];
      if (ok) {
        for (int a = 0; a < p; ++a)
          for (int b = 0; b < p; ++b) Gs[a + b * p] = G[a + b * p] / std::sqrt(G[a + a * p] * G[b + b * p]);
        std::vector<double> w;
        sym_eig(p, Gs, w);
        ok = w[0] > 0.0 && w[p - 1] <= kMaxCholQrCond * kMaxCholQrCond * w[0];
      }
    } else {
      double dev = 0.0;
      for (int a = 0; a < p; ++a)
        for (int b = 0; b < p; ++b) dev += (G[a + b * p] - (a == b ? 1.0 : 0.0)) * (G[a + b * p] - (a == b ? 1.0 : 0.0));
      ok = std::sqrt(dev) <= kMaxSecondPassDeviation;
    }
    ok = ok && cholesky(p, G, L, 1e-28);
    if (!ok) {
      if (pass == 1) {
        // undo the first pass (W = Q1 R1), so the caller's column path starts from the block
        std::vector<double> Rt(Rtot);
        to_dev(B.small.p, Rt, s);
        gemm_tall(B.n, p, p, B.v(j), B.n, B.small.p, p, B.tmp.p, B.n, 1.0, 0.0, s);
        copy_cols(B.n, p, B.tmp.p, B.n, B.v(j), B.n, s);
      }
      return {};
    }
    // W = W L^{-T}  (W^T B W = L L^T -> (W L^{-T})^T B (W L^{-T}) = I)
    std::vector<double> Linv = lower_inverse(p, L);
    std::vector<double> LinvT(static_cast<std::size_t>(p) * p);
    for (int a = 0; a < p; ++a)
      for (int b = 0; b < p; ++b) LinvT[a + b * p] = Linv[b + a * p];
    to_dev(B.small.p, LinvT, s);
    gemm_tall(B.n, p, p, B.v(j), B.n, B.small.p, p, B.tmp.p, B.n, 1.0, 0.0, s);
    copy_cols(B.n, p, B.tmp.p, B.n, B.v(j), B.n, s);
    if (!B.bid) {
      gemm_tall(B.n, p, p, B.bv(j), B.n, B.small.p, p, B.tmp.p, B.n, 1.0, 0.0, s);
      copy_cols(B.n, p, B.tmp.p, B.n, B.bv(j), B.n, s);
    }
    // R_total = L^T R_total
    std::vector<double> LT(static_cast<std::size_t>(p) * p);
    for (int a = 0; a < p; ++a)
      for (int b = 0; b < p; ++b) LT[a + b * p] = L[b + a * p];
    Rtot = matmul(p, p, p, LT, Rtot);
  }
  for (int i = 0; i < p; ++i)
    if (!(std::fabs(Rtot[i + i * p]) > kDeficientRatio * before[i])) {
      // a column left with no more than its deficiency share after both passes: the column path
      std::vector<double> Rt(Rtot);
      to_dev(B.small.p, Rt, s);
      gemm_tall(B.n, p, p, B.v(j), B.n, B.small.p, p, B.tmp.p, B.n, 1.0, 0.0, s);
      copy_cols(B.n, p, B.tmp.p, B.n, B.v(j), B.n, s);
      return {};
    }
  return Rtot;
}

void random_block(Basis& B, int j, int p, std::mt19937_64& rng, cudaStream_t s) {
  fill_normal(B.n, p, B.v(j), B.n, rng(), s);
}

// B-norm of column c of the basis (after refreshing B v(c) when B is not the identity).
double column_norm(Basis& B, KrylovOperator& op, int c, cudaStream_t s) {
  if (!B.bid) op.bprod(B.v(c), B.n, B.bv(c), B.n, 1);
  gram(B.n, 1, 1, B.v(c), B.n, B.bv(c), B.n, B.g.p, B.part.p, B.part_cap, s);
  std::vector<double> g;
  to_host(g, B.g.p, 1, s);
  return std::sqrt(std::max(g[0], 0.0));
}

// Column c projected twice (CGS2) against columns [0, c) in the B inner product; returns the
// accumulated coefficients (c of them).
std::vector<double> project_column(Basis& B, int c, cudaStream_t s) {
  std::vector<double> tot(c, 0.0), g;
  if (c == 0) return tot;
  for (int pass = 0; pass < 2; ++pass) {
    gram(B.n, c, 1, B.bid ? B.v(0) : B.bv(0), B.n, B.v(c), B.n, B.g.p, B.part.p, B.part_cap, s);
    gemm_tall(B.n, c, 1, B.v(0), B.n, B.g.p, c, B.v(c), B.n, -1.0, 1.0, s);
    to_host(g, B.g.p, static_cast<std::size_t>(c), s);
    for (int t = 0; t < c; ++t) tot[t] += g[t];
  }
  return tot;
}

// Column-by-column fallback (hsolve's column_fallback, src/eigen/block_ortho.cpp:340): each column
// of the block is projected by CGS2 against the basis and the block's earlier columns; a column
// whose B-norm falls to kDeficientRatio of its input norm is dependent on the basis (a block
// breakdown), gets R(c, c) = 0 and is replaced by a random vector projected the same way; where no
// direction is left (the basis spans the space), the column stays zero with zero coupling.
std::vector<double> column_fallback(Basis& B, KrylovOperator& op, int j, int p, std::vector<double>& H,
                                    const std::vector<double>& before, std::mt19937_64& rng, cudaStream_t s) {
  std::vector<double> R(static_cast<std::size_t>(p) * p, 0.0);
  for (int c = 0; c < p; ++c) {
    const int col = j + c;
    std::vector<double> g = project_column(B, col, s);
    for (int t = 0; t < j; ++t) H[t + static_cast<std::size_t>(c) * j] += g[t];
    for (int t = j; t < col; ++t) R[(t - j) + static_cast<std::size_t>(c) * p] = g[t];
    double nrm = column_norm(B, op, col, s);
    if (nrm > kDeficientRatio * before[c]) {
      R[c + static_cast<std::size_t>(c) * p] = nrm;
    } else {
      nrm = 0.0;
      for (int attempt = 0; attempt < 3 && !(nrm > 0.0); ++attempt) {
        random_block(B, col, 1, rng, s);
        const double r0 = column_norm(B, op, col, s);
        project_column(B, col, s);
        nrm = column_norm(B, op, col, s);
        if (!(nrm > 1e-8 * r0)) nrm = 0.0;  // the random vector lies in the basis' span as well
      }
    }
    if (nrm > 0.0) {
      scale_cols(B.n, 1, 1.0 / nrm, B.v(col), B.n, s);
      if (!B.bid) scale_cols(B.n, 1, 1.0 / nrm, B.bv(col), B.n, s);
    } else {
      scale_cols(B.n, 1, 0.0, B.v(col), B.n, s);
      if (!B.bid) scale_cols(B.n, 1, 0.0, B.bv(col), B.n, s);
    }
  }
  return R;
}

// New block [j, j+p) made orthonormal to [0, j): returns R (the coupling W_old = W_new R, zero in
// the columns that had to be replaced) and the projections H (j x p) on the basis.
std::vector<double> ortho_block(Basis& B, KrylovOperator& op, int j, int p, std::vector<double>& H, std::mt19937_64& rng,
                                cudaStream_t s) {
  H = orthogonalize(B, j, p, s);
  std::vector<double> hn2(p, 0.0), before;
  for (int c = 0; c < p; ++c)
    for (int t = 0; t < j; ++t) hn2[c] += H[t + static_cast<std::size_t>(c) * j] * H[t + static_cast<std::size_t>(c) * j];
  std::vector<double> R = normalize(B, op, j, p, hn2, before, s);
  if (!R.empty()) return R;
  return column_fallback(B, op, j, p, H, before, rng, s);
}

}  // namespace

KsResult krylov_schur(KrylovOperator& op, std::int64_t n, const KsOptions& opt, cudaStream_t s) {
  const int p = std::max(1, std::min(opt.block, kMaxKrylovBlock));
  const int nev = std::max(1, opt.nev);
  int mmax = opt.ncv > 0 ? opt.ncv : std::max(2 * nev + 1, nev + 16) + 4 * p;
  mmax = std::max(mmax, nev + 2 * p);
  mmax = (mmax + p - 1) / p * p;
  if (mmax > n) mmax = static_cast<int>(n / p * p);
  HSG_REQUIRE(mmax >= p && nev <= mmax - p + p, HSG_INVALID_INPUT, "Krylov basis larger than the problem (n = " << n << ")");
  Basis B;
  B.n = n;
  B.bid = op.b_identity();
  B.cols = mmax + p;
  B.V.alloc(static_cast<std::size_t>(n) * B.cols);
  if (!B.bid) B.BV.alloc(static_cast<std::size_t>(n) * B.cols);
  B.tmp.alloc(static_cast<std::size_t>(n) * std::max(p, mmax));
  if (!B.bid) B.tmpB.alloc(static_cast<std::size_t>(n) * mmax);
  B.g.alloc(static_cast<std::size_t>(B.cols) * std::max(p, mmax));
  B.part_cap = gram_part_size(n, B.cols, p);
  B.part.alloc(static_cast<std::size_t>(B.part_cap));
  B.small.alloc(static_cast<std::size_t>(std::max(p * p, mmax * mmax)));
  std::mt19937_64 rng(opt.seed);
  KsResult res;
  // starting block
  random_block(B, 0, p, rng, s);
  {
    std::vector<double> H;
    std::vector<double> R = ortho_block(B, op, 0, p, H, rng, s);
    (void)R;
  }
  const int tdim = mmax + p;
  std::vector<double> T(static_cast<std::size_t>(tdim) * tdim, 0.0);
  auto Tm = [&](int i, int j) -> double& { return T[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * tdim]; };
  int m = 0;
  std::vector<double> S, w;
  std::vector<int> order;
  while (true) {
    while (m + p <= mmax) {
      const int j0 = m;
      auto tp = std::chrono::steady_clock::now();
      op.apply(B.v(j0), n, B.v(j0 + p), n, p);
      res.t_apply += seconds_since(tp);
      res.applies += p;
      res.block_steps += 1;
      std::vector<double> H;
      tp = std::chrono::steady_clock::now();
      std::vector<double> R = ortho_block(B, op, j0 + p, p, H, rng, s);
      res.t_ortho += seconds_since(tp);
      const int jh = j0 + p;  // H is jh x p
      for (int c = 0; c < p; ++c)
        for (int i = 0; i < jh; ++i) {
          Tm(i, j0 + c) = H[i + static_cast<std::size_t>(c) * jh];
          Tm(j0 + c, i) = H[i + static_cast<std::size_t>(c) * jh];
        }
      for (int a = 0; a < p; ++a)
        for (int b = 0; b < a; ++b) {
          const double mm = 0.5 * (Tm(j0 + a, j0 + b) + Tm(j0 + b, j0 + a));
          Tm(j0 + a, j0 + b) = mm;
          Tm(j0 + b, j0 + a) = mm;
        }
      for (int c = 0; c < p; ++c)
        for (int a = 0; a < p; ++a) {
          Tm(jh + a, j0 + c) = R[a + c * p];
          Tm(j0 + c, jh + a) = R[a + c * p];
        }
      m += p;
    }
    // Rayleigh-Ritz on T[0:m, 0:m]
    const auto trr = std::chrono::steady_clock::now();
    S.assign(static_cast<std::size_t>(m) * m, 0.0);
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) S[i + static_cast<std::size_t>(j) * m] = Tm(i, j);
    sym_eig(m, S, w);
    order.resize(m);
    std::iota(order.begin(), order.end(), 0);
    auto key = [&](int i) {
      switch (opt.which) {
        case Which::LargestMagnitude: return -std::fabs(w[i]);
        case Which::LargestAlgebraic: return -w[i];
        default: return w[i];
      }
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key(a) < key(b); });
    // residual norms ||T[m:m+p, 0:m] s_i||
    std::vector<double> rn(m, 0.0);
    for (int i = 0; i < m; ++i) {
      double acc = 0.0;
      for (int a = 0; a < p; ++a) {
        double t = 0.0;
        for (int q = 0; q < m; ++q) t += Tm(m + a, q) * S[q + static_cast<std::size_t>(i) * m];
        acc += t * t;
      }
      rn[i] = std::sqrt(acc);
    }
    // equal Ritz values (a multiple eigenvalue, possibly with more copies in the basis than the
    // wanted set takes) are ranked by residual, so the wanted set and the kept basis take the
    // converged copies first instead of an arbitrary subset of the cluster
    for (int q0 = 0; q0 < m;) {
      int q1 = q0 + 1;
      const double ref = std::fabs(w[order[q0]]);
      while (q1 < m && std::fabs(w[order[q1]] - w[order[q0]]) <= 1e-12 * ref) ++q1;
      if (q1 - q0 > 1)
        std::stable_sort(order.begin() + q0, order.begin() + q1, [&](int a, int b) { return rn[a] < rn[b]; });
      q0 = q1;
    }
    const int strict = opt.nev_strict > 0 ? std::min(opt.nev_strict, nev) : nev;
    auto tol_at = [&](int q) { return q < strict ? opt.tol : std::max(opt.tol, opt.tol_buffer); };
    int nconv = 0;
    for (int q = 0; q < nev && q < m; ++q) {
      const int i = order[q];
      if (rn[i] <= tol_at(q) * std::fabs(w[i])) ++nconv;
    }
    res.t_rr += seconds_since(trr);
    const bool done = nconv >= std::min(nev, m) || res.restarts >= opt.max_restarts;
    if (done) {
      const int take = std::min(nev, m);
      res.theta.resize(take);
      res.resid.resize(take);
      res.converged.resize(take);
      std::vector<double> Q(static_cast<std::size_t>(m) * take);
      for (int q = 0; q < take; ++q) {
        const int i = order[q];
        res.theta[q] = w[i];
        res.resid[q] = rn[i];
        res.converged[q] = rn[i] <= tol_at(q) * std::fabs(w[i]);
        std::copy(S.begin() + static_cast<std::ptrdiff_t>(i) * m, S.begin() + static_cast<std::ptrdiff_t>(i + 1) * m,
                  Q.begin() + static_cast<std::ptrdiff_t>(q) * m);
      }
      res.nconv = nconv;
      for (int q = take; q < m; ++q) {
        res.other_theta.push_back(w[order[q]]);
        res.other_resid.push_back(rn[order[q]]);
      }
      if (opt.ritz_vectors) {
        res.X.alloc(static_cast<std::size_t>(n) * take);
        B.small.alloc(Q.size());
        to_dev(B.small.p, Q, s);
        gemm_tall(n, m, take, B.v(0), n, B.small.p, m, res.X.p, n, 1.0, 0.0, s);
        cuda_check(cudaStreamSynchronize(s), "ritz vectors");
      }
      return res;
    }
    // thick restart
    const auto trs = std::chrono::steady_clock::now();
    const int keep = std::min(mmax - p, std::max(nev + p, (nev + mmax) / 2));
    std::vector<double> Q(static_cast<std::size_t>(m) * keep);
    std::vector<double> th(keep);
    for (int q = 0; q < keep; ++q) {
      const int i = order[q];
      th[q] = w[i];
      std::copy(S.begin() + static_cast<std::ptrdiff_t>(i) * m, S.begin() + static_cast<std::ptrdiff_t>(i + 1) * m,
                Q.begin() + static_cast<std::ptrdiff_t>(q) * m);
    }
    B.small.alloc(Q.size());
    to_dev(B.small.p, Q, s);
    gemm_tall(n, m, keep, B.v(0), n, B.small.p, m, B.tmp.p, n, 1.0, 0.0, s);
    if (!B.bid) gemm_tall(n, m, keep, B.bv(0), n, B.small.p, m, B.tmpB.p, n, 1.0, 0.0, s);
    // residual block to [keep, keep+p), then the kept vectors to [0, keep)
    copy_cols(n, p, B.v(m), n, B.v(keep), n, s);
    copy_cols(n, keep, B.tmp.p, n, B.v(0), n, s);
    if (!B.bid) {
      copy_cols(n, p, B.bv(m), n, B.bv(keep), n, s);
      copy_cols(n, keep, B.tmpB.p, n, B.bv(0), n, s);
    }
    // coupling b = T[m:m+p, 0:m] Q
    std::vector<double> Tn(static_cast<std::size_t>(tdim) * tdim, 0.0);
    auto Tnm = [&](int i, int j) -> double& { return Tn[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * tdim]; };
    for (int q = 0; q < keep; ++q) Tnm(q, q) = th[q];
    for (int a = 0; a < p; ++a)
      for (int q = 0; q < keep; ++q) {
        double t = 0.0;
        for (int r = 0; r < m; ++r) t += Tm(m + a, r) * Q[r + static_cast<std::size_t>(q) * m];
        Tnm(keep + a, q) = t;
        Tnm(q, keep + a) = t;
      }
    // locking: a kept pair whose coupling column to the residual block is at rounding level
    // relative to every wanted Ritz value (|b(:, q)| <= 4 eps min |theta_wanted|) is decoupled, so
    // later cycles leave it converged (the reference's rule, src/eigen/block_lanczos.cpp:65)
    {
      double min_wanted = std::numeric_limits<double>::infinity();
      for (int q = 0; q < std::min(nev, m); ++q) min_wanted = std::min(min_wanted, std::fabs(w[order[q]]));
      const double lock_tol = 4.0 * std::numeric_limits<double>::epsilon() * min_wanted;
      for (int q = 0; q < keep; ++q) {
        double c2 = 0.0;
        for (int a = 0; a < p; ++a) c2 += Tnm(keep + a, q) * Tnm(keep + a, q);
        if (std::sqrt(c2) <= lock_tol) {
          for (int a = 0; a < p; ++a) { Tnm(keep + a, q) = 0.0; Tnm(q, keep + a) = 0.0; }
          ++res.locked;
        }
      }
    }
    T.swap(Tn);
    m = keep;
    res.restarts += 1;
    cuda_check(cudaStreamSynchronize(s), "restart");
    res.t_restart += seconds_since(trs);
  }
}

double exclusion_failure_bound(double eps, std::int64_t s, std::int64_t N, std::int64_t p, double kappa,
                               bool complex_scalars) {
  HSG_REQUIRE(s >= 1, HSG_INVALID_INPUT, "exclusion bound: block steps must be >= 1");
  HSG_REQUIRE(p >= 1, HSG_INVALID_INPUT, "exclusion bound: block size must be >= 1");
  HSG_REQUIRE(kappa >= 1.0, HSG_INVALID_INPUT, "exclusion bound: kappa must be >= 1");
  if (N <= 0) return 0.0;
  if (!(eps > 0.0)) return 1.0;
  const double e = std::min(eps, 1.0);
  const double inf = std::numeric_limits<double>::infinity();
  auto cheb = [&](double steps, double x) {  // T_k(x) = cosh(k acosh x), x >= 1
    const double a = steps * std::acosh(x);
    return a < 700.0 ? std::cosh(a) : inf;
  };
  // direct bound: T_{s-1} mapped from [-Theta, (1 - eps) Theta] to [-1, 1]
  const double c1 = cheb(static_cast<double>(s - 1), (2.0 + e) / (2.0 - e));
  double t = (2.0 - e) / (e * c1 * c1 + 2.0 - e);
  if (s >= 2) {
    // squared bound: T_k in theta^2 on [0, (1 - eps)^2 Theta^2], k = floor((s - 2) / 2)
    const double q = (1.0 - e) * (1.0 - e), e2 = 1.0 - q;
    const std::int64_t k = (s - 2) / 2;
    const double c2 = k == 0 ? 1.0 : (q > 0.0 ? cheb(static_cast<double>(k), (1.0 + e2) / (1.0 - e2)) : inf);
    t = std::min(t, q / (e2 * c2 * c2 + q));
  }
  // the first coordinate of a uniform unit vector: real P(z^2 < x) <= sqrt(N x), complex <= (N-1) x
  const double f = complex_scalars ? static_cast<double>(N - 1) * kappa * t
                                   : std::sqrt(static_cast<double>(N) * kappa * t);
  return std::pow(std::min(f, 1.0), static_cast<double>(p));
}

std::int64_t exclusion_block_steps(double eps, double delta, std::int64_t N, std::int64_t p, double kappa,
                                   bool complex_scalars) {
  if (!(eps > 0.0) || !(delta > 0.0 && delta < 1.0)) return -1;
  HSG_REQUIRE(p >= 1, HSG_INVALID_INPUT, "exclusion steps: block size must be >= 1");
  if (N <= 0) return 1;
  const std::int64_t cover = (N + p - 1) / p + 1;
  auto ok = [&](std::int64_t st) { return exclusion_failure_bound(eps, st, N, p, kappa, complex_scalars) <= delta; };
  if (ok(1)) return 1;
  std::int64_t hi = 1;
  while (!ok(hi)) {  // doubling, then bisection on the monotone bound
    if (hi >= cover) return cover;
    hi *= 2;
  }
  std::int64_t lo = hi / 2;
  while (hi - lo > 1) {
    const std::int64_t mid = lo + (hi - lo) / 2;
    if (ok(mid)) hi = mid;
    else lo = mid;
  }
  return std::min(hi, cover);
}

namespace {

void alloc_basis(Basis& B, std::int64_t n, bool bid, int cols, int pmax) {
  B.n = n;
  B.bid = bid;
  B.cols = cols;
  B.V.alloc(static_cast<std::size_t>(n) * cols);
  if (!bid) B.BV.alloc(static_cast<std::size_t>(n) * cols);
  B.tmp.alloc(static_cast<std::size_t>(n) * pmax);
  B.g.alloc(static_cast<std::size_t>(2) * cols * pmax);
  B.part_cap = gram_part_size(n, cols, pmax);
  B.part.alloc(static_cast<std::size_t>(B.part_cap));
  B.small.alloc(static_cast<std::size_t>(pmax) * pmax);
}

// largest eigenvalue of the symmetric part of a k x k matrix (host)
double sym_max_eig(int k, std::vector<double> G) {
  for (int a = 0; a < k; ++a)
    for (int b = 0; b < a; ++b) { const double v = 0.5 * (G[a + b * k] + G[b + a * k]); G[a + b * k] = v; G[b + a * k] = v; }
  std::vector<double> w;
  sym_eig(k, G, w);
  return w.empty() ? 0.0 : w.back();
}

}  // namespace

ExclusionResult exclusion_check(KrylovOperator& op, std::int64_t n, const double* x, int m,
                                const ExclusionOptions& opt, const double* start_scale, cudaStream_t s) {
  HSG_REQUIRE(m >= 1 && m < n, HSG_INVALID_INPUT, "exclusion check: need 1 <= found vectors < n");
  HSG_REQUIRE(opt.radius > 0.0 && opt.pass_radius > opt.radius, HSG_INVALID_INPUT,
              "exclusion check: need 0 < radius < pass_radius");
  HSG_REQUIRE(opt.delta > 0.0 && opt.delta < 1.0, HSG_INVALID_INPUT, "exclusion check: delta must lie in (0, 1)");
  HSG_REQUIRE(opt.kappa >= 1.0, HSG_INVALID_INPUT, "exclusion check: kappa must be >= 1");
  HSG_REQUIRE(opt.rounding_margin >= 0.0 && opt.rounding_margin < 0.5, HSG_INVALID_INPUT,
              "exclusion check: rounding margin must lie in [0, 0.5)");
  ExclusionResult res;
  const int p = std::max(1, std::min(opt.block, kMaxKrylovBlock));
  res.block = p;
  res.kappa = opt.kappa;
  res.deflated = m;
  res.dimension = n - m;
  const std::int64_t N = n - m;
  const bool bid = op.b_identity();
  std::mt19937_64 rng(opt.seed);
  auto t0 = std::chrono::steady_clock::now();
  // ---- X made B-orthonormal, and the coupling e = ||OP X - X H11||_B with H11 = X^T B OP X
  Basis X1;
  alloc_basis(X1, n, bid, 2 * m, m);
  copy_cols(n, m, x, n, X1.v(0), n, s);
  {
    std::vector<double> H;
    ortho_block(X1, op, 0, m, H, rng, s);
  }
  op.apply(X1.v(0), n, X1.v(m), n, m);
  res.op_applications += m;
  std::vector<double> H11, G;
  gram(n, m, m, bid ? X1.v(0) : X1.bv(0), n, X1.v(m), n, X1.g.p, X1.part.p, X1.part_cap, s);
  to_host(H11, X1.g.p, static_cast<std::size_t>(m) * m, s);
  gemm_tall(n, m, m, X1.v(0), n, X1.g.p, m, X1.v(m), n, -1.0, 1.0, s);
  if (!bid) op.bprod(X1.v(m), n, X1.bv(m), n, m);
  gram(n, m, m, X1.v(m), n, bid ? X1.v(m) : X1.bv(m), n, X1.g.p, X1.part.p, X1.part_cap, s);
  to_host(G, X1.g.p, static_cast<std::size_t>(m) * m, s);
  {
    std::vector<double> Hs(H11), mu;
    for (int a = 0; a < m; ++a)
      for (int b = 0; b < a; ++b) { const double v = 0.5 * (Hs[a + b * m] + Hs[b + a * m]); Hs[a + b * m] = v; Hs[b + a * m] = v; }
    sym_eig(m, Hs, mu);
    std::sort(mu.begin(), mu.end(), [](double a, double b) { return std::fabs(a) > std::fabs(b); });
    res.deflated_theta = mu;
  }
  const double mu_max = res.deflated_theta.empty() ? 0.0 : std::fabs(res.deflated_theta.front());
  // the B-norm of the residual block, with a guard for the rounding of H11 and of the Gram matrix
  res.coupling = std::sqrt(std::max(0.0, sym_max_eig(m, G))) + 64.0 * std::numeric_limits<double>::epsilon() * mu_max;
  const double e = res.coupling;
  const double theta_c = 1.0 / opt.radius - e;
  res.claim_threshold = theta_c * (1.0 - opt.rounding_margin);
  res.pass_threshold = 1.0 / opt.pass_radius;
  res.epsilon = res.claim_threshold > 0.0 ? 1.0 - res.pass_threshold / res.claim_threshold : 0.0;
  for (double mv : res.deflated_theta) {
    if (std::fabs(mv) >= theta_c) ++res.found_inside;
    if (std::fabs(mv) >= 1.0 / opt.radius + e) ++res.certified_inside;
  }
  res.setup_s = seconds_since(t0);
  if (!(res.epsilon > 0.0)) return res;  // no statement: the gap is too small for the coupling
  // ---- the plan: s block steps fixed before the run
  std::int64_t steps = exclusion_block_steps(res.epsilon, opt.delta, N, p, opt.kappa, false);
  if (steps < 1) return res;
  res.block_steps_planned = static_cast<int>(std::min<std::int64_t>(steps, 1 << 30));
  bool capped = false;
  if (opt.max_block_steps > 0 && steps > opt.max_block_steps) { steps = opt.max_block_steps; capped = true; }
  res.exact = steps * p >= N;
  const std::int64_t vectors = res.exact ? N : steps * p;
  res.krylov_vectors_planned = static_cast<int>(std::min<std::int64_t>(vectors, 1 << 30));
  if (opt.max_krylov_vectors > 0 && vectors > opt.max_krylov_vectors) {
    res.over_budget = true;
    return res;
  }
  if (res.exact) steps = (N + p - 1) / p;
  const int S = static_cast<int>(steps);
  // ---- block Lanczos on the complement of span X, full CGS2 re-orthogonalization against [X V]
  t0 = std::chrono::steady_clock::now();
  Basis B;
  alloc_basis(B, n, bid, m + (S + 1) * p, std::max(m, p));
  copy_cols(n, m, X1.v(0), n, B.v(0), n, s);
  if (!bid) copy_cols(n, m, X1.bv(0), n, B.bv(0), n, s);
  random_block(B, m, p, rng, s);
  if (start_scale) diag_scale(n, p, start_scale, B.v(m), n, B.v(m), n, s);
  {
    std::vector<double> H;
    ortho_block(B, op, m, p, H, rng, s);
  }
  const int k = S * p;
  std::vector<double> T(static_cast<std::size_t>(k) * k, 0.0);
  for (int st = 0; st < S; ++st) {
    const int j = m + (st + 1) * p;
    op.apply(B.v(j - p), n, B.v(j), n, p);
    res.op_applications += p;
    std::vector<double> H;
    std::vector<double> R = ortho_block(B, op, j, p, H, rng, s);
    const int rows = (st + 1) * p;  // the rows of H on V_0 .. V_st (below the m rows of X)
    for (int c = 0; c < p; ++c) {
      for (int t = 0; t < rows; ++t) T[t + static_cast<std::size_t>(st * p + c) * k] = H[(m + t) + static_cast<std::size_t>(c) * j];
      if (st + 1 < S)
        for (int a = 0; a < p; ++a) T[(rows + a) + static_cast<std::size_t>(st * p + c) * k] = R[a + static_cast<std::size_t>(c) * p];
    }
    res.block_steps = st + 1;
  }
  for (int a = 0; a < k; ++a)
    for (int b = 0; b < a; ++b) { const double v = 0.5 * (T[a + static_cast<std::size_t>(b) * k] + T[b + static_cast<std::size_t>(a) * k]); T[a + static_cast<std::size_t>(b) * k] = v; T[b + static_cast<std::size_t>(a) * k] = v; }
  sym_eig(k, T, res.ritz);
  for (double th : res.ritz) {
    res.max_ritz = std::max(res.max_ritz, std::fabs(th));
    if (std::fabs(th) >= res.pass_threshold) ++res.new_count;
    if (std::fabs(th) >= 1.0 / opt.radius) ++res.new_inside;
  }
  res.krylov_s = seconds_since(t0);
  res.failure_probability = res.exact ? 0.0 : exclusion_failure_bound(res.epsilon, S, N, p, opt.kappa, false);
  if (res.max_ritz >= res.pass_threshold) res.status = ExclusionStatus::Detected;
  else if (!capped || res.failure_probability <= opt.delta) res.status = ExclusionStatus::Passed;
  return res;
}

}  // namespace hsg

namespace hsg {

GeneralKsResult krylov_schur_general(KrylovOperator& op, std::int64_t n, const KsOptions& opt, cudaStream_t s) {
  using cplx = std::complex<double>;
  const int p = std::max(1, std::min(opt.block, kMaxKrylovBlock));
  const int nev = std::max(1, opt.nev);
  int mmax = opt.ncv > 0 ? opt.ncv : std::max(2 * nev + 1, nev + 16) + 4 * p;
  mmax = std::max(mmax, nev + 2 * p + 2);
  mmax = (mmax + p - 1) / p * p;
  if (mmax > n) mmax = static_cast<int>(n / p * p);
  HSG_REQUIRE(mmax >= p + 1 && nev < mmax, HSG_INVALID_INPUT, "Krylov basis larger than the problem (n = " << n << ")");
  Basis B;
  B.n = n;
  B.bid = true;  // Euclidean inner product: B is indefinite, no inner product comes from it
  B.cols = mmax + p;
  B.V.alloc(static_cast<std::size_t>(n) * B.cols);
  B.tmp.alloc(static_cast<std::size_t>(n) * std::max(p, mmax));
  B.g.alloc(static_cast<std::size_t>(B.cols) * std::max(p, mmax));
  B.part_cap = gram_part_size(n, B.cols, p);
  B.part.alloc(static_cast<std::size_t>(B.part_cap));
  B.small.alloc(static_cast<std::size_t>(std::max(p * p, mmax * mmax)));
  std::mt19937_64 rng(opt.seed);
  GeneralKsResult res;
  random_block(B, 0, p, rng, s);
  {
    std::vector<double> H;
    ortho_block(B, op, 0, p, H, rng, s);
  }
  const int hd = mmax + p;
  std::vector<double> Hm(static_cast<std::size_t>(hd) * hd, 0.0);
  auto Hij = [&](int i, int j) -> double& { return Hm[static_cast<std::size_t>(i) + static_cast<std::size_t>(j) * hd]; };
  int m = 0;
  const int strict = opt.nev_strict > 0 ? std::min(opt.nev_strict, nev) : nev;
  while (true) {
    while (m + p <= mmax) {
      const int j0 = m;
      auto tp = std::chrono::steady_clock::now();
      op.apply(B.v(j0), n, B.v(j0 + p), n, p);
      res.t_apply += seconds_since(tp);
      res.applies += p;
      std::vector<double> H;
      tp = std::chrono::steady_clock::now();
      std::vector<double> R = ortho_block(B, op, j0 + p, p, H, rng, s);
      res.t_ortho += seconds_since(tp);
      const int jh = j0 + p;
      for (int c = 0; c < p; ++c) {
        for (int i = 0; i < jh; ++i) Hij(i, j0 + c) = H[i + static_cast<std::size_t>(c) * jh];
        for (int a = 0; a < p; ++a) Hij(jh + a, j0 + c) = R[a + c * p];
      }
      m += p;
    }
    // Rayleigh-Ritz: complex Schur form of G = H[0:m, 0:m], wanted values (largest |theta|) first
    const auto trr = std::chrono::steady_clock::now();
    std::vector<double> G(static_cast<std::size_t>(m) * m);
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) G[i + static_cast<std::size_t>(j) * m] = Hij(i, j);
    std::vector<cplx> T, U;
    complex_schur(m, G, T, U);
    std::vector<double> key(m);
    for (int i = 0; i < m; ++i) key[i] = -std::abs(T[static_cast<std::size_t>(i) * (m + 1)]);
    schur_sort(m, T, U, key);
    auto diag = [&](int i) { return T[static_cast<std::size_t>(i) * (m + 1)]; };
    // a set closed under conjugation: a complex value at its end takes its partner along
    auto closed = [&](int w) {
      if (w > 0 && w < m && std::abs(diag(w - 1).imag()) > 1e-12 * std::abs(diag(w - 1)) &&
          std::abs(diag(w) - std::conj(diag(w - 1))) <= 1e-8 * std::abs(diag(w - 1)))
        ++w;
      return w;
    };
    const int want = closed(std::min(nev, m));
    const std::vector<cplx> Y = schur_eigenvectors(m, T, want, 1e-8);
    std::vector<cplx> C(static_cast<std::size_t>(m) * want, cplx(0.0));  // U Y
    for (int k = 0; k < want; ++k)
      for (int t = 0; t < m; ++t) {
        const cplx y = Y[static_cast<std::size_t>(k) * m + t];
        if (y == cplx(0.0)) continue;
        for (int i = 0; i < m; ++i) C[static_cast<std::size_t>(k) * m + i] += U[static_cast<std::size_t>(t) * m + i] * y;
      }
    std::vector<double> rn(want);
    int nconv = 0, nstrict = 0;
    for (int k = 0; k < want; ++k) {
      double acc = 0.0;
      for (int a = 0; a < p; ++a) {
        cplx v = 0.0;
        for (int i = 0; i < m; ++i) v += Hij(m + a, i) * C[static_cast<std::size_t>(k) * m + i];
        acc += std::norm(v);
      }
      rn[k] = std::sqrt(acc);
      const double tl = k < strict ? opt.tol : std::max(opt.tol, opt.tol_buffer);
      if (rn[k] <= tl * std::abs(diag(k))) {
        ++nconv;
        if (k < strict) ++nstrict;
      }
    }
    res.t_rr += seconds_since(trr);
    if (nconv >= want || res.restarts >= opt.max_restarts) {
      res.theta.resize(want);
      res.resid = rn;
      res.converged.resize(want);
      for (int k = 0; k < want; ++k) {
        res.theta[k] = diag(k);
        const double tl = k < strict ? opt.tol : std::max(opt.tol, opt.tol_buffer);
        res.converged[k] = rn[k] <= tl * std::abs(diag(k));
      }
      res.coef = C;
      res.m = m;
      res.V = std::move(B.V);
      return res;
    }
    // thick restart on the real basis of the invariant subspace of the first `keep` Schur vectors
    const auto trs = std::chrono::steady_clock::now();
    // a conjugate pair split at the end of the kept set is completed, or dropped when the basis has
    // no room for its partner
    int keep0 = std::min(mmax - p, std::max(nev + p, (nev + mmax) / 2));
    if (closed(keep0) != keep0) keep0 += keep0 + 1 <= mmax - p ? 1 : -1;
    // (greedy on the real and imaginary parts of the Schur vectors: for a conjugation-closed set the
    // invariant subspace is real, of dimension keep0, and rounding-noise parts are never taken)
    std::vector<double> pool(static_cast<std::size_t>(m) * 2 * keep0);
    for (int t = 0; t < keep0; ++t)
      for (int i = 0; i < m; ++i) {
        pool[static_cast<std::size_t>(2 * t) * m + i] = U[static_cast<std::size_t>(t) * m + i].real();
        pool[static_cast<std::size_t>(2 * t + 1) * m + i] = U[static_cast<std::size_t>(t) * m + i].imag();
      }
    int keep = 0;
    std::vector<double> Q = pivoted_basis(m, 2 * keep0, pool, keep0, 1e-6, keep);
    HSG_REQUIRE(keep >= 1 && keep + p <= mmax, HSG_NOT_CONVERGED, "general Krylov-Schur: restart basis degenerate");
    // Tn = Q^T G Q, coupling Hres Q
    std::vector<double> GQ = matmul(m, m, keep, G, Q);
    std::vector<double> QT(static_cast<std::size_t>(keep) * m);
    for (int a = 0; a < keep; ++a)
      for (int i = 0; i < m; ++i) QT[a + static_cast<std::size_t>(i) * keep] = Q[i + static_cast<std::size_t>(a) * m];
    std::vector<double> Tn = matmul(keep, m, keep, QT, GQ);
    std::vector<double> Hres(static_cast<std::size_t>(p) * m);
    for (int j = 0; j < m; ++j)
      for (int a = 0; a < p; ++a) Hres[a + static_cast<std::size_t>(j) * p] = Hij(m + a, j);
    std::vector<double> Cp = matmul(p, m, keep, Hres, Q);
    B.small.alloc(Q.size());
    to_dev(B.small.p, Q, s);
    gemm_tall(n, m, keep, B.v(0), n, B.small.p, m, B.tmp.p, n, 1.0, 0.0, s);
    copy_cols(n, p, B.v(m), n, B.v(keep), n, s);
    copy_cols(n, keep, B.tmp.p, n, B.v(0), n, s);
    std::fill(Hm.begin(), Hm.end(), 0.0);
    for (int j = 0; j < keep; ++j) {
      for (int i = 0; i < keep; ++i) Hij(i, j) = Tn[i + static_cast<std::size_t>(j) * keep];
      for (int a = 0; a < p; ++a) Hij(keep + a, j) = Cp[a + static_cast<std::size_t>(j) * p];
    }
    m = keep;
    res.restarts += 1;
    cuda_check(cudaStreamSynchronize(s), "restart");
    res.t_restart += seconds_since(trs);
  }
}

}  // namespace hsg
