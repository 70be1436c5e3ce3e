// Shift-invert driver for HEP / GHEP (see driver.hpp). The logic follows hsolve's driver at the
// level of its documented contract (include/hsolve/solver.hpp): nearest targets
// (src/driver/definite.cpp:462 solve_nearest) with the exact Sylvester certificate at gap
// midpoints (:700-745, src/driver/steps.cpp:549-571), interval targets by spectrum slicing
// (definite.cpp:1020-2275 WindowSolver: window-end counts, cuts, one shift per slice), backward
// errors eta = ||Ax - lambda Bx|| / ((||A|| + |lambda| ||B||) ||x||) with Lanczos lower bounds of
// the norms (solver.hpp:7-12, src/driver/projection.cpp:54). Everything n-sized stays on the GPU.
#include "driver.hpp"

#include <algorithm>
#include <atomic>
#include <exception>
#include <mutex>
#include <future>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <map>
#include <memory>
#include <sstream>

#include "blas_kernels.cuh"
#include "common.hpp"
#include "dense_host.hpp"
#include "eigen.hpp"
#include "gpu_factor.hpp"

namespace hsg {

namespace {

using Clock = std::chrono::steady_clock;
double since(Clock::time_point t) { return std::chrono::duration<double>(Clock::now() - t).count(); }

// A full CSR matrix on the device; copies share the arrays (the views of concurrent slices).
struct DevCsr {
  std::shared_ptr<DevBuf<std::int64_t>> rp = std::make_shared<DevBuf<std::int64_t>>();
  std::shared_ptr<DevBuf<std::int32_t>> ci = std::make_shared<DevBuf<std::int32_t>>();
  std::shared_ptr<DevBuf<double>> v = std::make_shared<DevBuf<double>>();
  CsrDev view(std::int64_t n) const { return CsrDev{n, rp->p, ci->p, v->p}; }
};

void upload(DevCsr& d, const CsrHost& h, cudaStream_t s) {
  d.rp->upload(h.rp, s);
  d.ci->upload(h.ci, s);
  d.v->upload(h.v, s);
}

CsrHost upper_of(const CsrHost& m) {
  CsrHost u;
  u.n = m.n;
  u.rp.assign(m.n + 1, 0);
  for (std::int64_t i = 0; i < m.n; ++i) {
    for (std::int64_t p = m.rp[i]; p < m.rp[i + 1]; ++p)
      if (m.ci[p] >= i) { u.ci.push_back(m.ci[p]); u.v.push_back(m.v[p]); }
    u.rp[i + 1] = static_cast<std::int64_t>(u.ci.size());
  }
  return u;
}

bool is_diagonal(const CsrHost& m) {
  for (std::int64_t i = 0; i < m.n; ++i)
    for (std::int64_t p = m.rp[i]; p < m.rp[i + 1]; ++p)
      if (m.ci[p] != i && m.v[p] != 0.0) return false;
  return true;
}

// The pencil on the device and the stream its vector work is queued on. Copies share the device
// data, so concurrent slices each take a copy with a stream of their own.
struct Problem {
  std::int64_t n = 0;
  DevCsr A, B;
  bool b_identity = true;
  bool b_diagonal = false;
  std::shared_ptr<DevBuf<double>> bdiag = std::make_shared<DevBuf<double>>();
  double normA = 0.0, normB = 1.0;
  cudaStream_t s = nullptr;
  void bprod(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p) {
    if (b_identity) copy_cols(n, p, x, ldx, y, ldy, s);
    else if (b_diagonal) diag_scale(n, p, bdiag->p, x, ldx, y, ldy, s);
    else spmm(B.view(n), x, ldx, y, ldy, p, 1.0, 0.0, s);
  }
};

struct SpmvOp : KrylovOperator {
  CsrDev M;
  cudaStream_t s;
  SpmvOp(CsrDev m, cudaStream_t st) : M(m), s(st) {}
  void apply(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p) override {
    spmm(M, x, ldx, y, ldy, p, 1.0, 0.0, s);
  }
};

// An operator application with an FP32 factor whose refinement did not reach the accuracy the
// driver needs (hsolve's InexactFactorFailure, src/driver/steps.cpp:133-143): the solve falls back
// to FP64 factors.
struct InexactFactorFailure : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Refinement policy of applications with an inexact (FP32) factor (hsolve SolveRefinement,
// include/hsolve/operator.hpp:51-57, with the driver's values, src/driver/internal.hpp:233-236):
// at most 10 corrections per apply, a column is done at ||r|| <= 0.1 tol_inner ||B x|| or when its
// componentwise backward error is at the rounding level (8 eps); a correction that does not reduce
// ||r|| is discarded (every column keeps its best iterate).
constexpr int kRefineSteps = 10;
constexpr double kRefineTolFactor = 0.1;
constexpr double kRoundingLevel = 8.0 * std::numeric_limits<double>::epsilon();

struct ShiftInvertOp : KrylovOperator {
  Problem& P;
  GpuFactor& F;
  long long columns = 0;
  // refinement (FP32 factors): sigma of the factor, relative tolerances, statistics
  bool refine = false;
  double sigma = 0.0, rel_tol = 0.0, accept_rel = 0.0;
  long long refine_steps = 0, refined_applies = 0;
  double worst_rel = 0.0, worst_omega = 0.0;
  DevBuf<double> R, C, stats;
  ShiftInvertOp(Problem& pr, GpuFactor& f) : P(pr), F(f) {}
  void set_refinement(double sig, double tol_inner) {
    refine = F.single();
    sigma = sig;
    rel_tol = tol_inner * kRefineTolFactor;
    accept_rel = tol_inner;
  }
  void apply(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p) override {
    P.bprod(x, ldx, y, ldy, p);
    // the factor's object may run on its own stream (the FP32 object of the mixed path): its solve
    // waits for the work queued on the pencil's stream; it returns after its own stream finished
    F.order_after(P.s);
    if (!refine) {
      F.solve(y, p, ldy, true);
      columns += p;
      return;
    }
    apply_refined(x, ldx, y, ldy, p);
    columns += p;
  }
  // Y = K^{-1} B X with the FP32 factor K~ of K = A - sigma B and FP64 iterative refinement
  // y <- y + K~^{-1} (B x - K y), the residual r = B (x + sigma y) - A y from the FP64 pencil in one
  // sweep (ShiftInvertOperator::do_apply, hsolve src/ops/shift_invert_operator.cpp:83-177).
  void apply_refined(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p) {
    const std::int64_t n = P.n;
    cudaStream_t s = P.s;
    R.alloc(static_cast<std::size_t>(n) * p);
    C.alloc(static_cast<std::size_t>(n) * p);
    stats.alloc(3 * static_cast<std::size_t>(p));  // ||Bx||^2 | ||r||^2 | omega
    double* bxn = stats.p;
    double* rn = stats.p + p;
    double* om = stats.p + 2 * p;
    const CsrDev A = P.A.view(n);
    const CsrDev B = P.B.view(n);
    const CsrDev* Bp = P.b_identity ? nullptr : &B;
    col_dots(n, p, y, ldy, y, ldy, bxn, s);  // y = B x here
    F.order_after(s);
    F.solve(y, p, ldy, true);
    shifted_residual(A, Bp, sigma, x, ldx, y, ldy, R.p, n, p, om, s);
    col_dots(n, p, R.p, n, R.p, n, rn, s);
    std::vector<double> h(3 * static_cast<std::size_t>(p));
    auto fetch = [&] {
      cuda_check(cudaMemcpyAsync(h.data(), stats.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "refine stats");
      cuda_check(cudaStreamSynchronize(s), "refine stats");
    };
    fetch();
    std::vector<double> bx(p), rel(p), omega(p);
    std::vector<char> active(p);
    int remaining = 0;
    auto relative = [&](int k) {
      const double r = std::sqrt(h[p + k]);
      if (r == 0.0) return 0.0;
      return bx[k] > 0.0 ? r / bx[k] : std::numeric_limits<double>::infinity();
    };
    for (int k = 0; k < p; ++k) {
      bx[k] = std::sqrt(h[k]);
      rel[k] = relative(k);
      omega[k] = h[2 * p + k];
      active[k] = rel[k] > rel_tol && omega[k] > kRoundingLevel;
      remaining += active[k];
    }
    for (int step = 0; step < kRefineSteps && remaining > 0; ++step) {
      // corrections of all p columns in one block solve (the solve's time hardly depends on the
      // column count), candidates y + K~^{-1} r and their residuals
      F.order_after(s);
      F.solve(R.p, p, n, true);
      add_cols(n, p, y, ldy, R.p, n, C.p, n, s);
      shifted_residual(A, Bp, sigma, x, ldx, C.p, n, R.p, n, p, om, s);
      col_dots(n, p, R.p, n, R.p, n, rn, s);
      ++refine_steps;
      fetch();
      unsigned take = 0u;
      for (int k = 0; k < p; ++k) {
        if (!active[k]) continue;
        const double cr = relative(k);
        if (cr < rel[k]) {
          take |= 1u << k;
          rel[k] = cr;
          omega[k] = h[2 * p + k];
          if (cr > rel_tol && omega[k] > kRoundingLevel) continue;
        }
        active[k] = 0;  // converged, at the rounding level, or the correction was rejected
        --remaining;
      }
      copy_cols_masked(n, p, take, C.p, n, y, ldy, s);
    }
    ++refined_applies;
    double wr = 0.0, wo = 0.0;
    bool converged = true;
    for (int k = 0; k < p; ++k) {
      wr = std::max(wr, rel[k]);
      wo = std::max(wo, omega[k]);
      converged = converged && (rel[k] <= rel_tol || omega[k] <= kRoundingLevel);
    }
    worst_rel = std::max(worst_rel, wr);
    worst_omega = std::max(worst_omega, wo);
    if (!converged && !(wr <= accept_rel)) {
      std::ostringstream os;
      os.precision(3);
      os << "the refinement of an operator application at sigma = " << sigma << " did not converge (relative residual "
         << wr << ", backward error " << wo << "): eps_factor * cond(K) is too large at this shift";
      throw InexactFactorFailure(os.str());
    }
  }
  bool b_identity() const override { return P.b_identity; }
  void bprod(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p) override { P.bprod(x, ldx, y, ldy, p); }
};

// ||M||_2 from below (hsolve's Lanczos estimate of the 2-norm): the largest |Ritz value| of 30 plain
// Lanczos steps from a Gaussian start vector. The recurrence runs on the device with its coefficients
// there (SpMV, two dot products and two vector updates per step, no host round trip); the tridiagonal
// matrix is read once at the end. Without reorthogonalization the Ritz values may repeat, but they
// stay within the spectrum, so the bound holds.
double norm_estimate(const CsrDev& m, std::int64_t n, cudaStream_t s, std::uint64_t seed) {
  const int steps = static_cast<int>(std::min<std::int64_t>(30, n));
  constexpr int kStride = 32;  // ab: alpha_j at [j], beta_j^2 at [kStride + j], the start norm at [2 kStride]
  DevBuf<double> V, w, ab;
  V.alloc(static_cast<std::size_t>(n) * 2);  // v_j and v_{j-1} (v_{j+1} overwrites v_{j-1})
  w.alloc(static_cast<std::size_t>(n));
  ab.alloc(2 * kStride + 1);
  fill_normal(n, 1, w.p, n, seed, s);
  col_dots(n, 1, w.p, n, w.p, n, ab.p + 2 * kStride, s);
  scale_by_norm(n, w.p, V.p, ab.p + 2 * kStride, s);
  for (int j = 0; j < steps; ++j) {
    double* vj = V.p + static_cast<std::int64_t>(j % 2) * n;
    double* vo = V.p + static_cast<std::int64_t>((j + 1) % 2) * n;  // v_{j-1}, then v_{j+1}
    spmm(m, vj, n, w.p, n, 1, 1.0, 0.0, s);
    col_dots(n, 1, vj, n, w.p, n, ab.p + j, s);
    lanczos_orth(n, w.p, vj, vo, ab.p, j, kStride, s);
    col_dots(n, 1, w.p, n, w.p, n, ab.p + kStride + j, s);
    scale_by_norm(n, w.p, vo, ab.p + kStride + j, s);
  }
  std::vector<double> h(2 * kStride + 1);
  cuda_check(cudaMemcpyAsync(h.data(), ab.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "lanczos");
  cuda_check(cudaStreamSynchronize(s), "lanczos");
  std::vector<double> T(static_cast<std::size_t>(steps) * steps, 0.0), ev;
  for (int j = 0; j < steps; ++j) {
    T[j + static_cast<std::size_t>(j) * steps] = h[j];
    if (j + 1 < steps) {
      const double b = std::sqrt(std::max(h[kStride + j], 0.0));
      T[j + 1 + static_cast<std::size_t>(j) * steps] = b;
      T[j + static_cast<std::size_t>(j + 1) * steps] = b;
    }
  }
  sym_eig(steps, T, ev);
  double mx = 0.0;
  for (double x : ev) mx = std::max(mx, std::fabs(x));
  return mx;
}

struct PairMetrics {
  double lambda, abs_res, rel_res, eta;
  bool accepted;
};

std::vector<PairMetrics> pair_metrics(Problem& P, const double* X, int m, const std::vector<double>& lam, double tol) {
  std::vector<PairMetrics> out(m);
  if (m == 0) return out;
  const std::int64_t n = P.n;
  cudaStream_t s = P.s;
  DevBuf<double> AX, BX, R, lamd, dots;
  AX.alloc(static_cast<std::size_t>(n) * m);
  BX.alloc(static_cast<std::size_t>(n) * m);
  R.alloc(static_cast<std::size_t>(n) * m);
  lamd.upload(lam, s);
  dots.alloc(3 * static_cast<std::size_t>(m));
  spmm(P.A.view(n), X, n, AX.p, n, m, 1.0, 0.0, s);
  P.bprod(X, n, BX.p, n, m);
  residual_cols(n, m, AX.p, n, BX.p, n, lamd.p, R.p, n, s);
  col_dots(n, m, R.p, n, R.p, n, dots.p, s);
  col_dots(n, m, X, n, X, n, dots.p + m, s);
  col_dots(n, m, BX.p, n, BX.p, n, dots.p + 2 * m, s);
  std::vector<double> h(3 * static_cast<std::size_t>(m));
  cuda_check(cudaMemcpyAsync(h.data(), dots.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "dots");
  cuda_check(cudaStreamSynchronize(s), "pair metrics");
  for (int j = 0; j < m; ++j) {
    const double r = std::sqrt(h[j]), x = std::sqrt(h[m + j]), bx = std::sqrt(h[2 * m + j]);
    PairMetrics& q = out[j];
    q.lambda = lam[j];
    q.abs_res = r;
    q.rel_res = lam[j] != 0.0 ? r / (std::fabs(lam[j]) * bx) : r / bx;
    q.eta = r / ((P.normA + std::fabs(lam[j]) * P.normB) * x);
    q.accepted = q.eta <= tol;
  }
  return out;
}

// --------------------------------------------------------------------------- JSON writing
struct Json {
  std::ostringstream os;
  bool first = true;
  std::vector<bool> stack;
  void sep() { if (!first) os << ","; first = false; }
  void key(const char* k) { sep(); os << "\"" << k << "\":"; first = true; }
  static std::string num(double v) {
    if (std::isnan(v)) return "null";
    if (std::isinf(v)) return v > 0 ? "1e308" : "-1e308";
    char b[40];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
  }
  void val(double v) { sep(); os << num(v); }
  void val(long long v) { sep(); os << v; }
  void val(int v) { sep(); os << v; }
  void val(bool v) { sep(); os << (v ? "true" : "false"); }
  void val(const std::string& v) {
    sep();
    os << "\"";
    for (char c : v) { if (c == '"' || c == '\\') os << '\\'; os << c; }
    os << "\"";
  }
  void open(char c) { sep(); os << c; first = true; }
  void close(char c) { os << c; first = false; }
  template <class T> void kv(const char* k, const T& v) { key(k); val(v); }
};

struct Certificate {
  bool performed = false;
  double lower = 0.0, upper = 0.0;
  long long count_inertia = -1, count_found = -1, endpoint_moves = 0;
  bool passed = false;
  std::string note, method = "none";
};

struct SliceRec {
  double lower, upper, sigma;
  long long count_inertia, count_found, nev, reruns, restarts, op_applies;
  bool passed;
};

constexpr double kBatchFlopsMax = 5e11;  // per factorization
constexpr std::size_t kConcurrentSlices = 3;  // slices of one window factorized and iterated at once

struct Timers {
  double setup = 0, factor = 0, iterate = 0, verify = 0, cert = 0;
  double kry_apply = 0, kry_ortho = 0, kry_rr = 0, kry_restart = 0;  // phases of `iterate`
};

// Inertia count nu_-(A - s B) with endpoint moves on singular shifts (steps.cpp:549-571 behaviour):
// returns the count and the (possibly moved) shift.
long long count_below(GpuFactor& F, double& s, double scale, double direction, long long& moves, Timers& tm,
                      bool shared = false) {
  const auto t0 = Clock::now();
  for (int t = 0; t < 8; ++t) {
    hsg_inertia_t in = F.count(1.0, -s, true, shared);  // inertia only: no factor kept
    if (in.valid) { tm.cert += since(t0); return in.neg; }
    s += direction * 1e-7 * (scale + std::fabs(s)) * (t + 1);
    ++moves;
  }
  tm.cert += since(t0);
  HSG_THROW(HSG_SINGULAR, "inertia count: singular at every moved endpoint near " << s);
}

bool factorize_at(GpuFactor& F, double& sigma, double scale, int retries, int& used_retries, Timers& tm,
                  bool shared = false) {
  const auto t0 = Clock::now();
  for (int t = 0; t <= retries; ++t) {
    hsg_inertia_t in = F.factorize(1.0, -sigma, true, shared);
    if (in.valid) { tm.factor += since(t0); return true; }
    const double step = 1e-6 * (scale + std::fabs(sigma)) * (t + 1);
    sigma += (t % 2 == 0 ? 1.0 : -2.0) * step;
    ++used_retries;
  }
  tm.factor += since(t0);
  return false;
}

struct NearestRun {
  std::vector<double> lam;       // converged eigenvalues sorted by distance to sigma
  std::vector<int> col;          // their column in X
  DevBuf<double> X;
  int restarts = 0, applies = 0;
};

NearestRun run_krylov(ShiftInvertOp& op, Problem& P, double sigma, int nev, int nev_strict,
                      const hsg_solve_config_t& cfg, int p, std::uint64_t seed, Timers& tm) {
  const auto t0 = Clock::now();
  KsOptions o;
  o.nev = nev;
  o.nev_strict = nev_strict;
  o.ncv = static_cast<int>(cfg.ncv);
  o.block = p;
  o.tol = cfg.tol * cfg.inner_tol_factor;
  o.max_restarts = cfg.max_restarts;
  o.seed = seed;
  o.which = Which::LargestMagnitude;
  KsResult r = krylov_schur(op, P.n, o, P.s);
  tm.iterate += since(t0);
  tm.kry_apply += r.t_apply;
  tm.kry_ortho += r.t_ortho;
  tm.kry_rr += r.t_rr;
  tm.kry_restart += r.t_restart;
  NearestRun out;
  out.restarts = r.restarts;
  out.applies = r.applies;
  std::vector<std::pair<double, int>> v;
  for (std::size_t i = 0; i < r.theta.size(); ++i)
    if (r.converged[i] && r.theta[i] != 0.0) v.push_back({sigma + 1.0 / r.theta[i], static_cast<int>(i)});
  std::stable_sort(v.begin(), v.end(), [&](const auto& a, const auto& b) { return std::fabs(a.first - sigma) < std::fabs(b.first - sigma); });
  for (auto& e : v) { out.lam.push_back(e.first); out.col.push_back(e.second); }
  out.X = std::move(r.X);
  return out;
}

int auto_block(int nev) { return nev >= 32 ? 8 : (nev >= 8 ? 4 : (nev >= 3 ? 2 : 1)); }

// B^{-1} A (B = I: A), self-adjoint in the B inner product: the operator of the spectrum-end estimate.
struct PencilOp : KrylovOperator {
  Problem& P;
  GpuFactor* FB;            // B's factorization (general B)
  DevBuf<double> inv_diag;  // 1 / diag(B) (diagonal B)
  PencilOp(Problem& pr, GpuFactor* fb) : P(pr), FB(fb) {}
  void apply(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p) override {
    spmm(P.A.view(P.n), x, ldx, y, ldy, p, 1.0, 0.0, P.s);
    if (P.b_identity) return;
    if (P.b_diagonal) {
      diag_scale(P.n, p, inv_diag.p, y, ldy, y, ldy, P.s);
      return;
    }
    FB->order_after(P.s);
    FB->solve(y, p, ldy, true);
  }
  bool b_identity() const override { return P.b_identity; }
  void bprod(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p) override { P.bprod(x, ldx, y, ldy, p); }
};

// Ritz estimate of the smallest (or largest) eigenvalue of the pencil: one cycle of Lanczos on
// B^{-1} A in the B inner product, the seed of the inertia search of one-end targets (hsolve
// src/driver/solver.cpp:452-480; a general B is factorized on F for it).
double spectrum_end_estimate(Problem& P, GpuFactor& F, const CsrHost* b, bool smallest, std::uint64_t seed,
                             Timers& tm) {
  const auto t0 = Clock::now();
  PencilOp op(P, &F);
  if (!P.b_identity && P.b_diagonal) {
    std::vector<double> d(P.n, 0.0);
    for (std::int64_t i = 0; i < P.n; ++i)
      for (std::int64_t q = b->rp[i]; q < b->rp[i + 1]; ++q)
        if (b->ci[q] == i) d[i] += b->v[q];
    for (double& x : d) x = 1.0 / x;
    op.inv_diag.upload(d, P.s);
  } else if (!P.b_identity) {
    HSG_REQUIRE(F.factorize(0.0, 1.0, true).valid, HSG_INVALID_INPUT, "B is singular: not a definite generalized problem");
  }
  KsOptions o;
  o.nev = 1;
  o.ncv = static_cast<int>(std::min<std::int64_t>(30, P.n - 1));
  o.block = 1;
  o.max_restarts = 0;
  o.tol = 0.0;
  o.which = smallest ? Which::SmallestAlgebraic : Which::LargestAlgebraic;
  o.ritz_vectors = false;
  o.seed = seed;
  KsResult r = krylov_schur(op, P.n, o, P.s);
  tm.setup += since(t0);
  return r.theta.at(0);
}

// ------------------------------------------------------------------------------------ GHIEP
// Nearest target of a pencil whose B is indefinite (hsolve src/driver/indefinite.cpp:723-1000,
// solve_indefinite, the plain run at sigma): one general Krylov-Schur run of OP = (A - sigma B)^{-1} B
// in the Euclidean inner product, candidates lambda = sigma + 1/theta from its wanted Ritz values,
// real/complex classification by SolverConfig::complex_tol (solver.hpp:231-233, the test of
// indefinite.cpp:477-479), and the k candidates nearest sigma by complex distance with trustworthy
// pairs first (select_nearest, indefinite.cpp:534-557).
constexpr double kTrustworthy = 1e-6;    // pairs above this backward error only fill a shortfall
constexpr double kGhiepZeroBand = 1e-8;  // |lambda| <= kGhiepZeroBand * scale: the zero cluster of A

struct GhiepCand {
  std::complex<double> lambda;
  bool real = true;
  PairMetrics pm{};
  int col = 0;  // real: column of the coefficient matrix; complex: its vector in GhiepRun::xc
};

struct GhiepRun {
  std::vector<GhiepCand> sel;             // the selection, nearest first
  std::vector<double> coef;               // m x cols real coefficients of the candidates' vectors
  int m = 0, cols = 0;
  DevBuf<double> V;                       // the run's basis (n x m)
  std::vector<double> xc;                 // host vectors (n x 2: re, im) of the complex candidates
  int restarts = 0, applies = 0, block = 0;
  long long good = 0, in_band = 0;
};

// Metrics of a pair given x, A x, B x on the host (complex lambda, vectors as re / im columns).
PairMetrics complex_metrics(const Problem& P, std::int64_t n, const double* x, const double* ax, const double* bx,
                            std::complex<double> lam, double tol) {
  double rr = 0.0, xx = 0.0, bb = 0.0;
  for (std::int64_t i = 0; i < n; ++i) {
    const std::complex<double> xv(x[i], x[n + i]), av(ax[i], ax[n + i]), bv(bx[i], bx[n + i]);
    rr += std::norm(av - lam * bv);
    xx += std::norm(xv);
    bb += std::norm(bv);
  }
  PairMetrics q{};
  q.lambda = lam.real();
  q.abs_res = std::sqrt(rr);
  const double al = std::abs(lam);
  q.rel_res = al != 0.0 ? q.abs_res / (al * std::sqrt(bb)) : q.abs_res / std::sqrt(bb);
  q.eta = q.abs_res / ((P.normA + al * P.normB) * std::sqrt(xx));
  q.accepted = q.eta <= tol;
  return q;
}

GhiepRun ghiep_run(ShiftInvertOp& op, Problem& P, double sigma, int nev, int k, const hsg_solve_config_t& cfg, int p,
                   double scale, double band_user, double complex_tol, Timers& tm) {
  using cplx = std::complex<double>;
  const std::int64_t n = P.n;
  cudaStream_t s = P.s;
  const auto t0 = Clock::now();
  KsOptions o;
  o.nev = nev;
  o.nev_strict = k;
  o.ncv = static_cast<int>(cfg.ncv);
  o.block = p;
  o.tol = cfg.tol * cfg.inner_tol_factor;
  o.max_restarts = cfg.max_restarts;
  o.seed = cfg.seed;
  GeneralKsResult r = krylov_schur_general(op, n, o, s);
  tm.iterate += since(t0);
  tm.kry_apply += r.t_apply;
  tm.kry_ortho += r.t_ortho;
  tm.kry_rr += r.t_rr;
  tm.kry_restart += r.t_restart;
  const auto tv = Clock::now();
  GhiepRun out;
  out.restarts = r.restarts;
  out.applies = r.applies;
  out.block = p;
  const int m = r.m;
  std::vector<cplx> mu;
  std::vector<int> src;
  for (std::size_t j = 0; j < r.theta.size(); ++j) {
    if (r.theta[j] == cplx(0.0)) continue;
    mu.push_back(sigma + 1.0 / r.theta[j]);
    src.push_back(static_cast<int>(j));
  }
  const int nc = static_cast<int>(mu.size());
  auto cf = [&](int q, int i) { return r.coef[static_cast<std::size_t>(src[q]) * m + i]; };
  std::vector<char> small(nc);
  for (int q = 0; q < nc; ++q) small[q] = std::fabs(mu[q].imag()) <= complex_tol * std::max(std::abs(mu[q]), scale);
  // real vector of every candidate: the real part of e^{i phi} c with the phase that maximizes its
  // norm (the top eigenvector of the 2 x 2 Gram matrix of Re c, Im c; the basis is orthonormal, so
  // this works on the coefficients)
  std::vector<int> cidx;
  for (int q = 0; q < nc; ++q)
    if (!small[q]) cidx.push_back(q);
  const int cols = nc + 2 * static_cast<int>(cidx.size());
  std::vector<double> Y(static_cast<std::size_t>(m) * std::max(cols, 1), 0.0);
  for (int q = 0; q < nc; ++q) {
    double aa = 0.0, bb = 0.0, ab = 0.0;
    for (int i = 0; i < m; ++i) {
      const cplx z = cf(q, i);
      aa += z.real() * z.real();
      bb += z.imag() * z.imag();
      ab += z.real() * z.imag();
    }
    const double phi = 0.5 * std::atan2(-2.0 * ab, aa - bb);
    const double c = std::cos(phi), sn = std::sin(phi);
    double nr = 0.0;
    double* y = &Y[static_cast<std::size_t>(q) * m];
    for (int i = 0; i < m; ++i) {
      y[i] = cf(q, i).real() * c - cf(q, i).imag() * sn;
      nr += y[i] * y[i];
    }
    nr = std::sqrt(nr);
    if (nr > 0.0)
      for (int i = 0; i < m; ++i) y[i] /= nr;
  }
  // a multiple real eigenvalue: its candidates take an orthonormal basis of its (real) eigenspace,
  // drawn greedily from their real vectors and the real and imaginary parts of their Ritz vectors
  // (the best-separated directions first, so that a part that is only rounding noise is never
  // taken), so the copies stay independent
  {
    std::vector<int> rs;
    for (int q = 0; q < nc; ++q)
      if (small[q]) rs.push_back(q);
    std::stable_sort(rs.begin(), rs.end(), [&](int a, int b) { return mu[a].real() < mu[b].real(); });
    for (std::size_t g0 = 0; g0 < rs.size();) {
      std::size_t g1 = g0 + 1;
      while (g1 < rs.size() && std::fabs(mu[rs[g1]].real() - mu[rs[g1 - 1]].real()) <=
                                   1e-8 * std::max(std::fabs(mu[rs[g1]].real()), scale))
        ++g1;
      const int g = static_cast<int>(g1 - g0);
      if (g > 1) {
        std::vector<double> pool(static_cast<std::size_t>(m) * 3 * g);
        for (int t = 0; t < g; ++t)
          for (int i = 0; i < m; ++i) {
            pool[static_cast<std::size_t>(t) * m + i] = Y[static_cast<std::size_t>(rs[g0 + t]) * m + i];
            pool[static_cast<std::size_t>(g + 2 * t) * m + i] = cf(rs[g0 + t], i).real();
            pool[static_cast<std::size_t>(g + 2 * t + 1) * m + i] = cf(rs[g0 + t], i).imag();
          }
        int rank = 0;
        std::vector<double> Qg = pivoted_basis(m, 3 * g, pool, g, 1e-3, rank);
        if (rank == g)
          for (int t = 0; t < g; ++t)
            std::copy(Qg.begin() + static_cast<std::ptrdiff_t>(t) * m, Qg.begin() + static_cast<std::ptrdiff_t>(t + 1) * m,
                      Y.begin() + static_cast<std::ptrdiff_t>(rs[g0 + t]) * m);
      }
      g0 = g1;
    }
  }
  for (std::size_t t = 0; t < cidx.size(); ++t)
    for (int i = 0; i < m; ++i) {
      Y[static_cast<std::size_t>(nc + 2 * t) * m + i] = cf(cidx[t], i).real();
      Y[static_cast<std::size_t>(nc + 2 * t + 1) * m + i] = cf(cidx[t], i).imag();
    }
  // vectors and their images on the device
  DevBuf<double> Yd, X, AX, BX, R, lamd, dots;
  Yd.upload(Y, s);
  X.alloc(static_cast<std::size_t>(n) * std::max(cols, 1));
  AX.alloc(static_cast<std::size_t>(n) * std::max(cols, 1));
  BX.alloc(static_cast<std::size_t>(n) * std::max(cols, 1));
  R.alloc(static_cast<std::size_t>(n) * std::max(nc, 1));
  dots.alloc(4 * static_cast<std::size_t>(std::max(nc, 1)));
  std::vector<double> h(4 * static_cast<std::size_t>(nc));
  std::vector<double> lam_r(nc);
  if (nc > 0) {
    gemm_tall(n, m, cols, r.V.p, n, Yd.p, m, X.p, n, 1.0, 0.0, s);
    spmm(P.A.view(n), X.p, n, AX.p, n, cols, 1.0, 0.0, s);
    P.bprod(X.p, n, BX.p, n, cols);
    col_dots(n, nc, X.p, n, AX.p, n, dots.p, s);
    col_dots(n, nc, X.p, n, BX.p, n, dots.p + nc, s);
    col_dots(n, nc, BX.p, n, BX.p, n, dots.p + 2 * nc, s);
    cuda_check(cudaMemcpyAsync(h.data(), dots.p, 3 * nc * sizeof(double), cudaMemcpyDeviceToHost, s), "ghiep dots");
    cuda_check(cudaStreamSynchronize(s), "ghiep dots");
    // lambda of a real vector: its Rayleigh quotient x^T A x / x^T B x (x^T is also a left
    // eigenvector of a real symmetric pencil, so the quotient is accurate to second order), unless
    // x^T B x is too small for it or it leaves the Ritz estimate; then Re(mu)
    for (int q = 0; q < nc; ++q) {
      lam_r[q] = mu[q].real();
      const double xbx = h[nc + q], bxn = std::sqrt(h[2 * nc + q]);
      if (std::fabs(xbx) >= 1e-3 * bxn && bxn > 0.0) {
        const double rq = h[q] / xbx;
        if (std::fabs(rq - mu[q].real()) <= 1e-6 * std::max(std::abs(mu[q]), scale)) lam_r[q] = rq;
      }
    }
    lamd.upload(lam_r, s);
    residual_cols(n, nc, AX.p, n, BX.p, n, lamd.p, R.p, n, s);
    col_dots(n, nc, R.p, n, R.p, n, dots.p, s);
    col_dots(n, nc, X.p, n, X.p, n, dots.p + nc, s);
    cuda_check(cudaMemcpyAsync(h.data(), dots.p, 2 * nc * sizeof(double), cudaMemcpyDeviceToHost, s), "ghiep dots");
    cuda_check(cudaStreamSynchronize(s), "ghiep dots");
  }
  std::vector<GhiepCand> cands(nc);
  for (int q = 0; q < nc; ++q) {
    GhiepCand& c = cands[q];
    c.lambda = cplx(lam_r[q], 0.0);
    c.col = q;
    PairMetrics& pm = c.pm;
    const double rn = std::sqrt(h[q]), xn = std::sqrt(h[nc + q]), bxn = std::sqrt(h[2 * nc + q]);
    pm.lambda = lam_r[q];
    pm.abs_res = rn;
    pm.rel_res = lam_r[q] != 0.0 ? rn / (std::fabs(lam_r[q]) * bxn) : rn / bxn;
    pm.eta = rn / ((P.normA + std::fabs(lam_r[q]) * P.normB) * xn);
    pm.accepted = pm.eta <= cfg.tol;
  }
  // candidates with a significant imaginary part: the complex pair is kept when the real
  // projection fails the tolerance and the complex pair does at least as well
  if (!cidx.empty()) {
    const std::size_t w = static_cast<std::size_t>(n) * 2;
    std::vector<double> hx(w * cidx.size()), hax(hx.size()), hbx(hx.size());
    const std::size_t off = static_cast<std::size_t>(n) * nc;
    cuda_check(cudaMemcpyAsync(hx.data(), X.p + off, hx.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "ghiep x");
    cuda_check(cudaMemcpyAsync(hax.data(), AX.p + off, hx.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "ghiep ax");
    cuda_check(cudaMemcpyAsync(hbx.data(), BX.p + off, hx.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "ghiep bx");
    cuda_check(cudaStreamSynchronize(s), "ghiep complex");
    out.xc = hx;
    for (std::size_t t = 0; t < cidx.size(); ++t) {
      const int q = cidx[t];
      const double* x = &hx[t * w];
      const double* ax = &hax[t * w];
      const double* bx = &hbx[t * w];
      // the unconjugated quotient x^T A x / x^T B x of the complex vector, under the same guard
      cplx lam = mu[q];
      cplx xax = 0.0, xbx = 0.0;
      double bb = 0.0;
      for (std::int64_t i = 0; i < n; ++i) {
        const cplx xv(x[i], x[n + i]);
        xax += xv * cplx(ax[i], ax[n + i]);
        xbx += xv * cplx(bx[i], bx[n + i]);
        bb += std::norm(cplx(bx[i], bx[n + i]));
      }
      if (std::abs(xbx) >= 1e-3 * std::sqrt(bb) && bb > 0.0) {
        const cplx rq = xax / xbx;
        if (std::abs(rq - mu[q]) <= 1e-6 * std::max(std::abs(mu[q]), scale)) lam = rq;
      }
      const PairMetrics pc = complex_metrics(P, n, x, ax, bx, lam, cfg.tol);
      GhiepCand& c = cands[q];
      if (c.pm.eta > cfg.tol && pc.eta <= c.pm.eta) {
        c.real = false;
        c.lambda = lam;
        c.pm = pc;
        c.col = static_cast<int>(t);
      }
    }
  }
  // selection (select_nearest): outside the user's zero band, trustworthy pairs first
  auto dist = [&](const GhiepCand& c) { return std::abs(c.lambda - cplx(sigma)); };
  std::vector<GhiepCand> good, poor;
  for (const auto& c : cands) {
    const bool trusted = c.pm.eta <= std::max(kTrustworthy, cfg.tol);
    if (band_user >= 0.0 && std::abs(c.lambda) <= band_user) {
      out.in_band += trusted;
      continue;
    }
    (trusted ? good : poor).push_back(c);
  }
  auto nearer = [&](const GhiepCand& a, const GhiepCand& b) { return dist(a) < dist(b); };
  std::stable_sort(good.begin(), good.end(), nearer);
  std::stable_sort(poor.begin(), poor.end(), nearer);
  if (good.size() > static_cast<std::size_t>(k)) good.resize(static_cast<std::size_t>(k));
  out.good = static_cast<long long>(good.size());
  out.sel = good;
  for (const auto& c : poor) {
    if (out.sel.size() >= static_cast<std::size_t>(k)) break;
    out.sel.push_back(c);
  }
  std::stable_sort(out.sel.begin(), out.sel.end(), nearer);
  out.coef = std::move(Y);
  out.m = m;
  out.cols = cols;
  out.V = std::move(r.V);
  cuda_check(cudaStreamSynchronize(s), "ghiep");
  tm.verify += since(tv);
  return out;
}

}  // namespace

struct Session::Impl {
  CsrHost a;
  std::unique_ptr<CsrHost> b;
  std::unique_ptr<GpuFactor> F;
  // two more factorization objects on the same analysis, created at first use: the inertia counts
  // of the window ends run on them concurrently with each other and with F's slice factorization
  std::unique_ptr<GpuFactor> C[2];
  hsg_options_t fopt{};
  GpuFactor& counter(int i) {
    if (!C[i]) {
      auto g = std::make_unique<GpuFactor>(fopt);
      g->analyze_like(*F);
      C[i] = std::move(g);
    }
    return *C[i];
  }
  // the FP32 operator factorization of the mixed-precision path (same analysis), created at first use
  std::unique_ptr<GpuFactor> FS;
  GpuFactor& single_op() {
    if (!FS) {
      hsg_options_t o = fopt;
      o.precision = 1;
      auto g = std::make_unique<GpuFactor>(o);
      g->analyze_like(*F);
      FS = std::move(g);
    }
    return *FS;
  }
  // factorization objects of concurrent slices (lane 0: F, or the FP32 object of the mixed path;
  // further lanes created at first use, per precision)
  std::vector<std::unique_ptr<GpuFactor>> lanes[2];
  std::mutex lanes_mu;
  GpuFactor& slice_object(int lane, bool single) {
    if (lane == 0) return single ? single_op() : *F;
    std::lock_guard<std::mutex> lk(lanes_mu);
    auto& v = lanes[single ? 1 : 0];
    if (static_cast<int>(v.size()) < lane) v.resize(lane);
    if (!v[lane - 1]) {
      hsg_options_t o = fopt;
      o.precision = single ? 1 : 0;
      auto g = std::make_unique<GpuFactor>(o);
      g->analyze_like(*F);
      v[lane - 1] = std::move(g);
    }
    return *v[lane - 1];
  }
  Problem P;
  std::string problem = "HEP";
  double scale = 0.0;
  Timers setup_tm;
  int device = 0;
  std::uint64_t seed = 2026;
};

Session::Session(const CsrHost& a_in, const CsrHost* b_in, int device, std::uint64_t seed) : d_(new Impl) {
  Impl& S = *d_;
  S.a = a_in;
  if (b_in) S.b = std::make_unique<CsrHost>(*b_in);
  S.device = device;
  S.seed = seed;
  const CsrHost& a = S.a;
  const CsrHost* b = S.b.get();
  Timers& tm = S.setup_tm;
  const std::int64_t n = a.n;
  HSG_REQUIRE(n > 0, HSG_INVALID_INPUT, "empty matrix");
  HSG_REQUIRE(!b || b->n == n, HSG_INVALID_INPUT, "A and B differ in size");
  hsg_options_t fo;
  hsg_default_options(&fo);
  fo.device = device;
  S.fopt = fo;
  S.F = std::make_unique<GpuFactor>(fo);
  GpuFactor& F = *S.F;
  Problem& P = S.P;
  P.n = n;
  P.s = F.stream();
  cuda_check(cudaSetDevice(device), "cudaSetDevice");
  PoolStreamScope scope(P.s);
  upload(P.A, a, P.s);
  if (b) {
    upload(P.B, *b, P.s);
    P.b_identity = false;
    P.b_diagonal = is_diagonal(*b);
    S.problem = "GHEP";
    if (P.b_diagonal) {
      std::vector<double> d(n, 0.0);
      for (std::int64_t i = 0; i < n; ++i)
        for (std::int64_t q = b->rp[i]; q < b->rp[i + 1]; ++q)
          if (b->ci[q] == i) d[i] += b->v[q];
      double mx = 0.0, mn = std::numeric_limits<double>::infinity();
      for (double x : d) { mx = std::max(mx, std::fabs(x)); mn = std::min(mn, x); }
      if (!(mn > 0.0)) S.problem = "GHIEP";  // a non-positive diagonal entry: B is not positive definite
      P.bdiag->upload(d, P.s);
      P.normB = mx;
    }
  }
  {
    const auto t0 = Clock::now();
    P.normA = norm_estimate(P.A.view(n), n, P.s, seed + 7);
    if (b && !P.b_diagonal) P.normB = norm_estimate(P.B.view(n), n, P.s, seed + 11);
    tm.setup += since(t0);
  }
  S.scale = P.normB > 0 ? P.normA / P.normB : P.normA;
  {
    const auto t0 = Clock::now();
    const CsrHost au = upper_of(a);
    CsrHost bu;
    if (b) bu = upper_of(*b);
    F.analyze(n, au.rp.data(), au.ci.data(), au.v.data(), b ? bu.rp.data() : nullptr, b ? bu.ci.data() : nullptr,
              b ? bu.v.data() : nullptr, nullptr);
    tm.factor += since(t0);
  }
  if (b && !P.b_diagonal) {
    // definiteness of B by its inertia (hsolve src/driver/solver.cpp:426-441): B singular or with a
    // negative pivot makes the pencil a GHIEP
    const auto t0 = Clock::now();
    hsg_inertia_t in = F.factorize(0.0, 1.0, true);
    tm.factor += since(t0);
    if (!(in.valid && in.neg == 0 && in.zero == 0)) S.problem = "GHIEP";
  }
}

Session::~Session() = default;

std::int64_t Session::order() const { return d_->a.n; }

hsg_estimate_t Session::estimate() const { return d_->F->estimate(); }

// Exclusion certificate on the session's factorization object, factorized at opt.sigma (hsolve's
// exclusion_check, include/hsolve/verify.hpp:110-175). The start block is B^-1/2 G for a diagonal B
// (kappa = 1 exactly), G for B = I; a general B takes the caller's kappa and the result is flagged
// as not rigorous.
hsg_exclusion_result_t Session::exclusion_check(const double* x, std::int64_t m, std::int64_t ldx,
                                                const hsg_exclusion_options_t& o) {
  Impl& S = *d_;
  HSG_REQUIRE(S.problem != "GHIEP", HSG_UNSUPPORTED, "exclusion check: B must be positive definite");
  const std::int64_t n = S.P.n;
  HSG_REQUIRE(x && m >= 1 && m < n && ldx >= n, HSG_INVALID_INPUT,
              "exclusion check: X must be n x m (1 <= m < n) with ld >= n");
  HSG_REQUIRE(std::isfinite(o.sigma), HSG_INVALID_INPUT, "exclusion check: sigma must be finite");
  cuda_check(cudaSetDevice(S.device), "cudaSetDevice");
  Problem& P = S.P;
  PoolStreamScope scope(P.s);
  GpuFactor& F = *S.F;
  double sigma = o.sigma;
  Timers tm;
  int used = 0;
  HSG_REQUIRE(factorize_at(F, sigma, S.scale, 4, used, tm), HSG_FACTORIZATION_FAILED,
              "exclusion check: A - sigma B could not be factorized near sigma");
  ShiftInvertOp op(P, F);
  DevBuf<double> X;
  X.alloc(static_cast<std::size_t>(n) * m);
  cuda_check(cudaMemcpy2DAsync(X.p, n * sizeof(double), x, ldx * sizeof(double), n * sizeof(double), m,
                               cudaMemcpyHostToDevice, P.s), "exclusion check: X");
  ExclusionOptions eo;
  eo.radius = o.radius;
  eo.pass_radius = o.pass_radius;
  eo.delta = o.delta;
  eo.block = o.block_size;
  eo.seed = o.seed;
  eo.rounding_margin = o.rounding_margin;
  eo.max_block_steps = o.max_block_steps;
  eo.max_krylov_vectors = o.max_krylov_vectors;
  DevBuf<double> sc;
  const double* start_scale = nullptr;
  bool rigorous = true;
  if (P.b_identity) {
    eo.kappa = 1.0;
  } else if (P.b_diagonal) {
    std::vector<double> d(static_cast<std::size_t>(n));
    cuda_check(cudaMemcpyAsync(d.data(), P.bdiag->p, n * sizeof(double), cudaMemcpyDeviceToHost, P.s), "B diagonal");
    cuda_check(cudaStreamSynchronize(P.s), "B diagonal");
    for (double& v : d) v = 1.0 / std::sqrt(v);
    sc.upload(d, P.s);
    start_scale = sc.p;
    eo.kappa = 1.0;
  } else {
    eo.kappa = std::max(1.0, o.kappa);
    rigorous = false;
  }
  const ExclusionResult r = hsg::exclusion_check(op, n, X.p, static_cast<int>(m), eo, start_scale, P.s);
  cuda_check(cudaStreamSynchronize(P.s), "exclusion check");
  hsg_exclusion_result_t out{};
  out.status = static_cast<int32_t>(r.status);
  out.exact = r.exact ? 1 : 0;
  out.over_budget = r.over_budget ? 1 : 0;
  out.rigorous = (rigorous || r.exact) ? 1 : 0;
  out.sigma = sigma;
  out.claim_threshold = r.claim_threshold;
  out.pass_threshold = r.pass_threshold;
  out.coupling = r.coupling;
  out.epsilon = r.epsilon;
  out.kappa = r.kappa;
  out.deflated = r.deflated;
  out.dimension = r.dimension;
  out.found_inside = r.found_inside;
  out.certified_inside = r.certified_inside;
  out.block_size = r.block;
  out.block_steps_planned = r.block_steps_planned;
  out.block_steps = r.block_steps;
  out.krylov_vectors_planned = r.krylov_vectors_planned;
  out.max_ritz = r.max_ritz;
  out.failure_probability = r.failure_probability;
  out.new_count = r.new_count;
  out.new_inside = r.new_inside;
  out.op_applications = r.op_applications;
  out.setup_s = r.setup_s;
  out.krylov_s = r.krylov_s;
  return out;
}

// factor_precision = single: the shift factorizations that serve the operator are FP32 with FP64
// refinement of every application; the inertia counts stay FP64. As in hsolve (solver.hpp:116-126),
// the attempt is abandoned for FP64 factors when an application's refinement does not converge or
// the result is not accepted (a pair above tol or a failed certificate).
SolveOutput Session::solve(const hsg_solve_config_t& cfg, bool include_setup) {
  if (cfg.factor_precision != 1) return solve_once(cfg, include_setup, "");
  std::string why;
  try {
    SolveOutput out = solve_once(cfg, include_setup, "");
    if (out.report_json.find("\"success\":true") != std::string::npos) return out;
    why = "the single-precision result was not accepted";
  } catch (const InexactFactorFailure& e) {
    why = e.what();
  }
  hsg_solve_config_t c2 = cfg;
  c2.factor_precision = 0;
  return solve_once(c2, include_setup, why);
}

SolveOutput Session::solve_once(const hsg_solve_config_t& cfg, bool include_setup, const std::string& fallback) {
  const auto t_start = Clock::now();
  Impl& S = *d_;
  Timers tm;
  if (include_setup) tm = S.setup_tm;
  const CsrHost& a = S.a;
  const CsrHost* b = S.b.get();
  const std::int64_t n = a.n;
  HSG_REQUIRE(cfg.tol > 0.0 && cfg.tol < 1.0, HSG_INVALID_INPUT, "tol outside (0, 1)");
  HSG_REQUIRE(cfg.mode >= 0 && cfg.mode <= 3, HSG_INVALID_INPUT, "target mode must be nearest, interval, smallest or largest");
  HSG_REQUIRE(cfg.factor_precision == 0 || cfg.factor_precision == 1, HSG_INVALID_INPUT, "factor_precision");
  HSG_REQUIRE(cfg.device == S.device, HSG_INVALID_INPUT, "config device differs from the session's device");
  GpuFactor& F = *S.F;
  Problem& P = S.P;
  PoolStreamScope scope(P.s);  // buffers released below are stream-ordered on the pencil's stream
  // the factorization object that serves the operator: F itself (FP64), or the FP32 object of the
  // mixed-precision path; F, C0 and C1 keep every inertia count in FP64
  const bool single = cfg.factor_precision == 1;
  GpuFactor& OPF = single ? S.single_op() : F;
  F.reset_device_stats();
  if (single) OPF.reset_device_stats();
  const long long launches0 = hsg_kernel_launches();
  const double scale = S.scale;
  const std::string problem = S.problem;
  std::vector<std::string> warnings;
  if (!fallback.empty()) warnings.push_back("single-precision factors abandoned: " + fallback);
  ShiftInvertOp op(P, OPF);
  const double tol_inner = cfg.tol * cfg.inner_tol_factor;
  SolveOutput out;
  out.n = n;
  Certificate cert;
  std::vector<SliceRec> slices;
  std::vector<double> lam_out;
  DevBuf<double> Xout;
  int shift_retries = 0, restarts = 0, block_used = 0;
  long long applies_before = 0;
  double sigma_used = cfg.sigma;
  const bool certify = cfg.certificate == 0;
  // concurrent shifts pay while a factorization is latency-bound; above kBatchFlopsMax flops the
  // fronts keep the whole device busy and shifts run one after another
  const bool batch = cfg.batch_shifts != 0 && F.estimate().flops <= kBatchFlopsMax;
  bool f_stale = false;  // F's factorization was overwritten by a count at another shift
  // GHIEP: B indefinite (detected), or the indefinite path asked for (problem = 3)
  HSG_REQUIRE(!(cfg.problem == 2 && problem == "GHIEP"), HSG_INVALID_INPUT,
              "problem = generalized_definite, but B is not positive definite");
  HSG_REQUIRE(!(cfg.problem == 3 && !b), HSG_INVALID_INPUT, "problem = generalized_indefinite needs B");
  const bool ghiep = problem == "GHIEP" || cfg.problem == 3;
  HSG_REQUIRE(!ghiep || cfg.mode == 0, HSG_UNSUPPORTED,
              "indefinite-B problems support target mode 'nearest' only: interval / smallest / largest need "
              "eigenvalue counts, which Sylvester inertia does not give for indefinite B");
  // smallest / largest k: the window (-inf, U] with nu(U) >= k, or [L, +inf) with n - nu(L) >= k, by
  // inertia search from a Ritz estimate of the spectrum's end (hsolve src/driver/definite.cpp:1918-
  // 1993), closed at a point beyond the end (count 0, or n); then solved as an interval and the k
  // smallest (ascending) or largest (descending) kept
  const bool one_end = !ghiep && (cfg.mode == 2 || cfg.mode == 3);
  double win_lo = cfg.lower, win_hi = cfg.upper;
  long long window_count = -1;
  if (one_end) {
    const std::int64_t k = cfg.k;
    HSG_REQUIRE(k >= 1 && k <= n, HSG_INVALID_INPUT, "k must be in [1, n]");
    const bool smallest = cfg.mode == 2;
    const double est = spectrum_end_estimate(P, F, b, smallest, cfg.seed + 3, tm);
    const double step0 = 1e-2 * (std::fabs(est) + scale);
    const double dir = smallest ? 1.0 : -1.0;  // from the end into the spectrum
    const long long slack = std::max<long long>(4, k / 4);
    long long moves = 0;
    // the closing point beyond the end: nu = 0 (smallest) or n (largest)
    double end = est - dir * step0;
    const long long end_count = smallest ? 0 : n;
    long long ne = count_below(F, end, scale, -dir, moves, tm);
    for (int t = 0; ne != end_count; ++t) {
      HSG_REQUIRE(t < 60, HSG_NOT_CONVERGED, "one-end target: no point beyond the end of the spectrum found");
      end -= dir * step0 * std::ldexp(1.0, t + 1);
      ne = count_below(F, end, scale, -dir, moves, tm);
    }
    // the inner end: grow the step until the window holds k, then bisect down to at most k + slack
    auto held = [&](long long nu) { return smallest ? nu : n - nu; };
    double a = end, c = est + dir * step0;
    long long nc = count_below(F, c, scale, dir, moves, tm);
    for (int t = 0; held(nc) < k; ++t) {
      HSG_REQUIRE(t < 60, HSG_NOT_CONVERGED, "one-end target: the window never reached k eigenvalues");
      a = c;
      c += dir * step0 * std::ldexp(1.0, t + 1);
      nc = count_below(F, c, scale, dir, moves, tm);
    }
    for (int t = 0; t < 40 && held(nc) > k + slack && std::fabs(c - a) > 1e-9 * (scale + std::fabs(c)); ++t) {
      double mid = 0.5 * (a + c);
      const long long nm = count_below(F, mid, scale, dir, moves, tm);
      if (held(nm) >= k) {
        c = mid;
        nc = nm;
      } else {
        a = mid;
      }
    }
    win_lo = smallest ? end : c;
    win_hi = smallest ? c : end;
    window_count = held(nc);
    if (window_count < k)
      warnings.push_back("the target window holds only " + std::to_string(window_count) + " eigenvalue(s), fewer than k");
  }
  std::vector<PairMetrics> cpm;  // GHIEP: metrics of the complex pairs (lambda_re in .lambda)
  std::vector<double> c_im;      // and their imaginary parts
  long long zero_cluster_dim = -1;

  if (cfg.mode == 0 && ghiep) {
    // ---------------------------------------------------------------- nearest, B indefinite
    const std::int64_t k = cfg.k;
    HSG_REQUIRE(k >= 1 && k < n, HSG_INVALID_INPUT, "k must be in [1, n)");
    double sigma = cfg.sigma;
    HSG_REQUIRE(std::isfinite(sigma), HSG_INVALID_INPUT, "sigma must be finite");
    HSG_REQUIRE(cfg.complex_tol >= 0.0, HSG_INVALID_INPUT, "complex_tol must be >= 0");
    cert.note = "not available for indefinite B (Sylvester inertia does not count eigenvalues)";
    const double band_user = cfg.zero_filter_tol >= 0.0 ? cfg.zero_filter_tol * scale : -1.0;
    const double band_zero = std::max(band_user, kGhiepZeroBand * scale);
    if (!factorize_at(OPF, sigma, scale, cfg.max_shift_retries, shift_retries, tm))
      HSG_THROW(HSG_SINGULAR, "A - sigma B is numerically singular at and near sigma = " << cfg.sigma);
    op.set_refinement(sigma, tol_inner);
    sigma_used = sigma;
    int nev = static_cast<int>(std::min<std::int64_t>(n - 1, k + std::max<std::int64_t>(4, (k + 1) / 2)));
    // the block width: multi-column solves cost little more than single ones on the GPU, and a block
    // of p takes up to p copies of a multiple eigenvalue at once
    const int p = cfg.block_size > 0
                      ? static_cast<int>(std::max<std::int64_t>(1, std::min<std::int64_t>({cfg.block_size, nev, kMaxKrylovBlock, n / 16})))
                      : auto_block(nev);
    block_used = p;
    GhiepRun run;
    for (int attempt = 0; attempt < 3; ++attempt) {
      run = ghiep_run(op, P, sigma, nev, static_cast<int>(k), cfg, p, scale, band_user, cfg.complex_tol, tm);
      restarts += run.restarts;
      if (run.good >= k || nev >= n - 1) break;
      warnings.push_back("fewer trustworthy pairs than k; rerun with more");
      nev = static_cast<int>(std::min<std::int64_t>(n - 1, 2 * nev));
    }
    // does the zero cluster of A interfere: a selected pair in its band, too few pairs, or the
    // selection disk reaching the band (indefinite.cpp:763-772)
    double radius = 0.0;
    bool touches = static_cast<std::int64_t>(run.sel.size()) < k;
    for (const auto& c : run.sel) {
      radius = std::max(radius, std::abs(c.lambda - std::complex<double>(sigma)));
      touches = touches || std::abs(c.lambda) <= band_zero;
    }
    touches = touches || radius >= std::fabs(sigma) - band_zero;
    if (touches) {
      // dim null(A): null pivots of an LDL^T of A on the same analysis (indefinite.cpp:561)
      const auto t0 = Clock::now();
      zero_cluster_dim = static_cast<long long>(F.factorize(1.0, 0.0, true).null_pivots);
      tm.factor += since(t0);
      HSG_REQUIRE(band_user < 0.0 && zero_cluster_dim == 0, HSG_UNSUPPORTED,
                  "the " << k << " eigenvalues nearest sigma = " << sigma << " reach the zero cluster of A (dimension "
                         << zero_cluster_dim << ", |lambda| <= " << band_zero
                         << "): the one-sided runs around the cluster are not built; choose sigma so that the k "
                            "nearest eigenvalues lie closer to sigma than 0 does");
    }
    // outputs: real pairs nearest first, then the complex ones
    std::vector<double> S;
    for (const auto& c : run.sel) {
      if (c.real) {
        lam_out.push_back(c.lambda.real());
        S.insert(S.end(), run.coef.begin() + static_cast<std::ptrdiff_t>(c.col) * run.m,
                 run.coef.begin() + static_cast<std::ptrdiff_t>(c.col + 1) * run.m);
      } else {
        out.complex_eigenvalues.push_back(c.lambda.real());
        out.complex_eigenvalues.push_back(c.lambda.imag());
        const double* x = &run.xc[static_cast<std::size_t>(c.col) * 2 * n];
        for (std::int64_t i = 0; i < n; ++i) {
          out.complex_vectors.push_back(x[i]);
          out.complex_vectors.push_back(x[n + i]);
        }
        cpm.push_back(c.pm);
        c_im.push_back(c.lambda.imag());
      }
    }
    const int kr = static_cast<int>(lam_out.size());
    Xout.alloc(static_cast<std::size_t>(n) * std::max(kr, 1));
    if (kr > 0) {
      DevBuf<double> Sd;
      Sd.upload(S, P.s);
      gemm_tall(n, run.m, kr, run.V.p, n, Sd.p, run.m, Xout.p, n, 1.0, 0.0, P.s);
      cuda_check(cudaStreamSynchronize(P.s), "ghiep vectors");
    }
    if (!cpm.empty())
      warnings.push_back(std::to_string(cpm.size()) + " genuinely complex eigenvalue(s) returned separately");
    if (static_cast<std::int64_t>(run.sel.size()) < k)
      warnings.push_back("only " + std::to_string(run.sel.size()) + " of " + std::to_string(k) + " pairs found");
  } else if (cfg.mode == 0) {
    // ---------------------------------------------------------------- nearest
    const std::int64_t k = cfg.k;
    HSG_REQUIRE(k >= 1 && k < n, HSG_INVALID_INPUT, "k must be in [1, n)");
    double sigma = cfg.sigma;
    HSG_REQUIRE(std::isfinite(sigma), HSG_INVALID_INPUT, "sigma must be finite");
    if (!factorize_at(OPF, sigma, scale, cfg.max_shift_retries, shift_retries, tm))
      HSG_THROW(HSG_SINGULAR, "A - sigma B is numerically singular at and near sigma = " << cfg.sigma);
    op.set_refinement(sigma, tol_inner);
    sigma_used = sigma;
    int nev = static_cast<int>(std::min<std::int64_t>(n - 1, k + std::max<std::int64_t>(4, (k + 1) / 2)));
    const int p = cfg.block_size > 0 ? cfg.block_size : auto_block(nev);
    block_used = p;
    for (int attempt = 0; attempt < 4; ++attempt) {
      // reruns keep the operator's factorization at sigma when the certificate's counts ran on
      // other objects
      if (f_stale && !factorize_at(OPF, sigma, scale, cfg.max_shift_retries, shift_retries, tm))
        HSG_THROW(HSG_SINGULAR, "A - sigma B is numerically singular at the working shift");
      f_stale = false;
      NearestRun run = run_krylov(op, P, sigma, nev, static_cast<int>(k), cfg, p, cfg.seed + attempt, tm);
      restarts += run.restarts;
      const std::size_t M = run.lam.size();
      if (static_cast<std::int64_t>(M) < k) {
        nev = static_cast<int>(std::min<std::int64_t>(n - 1, 2 * nev));
        warnings.push_back("fewer converged pairs than k; rerun with more");
        continue;
      }
      // window: midpoint of the first distance gap at or after the k-th pair
      std::vector<double> d(M);
      for (std::size_t i = 0; i < M; ++i) d[i] = std::fabs(run.lam[i] - sigma);
      long long q = -1;
      for (std::size_t i = static_cast<std::size_t>(k) - 1; i + 1 < M; ++i) {
        const double ctol = 1e-8 * (std::fabs(sigma) + d[i + 1] + scale * 1e-3);
        if (d[i + 1] - d[i] > ctol) { q = static_cast<long long>(i) + 1; break; }
      }
      bool passed = !certify;
      double R = 0.0, lo = 0.0, hi = 0.0;
      long long cnt = -1, moves = 0;
      if (certify) {
        if (q < 0) {
          nev = static_cast<int>(std::min<std::int64_t>(n - 1, nev + std::max<int>(4, nev / 2)));
          continue;  // no gap among the converged pairs yet
        }
        R = 0.5 * (d[q - 1] + d[q]);
        lo = sigma - R;
        hi = sigma + R;
        double lo_m = lo, hi_m = hi;
        long long nlo = -1, nhi = -1;
        if (batch) {
          long long moves_hi = 0;
          Timers t_lo, t_hi;
          GpuFactor& C0 = S.counter(0);
          GpuFactor& C1 = S.counter(1);
          auto f_hi = std::async(std::launch::async, [&] { return count_below(C1, hi_m, scale, +1.0, moves_hi, t_hi, true); });
          try {
            nlo = count_below(C0, lo_m, scale, -1.0, moves, t_lo, true);
          } catch (...) {
            f_hi.wait();
            throw;
          }
          nhi = f_hi.get();
          moves += moves_hi;
          tm.cert += std::max(t_lo.cert, t_hi.cert);
        } else {
          // plain path: the counts overwrite F's factorization, so a rerun refactorizes
          nlo = count_below(F, lo_m, scale, -1.0, moves, tm);
          nhi = count_below(F, hi_m, scale, +1.0, moves, tm);
          f_stale = &OPF == &F;
        }
        cnt = nhi - nlo;
        lo = lo_m;
        hi = hi_m;
        long long found = 0;
        for (std::size_t i = 0; i < M; ++i)
          if (run.lam[i] >= lo && run.lam[i] < hi) ++found;
        passed = cnt == found;
        cert.performed = true;
        cert.lower = lo;
        cert.upper = hi;
        cert.count_inertia = cnt;
        cert.count_found = found;
        cert.endpoint_moves += moves;
        cert.passed = passed;
        cert.method = "exact";
        if (!passed) {
          nev = static_cast<int>(std::min<std::int64_t>(n - 1, nev + (cnt - found) + 4));
          warnings.push_back("certificate found missing eigenvalues; deflated rerun with larger nev");
          continue;
        }
      }
      // select the k nearest
      std::vector<double> sel;
      std::vector<double> S(static_cast<std::size_t>(run.X.n / n) * k, 0.0);
      const int ncols = static_cast<int>(run.X.n / n);
      for (std::int64_t j = 0; j < k; ++j) {
        sel.push_back(run.lam[j]);
        S[static_cast<std::size_t>(run.col[j]) + static_cast<std::size_t>(j) * ncols] = 1.0;
      }
      DevBuf<double> Sd;
      Sd.upload(S, P.s);
      Xout.alloc(static_cast<std::size_t>(n) * k);
      gemm_tall(n, ncols, static_cast<int>(k), run.X.p, n, Sd.p, ncols, Xout.p, n, 1.0, 0.0, P.s);
      lam_out = sel;
      break;
    }
    HSG_REQUIRE(!lam_out.empty(), HSG_NOT_CONVERGED, "nearest target: no certified set of eigenpairs after reruns");
  } else {
    // ---------------------------------------------------------------- interval (slicing)
    double lo = win_lo, hi = win_hi;
    HSG_REQUIRE(std::isfinite(lo) && std::isfinite(hi) && lo < hi, HSG_INVALID_INPUT, "interval needs lower < upper");
    long long moves = 0, moves_hi = 0;
    const double mid0 = 0.5 * (lo + hi);
    double sigma_mid = mid0;
    bool mid_ok = false;
    long long nlo = -1, nhi = -1;
    if (batch) {
      // the window-end counts on two objects and, speculatively, the factorization at the window
      // midpoint (the slice shift when no split is needed, else the first cut) on F, all at once
      Timers t_lo, t_hi;
      GpuFactor& C0 = S.counter(0);
      GpuFactor& C1 = S.counter(1);
      auto f_lo = std::async(std::launch::async, [&] { return count_below(C0, lo, scale, -1.0, moves, t_lo, true); });
      auto f_hi = std::async(std::launch::async, [&] { return count_below(C1, hi, scale, +1.0, moves_hi, t_hi, true); });
      try {
        mid_ok = factorize_at(OPF, sigma_mid, scale, cfg.max_shift_retries, shift_retries, tm, true);
      } catch (...) {
        f_lo.wait();
        f_hi.wait();
        throw;
      }
      try {
        nlo = f_lo.get();
      } catch (...) {
        f_hi.wait();
        throw;
      }
      nhi = f_hi.get();
      moves += moves_hi;
      tm.cert += std::max(t_lo.cert, t_hi.cert);
    } else {
      nlo = count_below(F, lo, scale, -1.0, moves, tm);
      nhi = count_below(F, hi, scale, +1.0, moves, tm);
    }
    const long long N = nhi - nlo;
    cert.performed = true;
    cert.lower = lo;
    cert.upper = hi;
    cert.count_inertia = N;
    cert.method = "exact";
    cert.endpoint_moves = moves;
    std::vector<double> cuts{lo, hi};
    std::vector<long long> below{nlo, nhi};
    const long long target = cfg.slice_size > 0 ? cfg.slice_size : 96;
    bool spec_slice = mid_ok;  // OPF holds the factorization at sigma_mid
    if (N > target && mid_ok && sigma_mid > lo && sigma_mid < hi) {
      // the midpoint becomes the first cut; its count must be an FP64 one
      double cut = sigma_mid;
      const long long nm = single ? count_below(F, cut, scale, +1.0, cert.endpoint_moves, tm) : F.inertia().neg;
      cuts.insert(cuts.begin() + 1, cut);
      below.insert(below.begin() + 1, nm);
      spec_slice = false;
    }
    // split slices with too many eigenvalues at their midpoint (one count per cut)
    for (std::size_t i = 0; i + 1 < cuts.size();) {
      const long long c = below[i + 1] - below[i];
      if (c > target && cuts[i + 1] - cuts[i] > 1e-9 * (scale + std::fabs(cuts[i]))) {
        double mid = 0.5 * (cuts[i] + cuts[i + 1]);
        const long long nm = count_below(F, mid, scale, +1.0, cert.endpoint_moves, tm);
        cuts.insert(cuts.begin() + static_cast<std::ptrdiff_t>(i) + 1, mid);
        below.insert(below.begin() + static_cast<std::ptrdiff_t>(i) + 1, nm);
        continue;
      }
      ++i;
    }
    // one slice: its shift factorized on G (unless G holds it already), block Krylov-Schur of the
    // shift-invert operator with reruns for missing pairs, the slice's vectors; Q is the pencil with
    // G's stream, so slices on different objects run concurrently
    struct SliceOut {
      SliceRec rec{};
      std::vector<double> lam;
      DevBuf<double> X;
      int retries = 0;
      long long columns = 0, refine_steps = 0, refined_applies = 0;
      double worst_rel = 0.0, worst_omega = 0.0;
      Timers tm;
    };
    auto run_slice = [&](std::size_t i, GpuFactor& G, Problem Q, bool prefactored, double sigma0, bool shared) {
      PoolStreamScope scope(Q.s);
      SliceOut o;
      const long long c = below[i + 1] - below[i];
      o.rec = SliceRec{cuts[i], cuts[i + 1], 0.5 * (cuts[i] + cuts[i + 1]), c, 0, 0, 0, 0, 0, c == 0};
      if (c == 0) return o;
      double sigma = prefactored ? sigma0 : o.rec.sigma;
      if (!prefactored && !factorize_at(G, sigma, scale, cfg.max_shift_retries, o.retries, o.tm, shared))
        HSG_THROW(HSG_SINGULAR, "slice shift singular near " << o.rec.sigma);
      o.rec.sigma = sigma;
      ShiftInvertOp sop(Q, G);
      sop.set_refinement(sigma, tol_inner);
      int nev = static_cast<int>(std::min<std::int64_t>(n - 1, c + std::max<long long>(4, c / 4)));
      const int p = cfg.block_size > 0 ? cfg.block_size : auto_block(nev);
      for (int attempt = 0; attempt < 4; ++attempt) {
        // reruns reuse G's factorization at sigma
        const long long applies0 = sop.columns;
        NearestRun run = run_krylov(sop, Q, sigma, nev, static_cast<int>(c), cfg, p, cfg.seed + 17 * i + attempt, o.tm);
        o.rec.restarts += run.restarts;
        o.rec.op_applies += sop.columns - applies0;
        o.rec.nev = nev;
        std::vector<int> inside;
        for (std::size_t j = 0; j < run.lam.size(); ++j)
          if (run.lam[j] >= cuts[i] && run.lam[j] < cuts[i + 1]) inside.push_back(static_cast<int>(j));
        o.rec.count_found = static_cast<long long>(inside.size());
        if (o.rec.count_found != c && attempt + 1 < 4) {
          ++o.rec.reruns;
          nev = static_cast<int>(std::min<std::int64_t>(n - 1, nev + std::max<long long>(4, c - o.rec.count_found + 4)));
          continue;
        }
        o.rec.passed = o.rec.count_found == c;
        const int ncols = static_cast<int>(run.X.n / n);
        std::vector<double> Sel(static_cast<std::size_t>(ncols) * inside.size(), 0.0);
        for (std::size_t q = 0; q < inside.size(); ++q) {
          Sel[static_cast<std::size_t>(run.col[inside[q]]) + q * ncols] = 1.0;
          o.lam.push_back(run.lam[inside[q]]);
        }
        DevBuf<double> Sd;
        Sd.upload(Sel, Q.s);
        o.X.alloc(static_cast<std::size_t>(n) * std::max<std::size_t>(1, inside.size()));
        if (!inside.empty())
          gemm_tall(n, ncols, static_cast<int>(inside.size()), run.X.p, n, Sd.p, ncols, o.X.p, n, 1.0, 0.0, Q.s);
        cuda_check(cudaStreamSynchronize(Q.s), "slice vectors");
        break;
      }
      o.rec.op_applies = sop.columns;
      o.columns = sop.columns;
      o.refine_steps = sop.refine_steps;
      o.refined_applies = sop.refined_applies;
      o.worst_rel = sop.worst_rel;
      o.worst_omega = sop.worst_omega;
      return o;
    };
    const std::size_t nslices = cuts.size() - 1;
    std::vector<SliceOut> outs(nslices);
    std::size_t nonempty = 0;
    for (std::size_t i = 0; i < nslices; ++i) nonempty += below[i + 1] > below[i];
    auto view = [&](GpuFactor& G) {
      Problem Q = P;
      Q.s = G.stream();
      return Q;
    };
    if (spec_slice && nslices == 1) {
      outs[0] = run_slice(0, OPF, view(OPF), true, sigma_mid, false);  // factorized during the counts
    } else if (batch && nonempty > 1) {
      // the slices' shifts at once: up to kConcurrentSlices factorization objects sharing the
      // analysis (each with the shared cooperative plan), each taking the next slice when done
      const int lanes = static_cast<int>(std::min<std::size_t>(kConcurrentSlices, nonempty));
      std::atomic<std::size_t> next{0};
      std::vector<std::exception_ptr> errs(lanes);
      std::vector<std::future<void>> futs;
      // every lane's object exists before any lane runs: a new object copies F's analysis
      // (analyze_like), which a running factorization of F re-plans when pivots are delayed
      for (int lane = 0; lane < lanes; ++lane) S.slice_object(lane, single);
      for (int lane = 0; lane < lanes; ++lane) {
        GpuFactor& G = S.slice_object(lane, single);
        futs.push_back(std::async(std::launch::async, [&, lane] {
          GpuFactor& Gl = S.slice_object(lane, single);
          try {
            for (std::size_t i = next++; i < nslices; i = next++) outs[i] = run_slice(i, Gl, view(Gl), false, 0.0, true);
          } catch (...) {
            errs[lane] = std::current_exception();
            next = nslices;  // the other lanes stop after their current slice
          }
        }));
        (void)G;
      }
      for (auto& f : futs) f.wait();
      for (auto& e : errs)
        if (e) std::rethrow_exception(e);
    } else {
      for (std::size_t i = 0; i < nslices; ++i) outs[i] = run_slice(i, OPF, view(OPF), false, 0.0, false);
    }
    std::vector<std::vector<double>> vals;
    std::vector<DevBuf<double>> vecs;
    long long found_total = 0;
    bool all_pass = true;
    Timers slice_max;
    for (auto& o : outs) {
      slices.push_back(o.rec);
      shift_retries += o.retries;
      op.columns += o.columns;
      op.refine_steps += o.refine_steps;
      op.refined_applies += o.refined_applies;
      op.worst_rel = std::max(op.worst_rel, o.worst_rel);
      op.worst_omega = std::max(op.worst_omega, o.worst_omega);
      slice_max.factor += o.tm.factor;
      slice_max.iterate += o.tm.iterate;
      slice_max.kry_apply += o.tm.kry_apply;
      slice_max.kry_ortho += o.tm.kry_ortho;
      slice_max.kry_rr += o.tm.kry_rr;
      slice_max.kry_restart += o.tm.kry_restart;
      if (o.rec.count_inertia == 0) continue;
      block_used = std::max(block_used, cfg.block_size > 0 ? static_cast<int>(cfg.block_size)
                                                             : auto_block(static_cast<int>(o.rec.nev)));
      found_total += o.rec.count_found;
      all_pass = all_pass && o.rec.passed;
      restarts += static_cast<int>(o.rec.restarts);
      vals.push_back(o.lam);
      vecs.push_back(std::move(o.X));
    }
    // concurrent slices overlap: their summed phase times over the concurrency (a wall estimate)
    const double par = batch && nonempty > 1 ? static_cast<double>(std::min<std::size_t>(kConcurrentSlices, nonempty)) : 1.0;
    tm.factor += slice_max.factor / par;
    tm.iterate += slice_max.iterate / par;
    tm.kry_apply += slice_max.kry_apply / par;
    tm.kry_ortho += slice_max.kry_ortho / par;
    tm.kry_rr += slice_max.kry_rr / par;
    tm.kry_restart += slice_max.kry_restart / par;
    cert.count_found = found_total;
    cert.passed = all_pass && found_total == N;
    // gather ascending
    std::vector<std::pair<double, std::pair<int, int>>> all;
    for (std::size_t s = 0; s < vals.size(); ++s)
      for (std::size_t q = 0; q < vals[s].size(); ++q) all.push_back({vals[s][q], {static_cast<int>(s), static_cast<int>(q)}});
    std::stable_sort(all.begin(), all.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    Xout.alloc(static_cast<std::size_t>(n) * std::max<std::size_t>(1, all.size()));
    for (std::size_t j = 0; j < all.size(); ++j) {
      lam_out.push_back(all[j].first);
      const auto& src = vecs[all[j].second.first];
      copy_cols(n, 1, src.p + static_cast<std::int64_t>(all[j].second.second) * n, n, Xout.p + static_cast<std::int64_t>(j) * n, n, P.s);
    }
    sigma_used = slices.empty() ? 0.5 * (lo + hi) : slices.front().sigma;
  }
  (void)applies_before;
  if (one_end) {
    // keep the k smallest (ascending) or the k largest (descending) of the window's eigenpairs
    const std::size_t m_all = lam_out.size();
    const std::size_t keep = std::min<std::size_t>(m_all, static_cast<std::size_t>(cfg.k));
    DevBuf<double> Xk;
    Xk.alloc(static_cast<std::size_t>(n) * std::max<std::size_t>(1, keep));
    std::vector<double> lk;
    for (std::size_t j = 0; j < keep; ++j) {
      const std::size_t src = cfg.mode == 2 ? j : m_all - 1 - j;
      lk.push_back(lam_out[src]);
      copy_cols(n, 1, Xout.p + static_cast<std::int64_t>(src) * n, n, Xk.p + static_cast<std::int64_t>(j) * n, n, P.s);
    }
    lam_out = lk;
    Xout = std::move(Xk);
    if (cfg.mode == 2) cert.lower = -std::numeric_limits<double>::infinity();
    else cert.upper = std::numeric_limits<double>::infinity();
  }
  // verification
  const auto t_ver = Clock::now();
  const int m = static_cast<int>(lam_out.size());
  std::vector<PairMetrics> pm = pair_metrics(P, Xout.p, m, lam_out, cfg.tol);
  out.eigenvalues = lam_out;
  out.vectors.resize(static_cast<std::size_t>(n) * m);
  if (m > 0)
    cuda_check(cudaMemcpyAsync(out.vectors.data(), Xout.p, out.vectors.size() * sizeof(double), cudaMemcpyDeviceToHost, P.s), "vectors");
  cuda_check(cudaStreamSynchronize(P.s), "vectors");
  tm.verify += since(t_ver);
  bool all_ok = true;
  for (const auto& q : pm) all_ok = all_ok && q.accepted;
  for (const auto& q : cpm) all_ok = all_ok && q.accepted;
  if (ghiep) all_ok = all_ok && static_cast<std::int64_t>(m + cpm.size()) == cfg.k;
  const bool success = all_ok && (!cert.performed || cert.passed) && (cfg.mode != 1 || m == cert.count_inertia) &&
                       (!one_end || m == std::min<long long>(cfg.k, window_count));
  // report
  const hsg_estimate_t est = F.estimate();
  const hsg_inertia_t inr = F.inertia();
  Json j;
  j.open('{');
  j.kv("n", static_cast<long long>(n));
  j.kv("nnz_a", static_cast<long long>(a.rp[n]));
  j.kv("nnz_b", static_cast<long long>(b ? b->rp[n] : 0));
  j.kv("complex_scalars", false);
  j.kv("problem", std::string(ghiep ? "GHIEP" : problem));
  j.kv("norm2_a", P.normA);
  j.kv("norm2_b", P.normB);
  j.kv("scale", scale);
  j.kv("method", std::string(ghiep ? "shift_invert_krylov_schur" : "shift_invert_lanczos"));
  j.kv("candidate_source", std::string("iterative"));
  j.kv("sigma_requested", cfg.mode == 0 ? cfg.sigma : 0.5 * (win_lo + win_hi));
  j.kv("sigma_used", sigma_used);
  j.kv("shift_retries", shift_retries);
  j.kv("block_size", block_used);
  j.kv("restarts", restarts);
  j.kv("op_applies", static_cast<long long>(op.columns));
  const double total = since(t_start) + (include_setup ? S.setup_tm.setup + S.setup_tm.factor : 0.0);
  j.kv("time_total_s", total);
  j.kv("time_setup_s", tm.setup);
  j.kv("time_factor_s", tm.factor);
  j.kv("time_iterate_s", tm.iterate);
  j.kv("time_verify_s", tm.verify);
  j.kv("time_certificate_s", tm.cert);
  j.kv("batch_shifts", batch);
  j.key("iterate_split_s");
  j.open('{');
  j.kv("operator", tm.kry_apply);
  j.kv("orthonormalize", tm.kry_ortho);
  j.kv("rayleigh_ritz", tm.kry_rr);
  j.kv("restart", tm.kry_restart);
  j.close('}');
  j.key("factor_stats");
  j.open('{');
  j.kv("factor_entries", static_cast<long long>(est.factor_entries));
  j.kv("nnz_l", static_cast<long long>(est.nnz_l));
  j.kv("flops", est.flops);
  j.kv("supernodes", est.supernodes);
  j.kv("levels", est.levels);
  j.kv("max_front", est.max_front);
  j.kv("analyze_s", est.analyze_s);
  j.kv("ordering_s", est.ordering_s);
  j.kv("last_factorize_s", F.last_factor_seconds());
  j.kv("delayed_pivots", static_cast<long long>(inr.delayed_pivots));
  j.kv("two_by_two", static_cast<long long>(inr.two_by_two));
  j.close('}');
  {
    // F's work plus the FP32 operator object's (its factorizations and solves) on the mixed path
    GpuFactor::DeviceStats ds = F.device_stats();
    if (&OPF != &F) {
      const GpuFactor::DeviceStats& o = OPF.device_stats();
      ds.factorizations += o.factorizations;
      ds.factor_ms += o.factor_ms;
      ds.solves += o.solves;
      ds.solve_columns += o.solve_columns;
      ds.solve_ms += o.solve_ms;
    }
    j.key("device_timing");
    j.open('{');
    j.kv("factor_precision", std::string(single ? "single" : "double"));
    j.kv("factorizations", ds.factorizations);
    j.kv("factor_ms", ds.factor_ms);
    j.kv("flops_per_factorization", est.flops);
    j.kv("solves", ds.solves);
    j.kv("solve_columns", ds.solve_columns);
    j.kv("solve_ms", ds.solve_ms);
    j.kv("nnz_l", static_cast<long long>(est.nnz_l));
    j.kv("n", static_cast<long long>(n));
    j.kv("kernel_launches", static_cast<long long>(hsg_kernel_launches() - launches0));
    j.close('}');
  }
  j.key("precision");
  j.open('{');
  j.kv("requested", std::string(cfg.factor_precision == 1 || !fallback.empty() ? "single" : "double"));
  j.kv("used", std::string(single ? "single" : "double"));
  j.kv("fallback", fallback);
  j.key("refinement");
  j.open('{');
  j.kv("applies", op.refined_applies);
  j.kv("steps", op.refine_steps);
  j.kv("max_relative_residual", op.worst_rel);
  j.kv("max_backward_error", op.worst_omega);
  j.close('}');
  j.close('}');
  j.key("pairs");
  j.open('[');
  for (std::size_t i = 0; i < pm.size() + cpm.size(); ++i) {
    const PairMetrics& q = i < pm.size() ? pm[i] : cpm[i - pm.size()];
    j.open('{');
    j.kv("lambda_re", q.lambda);
    j.kv("lambda_im", i < pm.size() ? 0.0 : c_im[i - pm.size()]);
    j.kv("abs_residual", q.abs_res);
    j.kv("rel_residual", q.rel_res);
    j.kv("backward_error", q.eta);
    j.kv("accepted", q.accepted);
    j.close('}');
  }
  j.close(']');
  j.kv("zero_cluster_dim", zero_cluster_dim);
  j.key("certificate");
  j.open('{');
  j.kv("performed", cert.performed);
  j.kv("lower", cert.lower);
  j.kv("upper", cert.upper);
  j.kv("count_inertia", cert.count_inertia);
  j.kv("count_found", cert.count_found);
  j.kv("endpoint_moves", cert.endpoint_moves);
  j.kv("passed", cert.passed);
  j.kv("note", cert.note);
  j.kv("method", cert.method);
  j.kv("rigorous", cert.performed && cert.passed);
  j.kv("failure_probability", cert.performed && cert.passed ? 0.0 : 1.0);
  j.close('}');
  j.key("slices");
  j.open('[');
  for (const auto& r : slices) {
    j.open('{');
    j.kv("lower", r.lower);
    j.kv("upper", r.upper);
    j.kv("sigma", r.sigma);
    j.kv("which", std::string("largest_magnitude"));
    j.kv("count_inertia", r.count_inertia);
    j.kv("count_found", r.count_found);
    j.kv("nev", r.nev);
    j.kv("reruns", r.reruns);
    j.kv("restarts", r.restarts);
    j.kv("op_applies", r.op_applies);
    j.kv("passed", r.passed);
    j.close('}');
  }
  j.close(']');
  j.kv("success", success);
  j.key("warnings");
  j.open('[');
  for (const auto& w : warnings) j.val(w);
  j.close(']');
  j.close('}');
  out.report_json = j.os.str();
  return out;
}

SolveOutput solve_pencil(const CsrHost& a, const CsrHost* b, const hsg_solve_config_t& cfg) {
  Session s(a, b, cfg.device, cfg.seed);
  return s.solve(cfg, true);
}

}  // namespace hsg
