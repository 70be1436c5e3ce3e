// Block Krylov-Schur (thick-restart block Lanczos) with the basis resident on the GPU.
//
// Replaces hsolve's BlockThickRestartLanczos / lanczos_krylov_schur (src/eigen/block_lanczos.cpp:280-322,
// include/hsolve/eigen.hpp:144-146) for a B-self-adjoint operator such as OP = (A - sigma B)^{-1} B:
// full CGS2 re-orthogonalization in the B inner product and CholQR2 normalization of every new
// block (BlockOrthonormalizer, src/eigen/block_ortho.cpp:165,270), Rayleigh-Ritz on the projected
// matrix on the host, thick restart keeping the wanted Ritz vectors.
#pragma once

#include <complex>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "gpu_factor.hpp"

namespace hsg {

// Widest Krylov block: two 8-column chunks of one solve launch (a 16-column solve costs about 1.45x an
// 8-column one, whose sweeps are latency-bound).
constexpr int kMaxKrylovBlock = 16;

struct KrylovOperator {
  virtual ~KrylovOperator() = default;
  // y = OP x (device, n x p)
  virtual void apply(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p) = 0;
  // y = B x for the inner product; B = I when b_identity()
  virtual bool b_identity() const { return true; }
  virtual void bprod(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p) {
    (void)x; (void)ldx; (void)y; (void)ldy; (void)p;
  }
};

enum class Which { LargestMagnitude, LargestAlgebraic, SmallestAlgebraic };

struct KsOptions {
  int nev = 6;
  int ncv = 0;           // basis columns (0: automatic)
  int block = 1;         // block width p
  double tol = 1e-11;    // ||OP y - theta y||_B <= tol |theta|
  // The first nev_strict wanted pairs (by `which`) must meet tol; the others, which the callers
  // only use to place a window in a gap of the spectrum, meet max(tol, tol_buffer). 0: all nev.
  int nev_strict = 0;
  double tol_buffer = 1e-8;
  int max_restarts = 1000;
  std::uint64_t seed = 2026;
  Which which = Which::LargestMagnitude;
  bool ritz_vectors = true;
};

struct KsResult {
  std::vector<double> theta;   // the nev wanted Ritz values (ordered by `which`)
  std::vector<double> resid;   // their residual norms
  std::vector<char> converged;
  int nconv = 0;
  int restarts = 0;
  int applies = 0;             // operator applications (columns)
  int block_steps = 0;
  long long locked = 0;         // pairs decoupled by locking, summed over restarts
  std::vector<double> other_theta;  // the remaining Ritz values of the last basis (gap placement)
  std::vector<double> other_resid;
  DevBuf<double> X;            // n x nev Ritz vectors (B-orthonormal), if requested
  // host wall time (s) of the phases: operator applications, block orthonormalization,
  // Rayleigh-Ritz on the projected matrix, thick restarts
  double t_apply = 0.0, t_ortho = 0.0, t_rr = 0.0, t_restart = 0.0;
};

KsResult krylov_schur(KrylovOperator& op, std::int64_t n, const KsOptions& opt, cudaStream_t stream);

// Randomized exclusion check on the factorization already held at a shift sigma (hsolve's
// exclusion_check, include/hsolve/verify.hpp:18-80; src/verify/exclusion.cpp): with X the found
// eigenvectors of OP = (A - sigma B)^{-1} B (B positive definite), does the pencil have more
// eigenvalues than the found ones within `radius` of sigma? Weyl reduction with the coupling
// e = ||OP X - X H11||_B, then block Lanczos on the complement of span X from a Gaussian start
// block, s block steps fixed before the run from the failure bound (exclusion_block_steps); the
// check passes iff every Ritz value on the complement has |theta| < 1 / pass_radius.
struct ExclusionOptions {
  double radius = 0.0;           // r
  double pass_radius = 0.0;      // r' > r
  double delta = 1e-12;          // target failure probability
  int block = 4;                 // p
  std::uint64_t seed = 2026;
  double kappa = 1.0;            // >= cond(S B S) of the start block's covariance (1 for B = I)
  double rounding_margin = 1e-6;
  double coupling_bound = -1.0;  // >= 0: the caller's bound on e (no application of OP to X)
  int max_block_steps = 0;       // 0: no cap
  int max_krylov_vectors = 512;  // the plan's basis size above which the check is Inconclusive
};

enum class ExclusionStatus { Passed = 0, Detected = 1, Inconclusive = 2 };

struct ExclusionResult {
  ExclusionStatus status = ExclusionStatus::Inconclusive;
  double claim_threshold = 0.0;  // Theta_eff = (1/r - e)(1 - rounding_margin)
  double pass_threshold = 0.0;   // tau = 1/r'
  double coupling = 0.0;         // e
  double epsilon = 0.0;          // 1 - tau / Theta_eff
  double kappa = 1.0;
  std::int64_t deflated = 0, dimension = 0;
  std::int64_t found_inside = 0, certified_inside = 0;
  int block = 0, block_steps_planned = 0, block_steps = 0, krylov_vectors_planned = 0;
  bool exact = false, over_budget = false;
  double max_ritz = 0.0;
  double failure_probability = 1.0;
  std::int64_t new_count = 0, new_inside = 0;
  std::int64_t op_applications = 0;
  bool rigorous = true;                // false: kappa is the caller's estimate, not a proven bound
  std::vector<double> deflated_theta;  // eigenvalues of H11 by decreasing |mu|
  std::vector<double> ritz;            // Ritz values of the run, ascending
  double setup_s = 0.0, krylov_s = 0.0;
};

// P(pass and more than the found eigenvalues within r) for relative gap eps after s block steps of
// p columns on a complement of dimension N (verify.hpp:177-180); 1 for eps <= 0, 0 for N = 0.
double exclusion_failure_bound(double eps, std::int64_t s, std::int64_t N, std::int64_t p, double kappa,
                               bool complex_scalars);
// Smallest s >= 1 whose bound is <= delta, at most ceil(N / p) + 1 (a space covering the
// complement); -1 for eps <= 0 or delta outside (0, 1) (verify.hpp:182-188).
std::int64_t exclusion_block_steps(double eps, double delta, std::int64_t N, std::int64_t p, double kappa,
                                   bool complex_scalars);

// x: n x m device block (ld n), the found eigenvectors (any basis of their span). start_scale:
// optional positive diagonal S (device, n) of the Gaussian start columns S g (B^-1/2 for a diagonal
// B, which makes kappa = cond(S B S) = 1), or nullptr.
ExclusionResult exclusion_check(KrylovOperator& op, std::int64_t n, const double* x, int m,
                                const ExclusionOptions& opt, const double* start_scale, cudaStream_t stream);

}  // namespace hsg

namespace hsg {

// Block Krylov-Schur for a general (non-symmetric) operator, such as OP = (A - sigma B)^{-1} B with
// B indefinite (hsolve's krylov_schur_general, include/hsolve/eigen.hpp:254-256): Euclidean CGS2 /
// CholQR2 basis, projected matrix in complex Schur form (host), wanted Ritz values (largest |theta|)
// moved to the front, thick restart on the real basis of their invariant subspace.
struct GeneralKsResult {
  std::vector<std::complex<double>> theta;  // the wanted Ritz values, by decreasing |theta|
  std::vector<double> resid;
  std::vector<char> converged;
  std::vector<std::complex<double>> coef;   // m x wanted coefficients of the Ritz vectors in V
  int m = 0;
  DevBuf<double> V;                         // n x m basis (orthonormal)
  int restarts = 0, applies = 0;
  double t_apply = 0.0, t_ortho = 0.0, t_rr = 0.0, t_restart = 0.0;
};

GeneralKsResult krylov_schur_general(KrylovOperator& op, std::int64_t n, const KsOptions& opt, cudaStream_t stream);

}  // namespace hsg
