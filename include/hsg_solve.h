/* hsolve_b200 — C ABI of the whole shift-invert eigensolve (hs::solve, hsolve
 * include/hsolve/solver.hpp:545-547), the call behind hsolve.solve(A, B, sigma, k | interval).
 *
 * A and B are given in full storage (both triangles) as CSR with int64 row pointers and int32
 * columns (host pointers); B may be NULL (standard problem, B = I). The configuration mirrors the
 * SolverConfig keys this path honours (solver.hpp:71-235); the report is the SolveReport JSON
 * document (solver.hpp:457-516, docs/FORMATS.md section 3 in hsolve) with the keys this path fills.
 */
#ifndef HSG_SOLVE_H_
#define HSG_SOLVE_H_

#include <stdint.h>

#include "hsg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t mode;               /* hs::TargetMode: 0 nearest, 1 interval, 2 smallest, 3 largest */
  double sigma;               /* Target::sigma (nearest) */
  int64_t k;                  /* Target::k */
  double lower, upper;        /* Target::lower / upper (interval) */
  int32_t problem;            /* hs::ProblemType: 0 auto, 1 standard, 2 generalized definite, 3 indefinite */
  double tol;                 /* backward-error acceptance, default 1e-10 */
  double inner_tol_factor;    /* Krylov tolerance = tol * inner_tol_factor, default 0.1 */
  int64_t ncv;                /* Krylov basis columns, 0 = auto */
  int32_t block_size;         /* Krylov block width p, 0 = auto */
  int64_t slice_size;         /* eigenvalues per spectrum slice, 0 = auto */
  int32_t max_restarts;       /* default 1000 */
  uint64_t seed;              /* Krylov start vectors, default 2026 */
  int32_t certificate;        /* hs::CertificateMode: 0 exact, 3 off */
  int32_t max_shift_retries;  /* default 5 */
  int32_t factor_precision;   /* hs::FactorPrecision: 0 double, 1 single (FP32 factors + FP64 refinement) */
  int32_t device;             /* CUDA device */
  int32_t verbose;
  int32_t batch_shifts;       /* 1 (default): independent shifts of one solve (window-end counts, the
                                 slice factorization) run at once on several factorization objects;
                                 0: one after another on one object (the plain path). No counterpart
                                 in hsolve. */
  double complex_tol;         /* GHIEP: a pair is complex only if |Im lambda| > complex_tol *
                                 max(|lambda|, scale) and its real projection fails tol while the
                                 complex pair does at least as well; default 1e-8 */
  double zero_filter_tol;     /* GHIEP: < 0 (default) off; else eigenvalues with |lambda| <=
                                 zero_filter_tol * scale are zero modes, left out of the selection */
} hsg_solve_config_t;

typedef struct hsg_solution hsg_solution;

/* The SolverConfig defaults (solver.hpp:71-235). */
HSG_API void hsg_default_solve_config(hsg_solve_config_t* cfg);

/* hs::solve<double>(A, B, cfg): eigenpairs ordered by the target; HSG_OK also when the run did
 * not meet tol (report "success": false), an error status otherwise (hs::Error::Code + 1). */
HSG_API int hsg_eigsolve(int64_t n, const int64_t* a_rowptr, const int32_t* a_col, const double* a_val,
                         const int64_t* b_rowptr, const int32_t* b_col, const double* b_val,
                         const hsg_solve_config_t* cfg, hsg_solution** out);

/* A pencil resident on the GPU with its analysis and norm bounds computed once (the serving path:
 * symbolic analyses and device copies reused across targets and shifts). No counterpart type in
 * hsolve; hsg_session_solve(s, cfg) returns what hs::solve(A, B, cfg) returns for the session's
 * pencil. A session is used by one caller at a time. */
typedef struct hsg_session hsg_session;
HSG_API int hsg_session_create(int64_t n, const int64_t* a_rowptr, const int32_t* a_col, const double* a_val,
                               const int64_t* b_rowptr, const int32_t* b_col, const double* b_val, int32_t device,
                               uint64_t seed, hsg_session** out);
HSG_API int hsg_session_solve(hsg_session* s, const hsg_solve_config_t* cfg, hsg_solution** out);
HSG_API void hsg_session_free(hsg_session* s);
/* The analysis of the session's pencil: factor entries, nnz(L), flops and device memory of one
 * factorization object (a session holds one, or three while it batches shifts). */
HSG_API int hsg_session_estimate(const hsg_session* s, hsg_estimate_t* out);

/* Solution<double>::eigenvalues.size() and n. */
HSG_API int hsg_solution_sizes(const hsg_solution* s, int64_t* n, int64_t* m);
/* Copies eigenvalues (m) and eigenvectors (n x m column-major; NULL to skip). */
HSG_API int hsg_solution_copy(const hsg_solution* s, double* eigenvalues, double* eigenvectors);
/* Solution<double>::complex_eigenvalues.size(): the genuinely complex pairs of a GHIEP (usually 0). */
HSG_API int hsg_solution_complex_count(const hsg_solution* s, int64_t* mc);
/* Copies complex_eigenvalues (mc, as re, im pairs) and complex_eigenvectors (n x mc column-major,
 * every entry as re, im; NULL to skip), the layout of C99 double complex / std::complex<double>. */
HSG_API int hsg_solution_complex_copy(const hsg_solution* s, double* eigenvalues, double* eigenvectors);
/* SolveReport::to_json(). Valid until hsg_solution_free. */
HSG_API const char* hsg_solution_report(const hsg_solution* s);
HSG_API void hsg_solution_free(hsg_solution* s);

/* Randomized exclusion certificate (hsolve's hs::exclusion_check, include/hsolve/verify.hpp:18-80,
 * 110-175): on the factorization of K = A - sigma B (B positive definite) and the found eigenvectors
 * X (host, n x m column-major, ld >= n), a block Lanczos run on the complement of span X from a
 * Gaussian start decides, with failure probability at most `delta`, whether the pencil has more
 * eigenvalues than the found ones within `radius` of sigma: status 0 passed (no Ritz value on the
 * complement with |theta| >= 1 / pass_radius), 1 detected, 2 inconclusive (the gap between radius
 * and pass_radius is too small for the coupling of X, or the plan exceeds max_krylov_vectors). The
 * session factorizes at sigma (moved slightly, like the solver's shifts, when K is singular there;
 * the shift used is returned). No counterpart in hsolve's C++ API beyond exclusion_check itself. */
typedef struct {
  double sigma, radius, pass_radius;
  double delta;            /* target failure probability, in (0, 1); default 1e-12 */
  int32_t block_size;      /* start columns p (1..16); default 4 */
  int32_t max_block_steps; /* 0: no cap */
  int32_t max_krylov_vectors; /* default 512 */
  int32_t pad;
  uint64_t seed;           /* default 2026 */
  double kappa;            /* general B only: the caller's bound on cond(B); default 1 */
  double rounding_margin;  /* default 1e-6 */
} hsg_exclusion_options_t;

typedef struct {
  int32_t status;          /* 0 passed, 1 detected, 2 inconclusive */
  int32_t exact;           /* the Krylov space covered the complement (failure probability 0) */
  int32_t over_budget, rigorous;
  double sigma;            /* the shift factorized */
  double claim_threshold, pass_threshold, coupling, epsilon, kappa;
  int64_t deflated, dimension, found_inside, certified_inside;
  int64_t block_size, block_steps_planned, block_steps, krylov_vectors_planned;
  double max_ritz, failure_probability;
  int64_t new_count, new_inside, op_applications;
  double setup_s, krylov_s;
} hsg_exclusion_result_t;

HSG_API void hsg_default_exclusion_options(hsg_exclusion_options_t* opt);
HSG_API int hsg_session_exclusion_check(hsg_session* s, const double* x, int64_t m, int64_t ldx,
                                        const hsg_exclusion_options_t* opt, hsg_exclusion_result_t* out);
/* The failure bound delta(s) and the planned block steps (verify.hpp:177-188). */
HSG_API double hsg_exclusion_failure_bound(double epsilon, int64_t block_steps, int64_t dimension,
                                           int64_t block_size, double kappa, int32_t complex_scalars);
HSG_API int64_t hsg_exclusion_block_steps(double epsilon, double delta, int64_t dimension, int64_t block_size,
                                          double kappa, int32_t complex_scalars);

#ifdef __cplusplus
}
#endif

#endif /* HSG_SOLVE_H_ */
