/* hsolve_b200 — C ABI of the B200 sparse symmetric-indefinite factorization and the
 * shift-invert kernels around it.
 *
 * The entry points replace hsolve's MUMPS-backed factorization boundary
 * (hs::SparseFactorization<T>, include/hsolve/factor.hpp:341-443 in hsolve) one for one; every
 * declaration below cites the member it replaces. Plain C types only: opaque handles, pointers,
 * sizes. Status codes are hs::Error::Code (include/hsolve/error.hpp:16-26) shifted by one, 0 = ok.
 *
 * Threading: one handle = one caller at a time (factor.hpp:337-340); distinct handles may be used
 * from different threads and run concurrently on the GPU (no process-wide lock, unlike MUMPS,
 * src/factor/mumps_api.hpp:23-63).
 */
#ifndef HSG_H_
#define HSG_H_

#include <stdint.h>

#if defined(__GNUC__)
#define HSG_API __attribute__((visibility("default")))
#else
#define HSG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status (hs::Error::Code + 1) */
enum {
  HSG_OK = 0,
  HSG_INVALID_INPUT = 1,         /* hs::Error::Code::InvalidInput */
  HSG_IO = 2,                    /* Io */
  HSG_NOT_HERMITIAN = 3,         /* NotHermitian */
  HSG_UNSUPPORTED = 4,           /* Unsupported */
  HSG_FACTORIZATION_FAILED = 5,  /* FactorizationFailed */
  HSG_SINGULAR = 6,              /* Singular */
  HSG_OUT_OF_MEMORY_BUDGET = 7,  /* OutOfMemoryBudget (device memory) */
  HSG_NOT_CONVERGED = 8,         /* NotConverged */
  HSG_INTERNAL = 9,              /* Internal (broken invariant, CUDA error) */
};

/* Text of a status code. */
HSG_API const char* hsg_status_string(int status);
/* Message of the last failing call on this thread (empty if none). */
HSG_API const char* hsg_last_error(void);
/* Kernel launches this library has issued in the process so far (instrumentation; no counterpart
 * in hsolve). */
HSG_API int64_t hsg_kernel_launches(void);

/* ------------------------------------------------------------------------ options, results */

/* hs::FactorOptions subset that the GPU backend honours (factor.hpp:248-292). */
typedef struct {
  int32_t precision;             /* 0 double, 1 single (FP32 factors; pair with refinement) */
  double null_pivot_tol;         /* CNTL(3) of double factorizations, default 1e-8 */
  double single_null_pivot_tol;  /* the same for single precision, default 1e-4 */
  double pivot_threshold;        /* threshold u of 1x1/2x2 pivot acceptance (CNTL(1)), 0.01 */
  int32_t device;                /* CUDA device ordinal */
  uint64_t ordering_seed;        /* seed of the nested dissection (OrderingOptions::seed) */
  int32_t scaling;               /* 1: symmetric equilibration at every factorization (ICNTL(8)=7) */
} hsg_options_t;

/* hs::Inertia (factor.hpp:295-300) plus the pivot statistics of FactorStats (:312-336). */
typedef struct {
  int64_t neg, zero, pos;
  int32_t valid;           /* 1: no null pivot, factors usable (solve works) */
  int64_t null_pivots;     /* INFOG(28) */
  int64_t delayed_pivots;  /* INFOG(13): columns moved to a parent front */
  int64_t two_by_two;      /* 2x2 pivots */
  int32_t replans;         /* re-plans of the front structure caused by delayed pivots */
} hsg_inertia_t;

/* hs::FactorEstimate (factor.hpp:303-310) + symbolic statistics. */
typedef struct {
  int64_t factor_entries;  /* panel storage (doubles) */
  int64_t nnz_l;           /* entries of L incl. D */
  double flops;            /* RINFOG(1) convention */
  double device_mb;        /* predicted device memory of a factorization (MB = 1e6 B) */
  int32_t supernodes;
  int32_t levels;
  int32_t max_front;
  double ordering_s;
  double analyze_s;
} hsg_estimate_t;

typedef struct hsg_factor hsg_factor;

HSG_API void hsg_default_options(hsg_options_t* opt);

/* -------------------------------------------------------------- factorization object (GPU) */

/* make_mumps_factorization<double> (factor.hpp:446-447). */
HSG_API int hsg_create(const hsg_options_t* opt, hsg_factor** out);
/* ~SparseFactorization */
HSG_API int hsg_destroy(hsg_factor* f);

/* SparseFactorization::analyze(pencil, alpha, beta) (factor.hpp:352-358) + set_pivot_order
 * (:425-432). The pencil K = alpha A + beta B is given by the upper triangles (row <= col) of
 * A and B as CSR (int64 row pointers, int32 columns, host pointers); B may be NULL (B = I).
 * pivot_order: NULL (nested dissection) or the 1-based pivot position of every variable
 * (MUMPS PERM_IN convention, factor.hpp:419-423). alpha, beta: representative values (unused
 * by the analysis itself, checked finite). */
HSG_API int hsg_analyze(hsg_factor* f, int64_t n, const int64_t* a_rowptr, const int32_t* a_col, const double* a_val,
                const int64_t* b_rowptr, const int32_t* b_col, const double* b_val, double alpha, double beta,
                const int32_t* pivot_order);

/* SparseFactorization::estimate() (factor.hpp:359-360). */
HSG_API int hsg_estimate(const hsg_factor* f, hsg_estimate_t* out);

/* SparseFactorization::factorize(alpha, beta) (factor.hpp:362-381): HSG_OK with out->valid = 0
 * when K is numerically singular (the object stays analysed). */
HSG_API int hsg_factorize(hsg_factor* f, double alpha, double beta, hsg_inertia_t* out);

/* SparseFactorization::count(alpha, beta) / InertiaCounter::count (factor.hpp:383-390,
 * :557-565): inertia of K without keeping usable factors. detection: null-pivot detection on/off.
 * The fronts of one tree level are factorized in a panel arena that the next level reuses, so the
 * count needs the largest level's panels instead of the whole factor; the handle holds no usable
 * factorization afterwards (hsg_solve fails until the next hsg_factorize). */
HSG_API int hsg_count(hsg_factor* f, double alpha, double beta, int32_t detection, hsg_inertia_t* out);

/* SparseFactorization::solve(b, nrhs, ldb) (factor.hpp:394-398): K X = B in place, column-major,
 * ldb >= n. b_on_device: 0 host memory, 1 device memory of the handle's device.
 * Stream contract of a device b: the solve runs on the handle's own (non-blocking) stream, ordered
 * after the work already queued on the legacy default stream (stream 0) when the call is made; a
 * caller that writes b on any other stream must complete that work (cudaStreamSynchronize, or an
 * event it waits on) before the call. The call returns after the solve has finished on the GPU. */
HSG_API int hsg_solve(hsg_factor* f, double* b, int64_t nrhs, int64_t ldb, int32_t b_on_device);

/* The same solve as hsg_solve with b in device memory, for callers that must not allocate device
 * memory: a process whose device memory is already fully claimed by a pooling allocator (where
 * cudaMalloc would fail), or a serving loop that cannot afford the device-wide synchronisation
 * that cudaFree implies. This call allocates nothing: its work space is one fixed array compiled
 * into the library, HSG_SOLVE_STATIC_SCRATCH_BYTES (16 MiB) on every device that loads the library,
 * held until the process exits. It needs 8 * (n * nrhs + c * min(nrhs, 16)) bytes, where c is the
 * total contribution-block row count of the factorization; a larger request returns
 * HSG_INVALID_INPUT with the sizes in hsg_last_error(), and the caller should split its right-hand
 * sides or use hsg_solve. The first call on a device looks up the array's device address (make
 * that first call before any stream capture). All calls on a device share the one array, so two
 * calls whose GPU work overlaps (from different host threads) race and give wrong results;
 * calls from one thread are safe because each call waits for its GPU work before returning.
 * b_device must be device (or managed) memory of the handle's device (HSG_INVALID_INPUT otherwise),
 * and the stream contract of a device b in hsg_solve applies: work on streams other than the legacy
 * default stream that writes b_device must be complete before the call.
 * No counterpart in hsolve. */
#define HSG_SOLVE_STATIC_SCRATCH_BYTES (16u << 20)
HSG_API int hsg_solve_static(hsg_factor* f, double* b_device, int64_t nrhs, int64_t ldb);

/* SparseFactorization::inertia() (factor.hpp:400-406). */
HSG_API int hsg_inertia(const hsg_factor* f, hsg_inertia_t* out);

/* SparseFactorization::release_factors() (factor.hpp:420-428): 1 in *released if anything was freed. */
HSG_API int hsg_release(hsg_factor* f, int32_t* released);

/* SparseFactorization::set_null_pivot_detection(on) (factor.hpp:430-438). */
HSG_API int hsg_set_null_pivot_detection(hsg_factor* f, int32_t on);

/* SparseFactorization::pivot_order() (factor.hpp:413-418): n entries, 1-based positions. */
HSG_API int hsg_pivot_order(const hsg_factor* f, int32_t* out);

/* SparseFactorization::order() (factor.hpp:441-442). */
HSG_API int64_t hsg_order(const hsg_factor* f);

/* Empties the process-wide cache of nested-dissection analyses (keyed by sparsity pattern), so that
 * the next analysis of any pattern runs the ordering and the symbolic factorization again; handles
 * that already hold an analysis keep it (instrumentation for cold-call timing; no counterpart in
 * hsolve, whose every hs::solve call analyses afresh). */
HSG_API int hsg_clear_analysis_cache(void);

/* Measured FP64 FMA throughput of the device (TFLOP/s), the denominator of the factorization's
 * roofline (instrumentation; no counterpart in hsolve). */
HSG_API int hsg_fp64_peak_probe(int32_t device, double* tflops);

/* ------------------------------------------------------- sparse kernels on device pointers */
/* The CSR arguments below hold FULL matrices (both triangles; int64 row pointers, int32 columns,
 * double values) in device memory of the current CUDA device, as do x, y and r (column-major).
 * Each call runs on the legacy default stream (ordered after the caller's work queued there) and
 * returns when its GPU work has finished. */

/* hs::spmm (include/hsolve/sparse.hpp:140-147): Y = alpha A X + beta Y for p columns; beta == 0
 * never reads Y. */
HSG_API int hsg_spmm(int64_t n, const int64_t* a_rowptr, const int32_t* a_col, const double* a_val,
                     const double* x, int64_t ldx, double* y, int64_t ldy, int64_t p, double alpha, double beta);

/* hs::shifted_residual (include/hsolve/sparse.hpp:149-174): R = B X - (A Y - sigma B Y) for p
 * columns (b_rowptr == NULL: B = I), computed as B (X + sigma Y) - A Y in one sweep over the rows,
 * and, when backward_error is not NULL (device, p doubles), every column's componentwise backward
 * error omega_k = max_i |r_ik| / (|B| |x_k + sigma y_k| + |A| |y_k|)_i with 0/0 = 0, r/0 = inf and
 * inf for a row whose r or s is not finite. r may be NULL (backward errors only). */
HSG_API int hsg_shifted_residual(int64_t n, const int64_t* a_rowptr, const int32_t* a_col, const double* a_val,
                                 const int64_t* b_rowptr, const int32_t* b_col, const double* b_val, double sigma,
                                 const double* x, int64_t ldx, const double* y, int64_t ldy, double* r, int64_t ldr,
                                 int64_t p, double* backward_error);

/* ----------------------------------------------------------------- host-only (no GPU needed) */

/* hs::compute_ordering (factor.hpp:630-633): nested-dissection pivot order of the symmetric
 * pattern given by its upper CSR; out: 1-based pivot position of every variable. */
HSG_API int hsg_compute_ordering(int64_t n, const int64_t* rowptr, const int32_t* col, uint64_t seed, int32_t* out);

/* Symbolic statistics of the analysis a handle would make (factor entries, flops, fronts). */
HSG_API int hsg_symbolic_stats(int64_t n, const int64_t* rowptr, const int32_t* col, const int32_t* pivot_order,
                       int32_t amalgamate, hsg_estimate_t* out);

/* Input checks of hsolve.solve on a real CSR matrix (python/hsolve/__init__.py:347-419 validates the
 * same properties), on host threads: flags[0] = 1 when every row's columns are strictly increasing
 * (sorted, no duplicates), flags[1] = 1 when an explicit zero is stored, flags[2] = 1 when the
 * pattern is structurally symmetric; counts[0] / counts[1] = entries strictly above / below the
 * diagonal; *defect = ||M - M^T||_F / ||M||_F (valid when flags[0] and flags[2]); sym (nullable, nnz
 * entries) receives (M + M^T) / 2 on M's pattern when the defect is positive. */
HSG_API int hsg_csr_inspect(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val, int32_t* flags,
                            int64_t* counts, double* defect, double* sym);

#ifdef __cplusplus
}
#endif

#endif /* HSG_H_ */
