// GPU sparse LDL^T object behind the C ABI: the B200 replacement of hsolve's MumpsFactorization
// (src/factor/mumps_factorization.{hpp,cpp}; contract hs::SparseFactorization<T>,
// include/hsolve/factor.hpp:341-443).
#pragma once

#include <cstdint>
#include <memory>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "common.hpp"
#include "device.cuh"
#include "hsg.h"
#include "symbolic.hpp"

namespace hsg {

void cuda_check(cudaError_t e, const char* what);

// Device memory through a per-device caching pool: blocks are rounded up to size classes of 1/8
// octave, returned to the pool on release and reused by later allocations of the same class, so
// the solves of a session do not call cudaMalloc / cudaFree (which synchronise the device) after
// their first call. A failed cudaMalloc releases the cached blocks of the device and retries.
void* pool_alloc(std::size_t bytes, std::size_t* cap, int* device);
void pool_free(void* p, std::size_t cap, int device);
// Releases every cached block of every device (the library's memory in use is not touched).
void pool_trim();

// The stream on which the calling thread queues the library's work while the scope is open. A
// block released inside a scope gets an event recorded on that stream, and a later allocation of
// the block (from any thread) waits for it: stream-ordered on its own scope's stream, or on the
// host without a scope. A block released outside every scope must be idle already (its stream
// synchronized). Scopes nest; the innermost one counts.
class PoolStreamScope {
 public:
  explicit PoolStreamScope(cudaStream_t s);
  ~PoolStreamScope();
  PoolStreamScope(const PoolStreamScope&) = delete;
  PoolStreamScope& operator=(const PoolStreamScope&) = delete;

 private:
  cudaStream_t prev_;
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  std::size_t n = 0;
  std::size_t cap = 0;  // bytes of the pooled block
  int dev = -1;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), cap(o.cap), dev(o.dev) { o.p = nullptr; o.n = 0; o.cap = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; cap = o.cap; dev = o.dev;
      o.p = nullptr; o.n = 0; o.cap = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) pool_free(p, cap, dev);
    p = nullptr;
    n = 0;
    cap = 0;
  }
  void alloc(std::size_t count) {
    if (count <= n && p) return;
    release();
    if (count == 0) return;
    p = static_cast<T*>(pool_alloc(count * sizeof(T), &cap, &dev));
    n = count;
  }
  void upload(const std::vector<T>& h, cudaStream_t s) {
    alloc(h.size());
    if (!h.empty()) cuda_check(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
  }
};

// Launch plan of one tree level of the fronts (built with the FrontPlan).
struct LevelPlan {
  std::int64_t zero_off = 0; int zero_n = 0; int zero_chunks = 1;
  std::int64_t s32_off = 0; int s32_n = 0;
  std::int64_t s64_off = 0; int s64_n = 0;
  std::int64_t app_off = 0; int app_n = 0;
  bool coop = false;                 // large fronts: one cooperative launch, CTAs split by work
  std::int64_t cta_off = 0; int coop_ctas = 0; int done_slot = 0;
  std::int64_t all_off = 0; int all_n = 0; int maxm = 0;
  std::vector<std::pair<std::int64_t, int>> ea;  // (offset into items, count) per child rank
  // solve sweeps: the level's CTA tasks (FrontPlan::tasks) of the forward and the backward sweep,
  // planned for launches of c + 1 column chunks; coop: some front has several CTAs (cooperative)
  std::int64_t fwd_task_off[2] = {0, 0}; int fwd_ctas[2] = {0, 0}; bool fwd_coop[2] = {false, false};
  std::int64_t bwd_task_off[2] = {0, 0}; int bwd_ctas[2] = {0, 0}; bool bwd_coop[2] = {false, false};
  bool tiny = false;                 // every front has m <= kTinyRows, k <= 32: one warp per front
  bool coop_shared = false;          // the level also fits the shared budget's co-resident grid
  std::int64_t cta_off_shared = 0; int coop_ctas_shared = 0;  // cooperative plan of the shared budget
  std::int64_t ent_off = 0, ent_n = 0;  // inertia-only counts: this level's entries in FrontPlan::ent_idx
  std::int64_t arena_used = 0;       // ... and its panels' extent in the arena
};

// The read-only front structure of one analysis on one device: level lists, cooperative CTA plans,
// scatter destinations and the solve tables, with the sizes of the per-object work arrays. Built
// once per analysis and shared, immutable, by every factorization object of that analysis
// (analyze_like), and kept beside the process-wide analysis cache, so that a new object on a known
// pattern builds and uploads no plan. A delayed-pivot re-plan gives its object a plan of its own.
struct FrontPlan {
  int device = -1;
  std::vector<LevelPlan> levels;
  std::int64_t vec_total = 0;      // contribution-vector rows of a solve
  std::int64_t arena_entries = 1;  // inertia-only counts: the largest level's panels
  std::int64_t scratch_max = 0, work_max = 0, w_total = 0;
  int ncoop = 0, nsbl = 0, ntiles = 0;
  std::int32_t hcnt_total = 0;     // backward helper counters (one per 32-column chunk of every front)
  DevBuf<std::int32_t> row, col;   // the union pattern's entries (row, column)
  DevBuf<std::int64_t> dest;       // their positions in the factor storage
  DevBuf<SnDev> sn;
  DevBuf<std::int32_t> lists, rmap, rows, child_ptr, children, iperm;
  DevBuf<int2> items;              // extend-add items by child rank
  // inertia-only counts: fronts with arena offsets, entries by level and their arena destinations
  DevBuf<SnDev> sn_cnt;
  DevBuf<std::int64_t> ent_idx, dest_cnt;
  DevBuf<SolveTask> tasks;         // solve sweep CTAs, level by level (forward and backward lists)
  DevBuf<std::int64_t> dpos;       // per pivot: panel index of its diagonal entry
  DevBuf<std::int32_t> pfirst;     // per pivot: first column of its front
  DevBuf<std::int32_t> cptr;       // children's contributions per front position
  DevBuf<ContribEntry> cent;
  DevBuf<int2> sbl;                // super-blocks of the solve operators
  DevBuf<int4> tiles;
};

class GpuFactor {
 public:
  explicit GpuFactor(const hsg_options_t& opt);
  ~GpuFactor();

  void analyze(std::int64_t n, const std::int64_t* a_rp, const std::int32_t* a_ci, const double* a_v,
               const std::int64_t* b_rp, const std::int32_t* b_ci, const double* b_v, const std::int32_t* order);
  // shared: use the cooperative plan sized for a third of the device, so that up to three
  // factorizations (of different shifts, on different objects) can run at once
  hsg_inertia_t factorize(double alpha, double beta, bool detection, bool shared = false);
  // Inertia only (SparseFactorization::count / InertiaCounter::count): the same pivoting and D, but
  // no factor is kept - the fronts of one tree level are factorized in a panel arena that the next
  // level overwrites (max over levels of the level's panel sizes instead of all of them), and no
  // solve operator is built. The handle holds no usable factorization afterwards.
  hsg_inertia_t count(double alpha, double beta, bool detection, bool shared = false);
  // The analysis of `src` (pattern, values of A and B, symbolic analysis) without recomputing it.
  void analyze_like(const GpuFactor& src);
  void solve(double* b, std::int64_t nrhs, std::int64_t ldb, bool on_device);
  // Doubles of work space that solve_with_scratch needs for nrhs right-hand sides: n x nrhs for the
  // permuted, scaled right-hand sides and (contribution rows) x min(nrhs, 8) for the update vectors.
  std::size_t solve_scratch_doubles(std::int64_t nrhs) const;
  // The solve of a device-resident b (column-major, leading dimension ldb) with its work space in
  // the caller's `scratch` (`cap` doubles, on this factorization's device). Allocates no device
  // memory; every scratch entry is written before it is read, so nothing needs to start at zero.
  void solve_with_scratch(double* b_dev, std::int64_t nrhs, std::int64_t ldb, double* scratch, std::size_t cap);
  // Orders the handle's stream (a non-blocking stream) after all work queued so far on the legacy
  // default stream, where a caller's own copies into a device right-hand side usually run; work on
  // the caller's other streams must be complete before a device solve is called.
  void order_after_legacy_stream();
  // Orders the handle's stream after the work queued so far on `other` (an event, no host wait).
  void order_after(cudaStream_t other);
  void release();
  hsg_estimate_t estimate() const;
  const hsg_inertia_t& inertia() const { return inertia_; }
  std::int64_t order() const { return n_; }
  void pivot_order(std::int32_t* out) const;
  void set_detection(bool on) { detection_ = on; }
  bool detection() const { return detection_; }
  bool analysed() const { return analysed_; }
  cudaStream_t stream() const { return stream_; }
  int device() const { return opt_.device; }
  // Device copies of the pencil (upper CSR of the union pattern), for SpMV users.
  const Symbolic& symbolic() const { return sym_; }
  double last_factor_seconds() const { return last_factor_s_; }
  double last_solve_seconds() const { return last_solve_s_; }
  // Device time (CUDA events on the handle's stream) and counts since the last reset.
  struct DeviceStats {
    long long factorizations = 0;  // numeric passes, re-plans included
    double factor_ms = 0.0;
    long long solves = 0;
    long long solve_columns = 0;
    double solve_ms = 0.0;
  };
  const DeviceStats& device_stats() const { return dstats_; }
  void reset_device_stats() { dstats_ = DeviceStats{}; }

 private:
  // plan_ = a new plan of sym_ (make_plan) and the per-object work arrays sized for it
  void build_plan();
  std::shared_ptr<FrontPlan> make_plan();
  void alloc_work();
  hsg_inertia_t run_factorization(double alpha, double beta, bool detection, bool shared, bool count_only);
  void run_numeric(double alpha, double beta, bool detection, bool count_only);
  template <class R>
  void run_numeric_t(double alpha, double beta, bool detection, bool count_only);
  // forward, diagonal and backward sweeps of nr right-hand sides gathered in xwork (n x nr); with
  // graph, the launches are captured once per (xwork, vec, nr) in a CUDA graph and replayed
  void run_sweeps(double* xwork, double* vec, int nr, bool graph);
  void clear_sweep_graphs();
  template <class F>
  void run_sweeps_t(double* xwork, double* vec, int nr);
  template <class F>
  void build_solve_operator_t();
  template <class R>
  R* panels_of();
  template <class R>
  R* cb_of();
  template <class R>
  R* w_of();

 public:
  // FP32 factors (hsg_options_t.precision == 1): the operator factorization of the mixed-precision
  // path, solved with FP64 right-hand sides and refined by the caller against the FP64 pencil.
  bool single() const { return opt_.precision == 1; }
  // Entries of the factor storage (panels + solve operators) times the element size.
  std::size_t factor_bytes() const;

 private:

  hsg_options_t opt_;
  cudaStream_t stream_ = nullptr;
  bool analysed_ = false;
  bool factored_ = false;
  bool detection_ = true;
  std::int64_t n_ = 0, nnz_ = 0;
  std::vector<std::int64_t> rp_;
  std::vector<std::int32_t> ci_, row_;
  Symbolic sym_;
  std::shared_ptr<const FrontPlan> plan_;
  // the cached analysis sym_ was copied from (null: own analysis, or re-planned since)
  std::shared_ptr<const Symbolic> sym_origin_;
  hsg_inertia_t inertia_{};
  double last_factor_s_ = 0.0, last_solve_s_ = 0.0;
  DeviceStats dstats_;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr, ev_in_ = nullptr;

  DevBuf<std::int32_t> d_pidx_, d_failed_;
  DevBuf<double> d_a_, d_b_, d_scale_, d_panels_, d_cb_, d_scratch_, d_vec_, d_xwork_, d_btmp_;
  DevBuf<float> d_panels_f_, d_cb_f_, d_w_f_;  // the same, for FP32 factors
  DevBuf<double> d_arena_;  // inertia-only counts: the panels of one level
  DevBuf<float> d_arena_f_;
  DevBuf<unsigned long long> d_r_;
  DevBuf<signed char> d_piv_;
  DevBuf<FactorCounters> d_cnt_;
  DevBuf<int> d_level_done_;
  DevBuf<double> d_work_;
  // super-block solve operators of every front (built at the first solve after a factorization)
  DevBuf<double> d_w_;
  DevBuf<int> d_err_;  // set by a solve sweep whose bounded wait ran out
  DevBuf<int> d_sweep_cnt_;       // per front: forward and backward publication counters, backward arrivals
  bool w_ready_ = false;
  void build_solve_operator();
  // captured sweep sequences (valid until the plan or the work buffers change)
  struct SweepGraph {
    double* xwork;
    double* vec;
    int nr;
    long long launches;
    cudaGraphExec_t exec;
  };
  std::vector<SweepGraph> graphs_;
  bool graphs_ok_ = true;  // false once a capture failed: launch directly
  // held while stream_ is capturing: another object's analyze_like synchronizes stream_, which is
  // not permitted during a capture
  mutable std::mutex capture_mu_;
  int solve_coop_max_ = 0;
  int coop_max_ = 0;
  bool shared_ = false;
  bool cached_analysis_ = false;  // the analysis came from (and teaches) the pattern cache
  static constexpr int kSharedParts = 3;
};

}  // namespace hsg
