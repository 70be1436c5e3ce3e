// Device-side types and helpers shared by the factorization and solve kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hsg {

// One front (supernode) as the kernels see it.
struct SnDev {
  std::int32_t first;     // first pivot position (global index of its first column)
  std::int32_t k;         // fully-summed columns
  std::int32_t m;         // rows of the front
  std::int32_t parent;    // -1: root
  std::int64_t panel_off; // m x k panel, ld m, in the factor storage
  std::int64_t cb_off;    // (m-k)^2 contribution block, ld m-k, in the CB arena (-1: none)
  std::int64_t rows_off;  // its rows in the row array
  std::int64_t rmap_off;  // its CB rows' positions in the parent's rows
  std::int64_t vec_off;   // contribution vector (m-k entries per rhs) in the solve arena
  std::int64_t scratch_off;  // pivoting scratch of the panel kernel (doubles)
  std::int64_t w_off;        // super-block solve operator (m x k, ld m) in the operator storage
  std::int64_t cptr_off;     // children's contributions per front position (m + 1 offsets)
};

// One child contribution to a front position: entry a of the child's contribution vector
// (mc rows per right-hand side, at vec_off * nrhs in the solve arena).
struct ContribEntry {
  std::int64_t vec_off;
  std::int32_t a;
  std::int32_t mc;
};

// One CTA of a solve sweep level: front s, the CTA's rank among the front's CTAs, and the offset of
// the front's work vectors. Backward, the contribution-row tiles of every 32-column chunk may be cut
// into `parts` parts: part 0 is the chunk owner's, parts 1.. belong to helper CTAs (ranks nr + h,
// h = chunk + nch (part - 1)) that publish partial sums through the chunk's counter.
struct SolveTask {
  std::int32_t s;
  std::int32_t rank;   // < nr: a chunk owner; nr + h: backward helper h
  std::int32_t nr;     // owner CTAs of the front
  std::int32_t parts;  // backward: parts of each chunk's contribution-row tiles (1: no helpers)
  std::int32_t hcnt;   // backward: first of the front's per-chunk helper counters
  std::int32_t pad;
  std::int64_t wofs;
};

// Column chunks of one solve sweep launch: chunk c (blockIdx.y) carries columns [8c, 8c + 8) of the
// launch's ncols right-hand sides, with its own contribution vectors, work array and counters at
// c times the strides.
struct SweepChunks {
  int ncols;
  int cnt_stride;
  std::int64_t x_stride;
  std::int64_t vec_stride;
  std::int64_t work_stride;
};

// Counters written by the factorization kernels (integers: sums are order independent).
struct FactorCounters {
  unsigned long long neg;
  unsigned long long zero;
  unsigned long long pos;
  unsigned long long two_by_two;
  unsigned long long failed;     // columns that could not be pivoted in their front
  unsigned long long forced;     // pivots accepted without the threshold test (roots)
  unsigned long long amax_bits;  // max |entry| of the scaled matrix (double bits)
  unsigned long long sync_timeouts;  // front barriers that gave up waiting (must stay 0)
};

struct FactorParams {
  double u;              // threshold of pivot acceptance
  double null_tol;       // relative null-pivot tolerance (0: detection off)
  const FactorCounters* cnt;  // amax lives in cnt->amax_bits
  std::int32_t failed_cap;
};

#if defined(__CUDACC__)
__device__ __forceinline__ double null_threshold(const FactorParams& p) {
  return p.null_tol > 0.0 ? p.null_tol * __longlong_as_double(static_cast<long long>(p.cnt->amax_bits)) : -1.0;
}

// atomic max of a non-negative double stored as its bit pattern (order independent)
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* slot, double v) {
  atomicMax(slot, static_cast<unsigned long long>(__double_as_longlong(v)));
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

#endif  // __CUDACC__

}  // namespace hsg
