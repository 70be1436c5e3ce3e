// Numeric multifrontal LDL^T kernels for sm_100a (FP64).
//
// What replaces MUMPS JOB=2 (hsolve src/factor/mumps_factorization.cpp:300-356; the arithmetic of
// MUMPS dfac_front_LDLT_type1.F / dfac_front_aux.F / dfac_asm.F): symmetric equilibration of
// K = alpha A + beta B, scatter of K into the fronts' panels, extend-add of children's contribution
// blocks, and the partial factorization of every front with 1x1 / 2x2 threshold pivots restricted
// to its fully-summed columns. Inertia (neg / zero / pos) is counted from D as pivots are accepted.
//
// Fronts are processed level by level (height in the assembly tree). Small fronts (m <= 64) are
// factorized entirely in shared memory by one CTA with right-looking threshold Bunch-Kaufman.
// Larger fronts use a-posteriori threshold pivoting by panels of NB columns: the diagonal block is
// factorized with Bunch-Kaufman restricted to the block, the rows below are solved against it while
// the largest |l| of every column is recorded, the longest acceptable prefix of pivots is kept
// (|l| <= 1/u), rejected columns are restored from a backup and moved behind the candidates, and
// the trailing matrix receives the rank-q update. Columns no candidate order can pivot are reported
// (failed) so that the host can move them into the parent front and factorize again.
#include <cooperative_groups.h>
#include <cstdint>
#include <mutex>

#include "common.hpp"
#include "device.cuh"
#include "factor_kernels.cuh"

namespace hsg {

namespace {

constexpr double kAlphaBK = 0.6403882032022076;  // (1 + sqrt(17)) / 8

// Determinant of a 2x2 pivot [a b; b c] in the factor's arithmetic R (the pivot test and the
// elimination use the same value).
template <class R>
__device__ __forceinline__ double pivot_det(double a, double b, double c) {
  const R ra = static_cast<R>(a), rb = static_cast<R>(b), rc = static_cast<R>(c);
  return static_cast<double>(ra * rc - rb * rb);
}

// two consecutive shared-memory values in one vector load (16-byte aligned pairs of doubles,
// 8-byte aligned pairs of floats)
__device__ __forceinline__ double2 load_pair(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ float2 load_pair(const float* p) { return *reinterpret_cast<const float2*>(p); }

// Asynchronous copy of one factor element (sizeof(R) bytes) from global to shared memory;
// valid == false fills the destination with zero.
template <class R>
__device__ __forceinline__ void cp_async_elem(R* dst, const R* src, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  if constexpr (sizeof(R) == 8) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
  }
}

// ------------------------------------------------------------------ scaling and assembly

__global__ void k_fill(double* x, std::int64_t n, double v) {
  for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::int64_t>(gridDim.x) * blockDim.x)
    x[i] = v;
}

__global__ void k_zero_u64(unsigned long long* x, std::int64_t n) {
  for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::int64_t>(gridDim.x) * blockDim.x)
    x[i] = 0ull;
}

// r[i] = max_j |d_i K_ij d_j| over both triangles (atomic max on non-negative doubles)
__global__ void k_scale_rowmax(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                               const double* b, double alpha, double beta, const double* d, unsigned long long* r) {
  for (std::int64_t p = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; p < nnz;
       p += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int32_t i = row[p], j = col[p];
    const double v = fabs((alpha * a[p] + beta * b[p]) * d[i] * d[j]);
    atomic_max_nonneg(&r[i], v);
    if (i != j) atomic_max_nonneg(&r[j], v);
  }
}

__global__ void k_scale_update(std::int64_t n, double* d, unsigned long long* r) {
  for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const double v = __longlong_as_double(static_cast<long long>(r[i]));
    if (v > 0.0) d[i] = d[i] / sqrt(v);
    r[i] = 0ull;
  }
}

// panels[dest[p]] = d_i d_j (alpha a_p + beta b_p) (rounded to the factor type R); records max |.|
// for the null-pivot threshold
template <class R>
__global__ void k_scatter(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                          const double* b, double alpha, double beta, const double* d, const std::int64_t* dest,
                          R* panels, FactorCounters* cnt) {
  double mx = 0.0;
  for (std::int64_t p = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; p < nnz;
       p += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int32_t i = row[p], j = col[p];
    const double v = (alpha * a[p] + beta * b[p]) * d[i] * d[j];
    panels[dest[p]] = static_cast<R>(v);
    mx = fmax(mx, fabs(v));
  }
  mx = warp_max(mx);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&cnt->amax_bits, mx);
}

// max |d_i d_j (alpha a_p + beta b_p)| alone (the null-pivot threshold of an inertia-only count,
// whose entries are scattered level by level)
__global__ void k_amax(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                       const double* b, double alpha, double beta, const double* d, FactorCounters* cnt) {
  double mx = 0.0;
  for (std::int64_t p = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; p < nnz;
       p += static_cast<std::int64_t>(gridDim.x) * blockDim.x)
    mx = fmax(mx, fabs((alpha * a[p] + beta * b[p]) * d[row[p]] * d[col[p]]));
  mx = warp_max(mx);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&cnt->amax_bits, mx);
}

// panels[dest[p]] = d_i d_j (alpha a_p + beta b_p) for the listed entries p = idx[t] (one level's)
template <class R>
__global__ void k_scatter_list(const std::int64_t* idx, std::int64_t count, const std::int32_t* row,
                               const std::int32_t* col, const double* a, const double* b, double alpha, double beta,
                               const double* d, const std::int64_t* dest, R* panels) {
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < count;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t p = idx[t];
    panels[dest[p]] = static_cast<R>((alpha * a[p] + beta * b[p]) * d[row[p]] * d[col[p]]);
  }
}

// zero the contribution blocks of the listed fronts (grid: fronts x chunks)
template <class R>
__global__ void k_zero_cb(const std::int32_t* list, const SnDev* sn, R* cb) {
  const SnDev s = sn[list[blockIdx.x]];
  const std::int64_t c = s.m - s.k;
  R* base = cb + s.cb_off;
  // the lower triangle only (column j: rows j .. c-1): no kernel reads a contribution block above
  // its diagonal. A warp per column, columns dealt over the chunk's warps.
  const int lane = threadIdx.x & 31;
  const std::int64_t nw = static_cast<std::int64_t>(gridDim.y) * (blockDim.x >> 5);
  for (std::int64_t j = static_cast<std::int64_t>(blockIdx.y) * (blockDim.x >> 5) + (threadIdx.x >> 5); j < c; j += nw) {
    R* col = base + j * c;
    for (std::int64_t i = j + lane; i < c; i += 32) col[i] = R(0);
  }
}

// Extend-add: item = (child, first column of a column block). Adds the child's lower CB
// columns [b0, b0 + EA_COLS) into its parent front (panel part or contribution block).
template <class R>
__global__ void k_extend_add(const int2* items, const SnDev* sn, const std::int32_t* rmap, R* panels, R* cb) {
  const int2 it = items[blockIdx.x];
  const SnDev c = sn[it.x];
  const SnDev p = sn[c.parent];
  const std::int32_t mc = c.m - c.k;
  const std::int32_t* rm = rmap + c.rmap_off;
  const R* src = cb + c.cb_off;
  const std::int32_t pc = p.m - p.k;
  const std::int32_t b0 = it.y;
  const std::int32_t bend = min(b0 + kExtendAddCols, mc);
  // the chunk's columns: destination column in the parent (its panel or its contribution block)
  // (rows of a contribution-block column are numbered from p.k: off = p.k there, 0 in the panel)
  R* dst[kExtendAddCols];
  std::int32_t off[kExtendAddCols];
#pragma unroll
  for (int u = 0; u < kExtendAddCols; ++u) {
    const std::int32_t bb = b0 + u;
    dst[u] = nullptr;
    off[u] = 0;
    if (bb < bend) {
      const std::int32_t pb = rm[bb];
      if (pb < p.k) dst[u] = panels + p.panel_off + static_cast<std::int64_t>(pb) * p.m;
      else { dst[u] = cb + p.cb_off + static_cast<std::int64_t>(pb - p.k) * pc; off[u] = p.k; }
    }
  }
  // a thread takes row a of every column of the chunk (lower triangle: a >= the column): all
  // sources and destinations are loaded before the stores, which could alias them for the compiler
  // (they do not: each destination entry receives exactly one addition per launch)
  for (std::int32_t a = b0 + threadIdx.x; a < mc; a += blockDim.x) {
    const std::int32_t ra = rm[a];
    R v[kExtendAddCols], d[kExtendAddCols];
#pragma unroll
    for (int u = 0; u < kExtendAddCols; ++u) {
      const bool in = dst[u] != nullptr && a >= b0 + u;
      v[u] = in ? src[static_cast<std::int64_t>(b0 + u) * mc + a] : R(0);
      d[u] = in ? dst[u][ra - off[u]] : R(0);
    }
#pragma unroll
    for (int u = 0; u < kExtendAddCols; ++u)
      if (dst[u] != nullptr && a >= b0 + u) dst[u][ra - off[u]] = d[u] + v[u];
  }
}

// ------------------------------------------------------------ dense pivoting in shared memory

// Decision of one pivot step (computed by warp 0).
enum : int { kFail = 0, kOneJ = 1, kOneR = 2, kTwoR = 3, kNull = 4 };

struct StepShared {
  int j, lim, prog, force, dec, r, stop;
  int neg, pos, zero, two, forced, eb;
};

// Warp 0: decide the pivot at column j of the lower-stored matrix F (order m, ld ld) with
// candidates [j, nfs). Row maxima cover all rows [j, m).
template <class R>
__device__ void decide_pivot(const R* F, int ld, int m, int nfs, int j, double u, double thr, bool force,
                             StepShared& st) {
  const int lane = threadIdx.x & 31;
  const R* cj = F + static_cast<std::int64_t>(j) * ld;
  double gc = 0.0, best = 0.0;
  int r = -1;
  for (int i = j + 1 + lane; i < m; i += 32) {
    const double v = fabs(cj[i]);
    gc = fmax(gc, v);
    if (i < nfs && v > best) { best = v; r = i; }
  }
  gc = warp_max(gc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int orr = __shfl_xor_sync(0xffffffffu, r, o);
    if (ob > best || (ob == best && orr >= 0 && (r < 0 || orr < r))) { best = ob; r = orr; }
  }
  const double dcc = fabs(cj[j]);
  int dec = kFail;
  if (thr >= 0.0 && fmax(dcc, gc) <= thr) dec = kNull;
  else if (dcc > 0.0 && dcc >= u * gc) dec = kOneJ;
  else if (force && (r < 0 || best == 0.0 || dcc >= kAlphaBK * gc)) dec = dcc > 0.0 ? kOneJ : kNull;
  if (dec == kFail && r >= 0 && best > 0.0) {
    // maxima of columns j and r excluding rows {j, r}
    const R* cr = F + static_cast<std::int64_t>(r) * ld;
    double gc2 = 0.0, gr2 = 0.0;
    for (int i = j + 1 + lane; i < m; i += 32) {
      if (i != r) gc2 = fmax(gc2, static_cast<double>(fabs(cj[i])));
      if (i < r && i != j) gr2 = fmax(gr2, static_cast<double>(fabs(F[r + static_cast<std::int64_t>(i) * ld])));
      if (i > r) gr2 = fmax(gr2, static_cast<double>(fabs(cr[i])));
    }
    gc2 = warp_max(gc2);
    gr2 = warp_max(gr2);
    const double a = cj[j], b = cj[r], c = cr[r];
    const double det = pivot_det<R>(a, b, c);
    if (force) {
      dec = det != 0.0 ? kTwoR : (dcc > 0.0 ? kOneJ : kNull);
    } else {
      if (det != 0.0) {
        const double ia = fabs(c / det), ib = fabs(b / det), ic = fabs(a / det);
        if (ia * gc2 + ib * gr2 <= 1.0 / u && ib * gc2 + ic * gr2 <= 1.0 / u) dec = kTwoR;
      }
      if (dec == kFail) {
        const double drr = fabs(c);
        if (drr > 0.0 && drr >= u * fmax(fabs(b), gr2)) dec = kOneR;
      }
    }
  }
  if (lane == 0) { st.dec = dec; st.r = r; }
}

// symmetric swap of positions p, q (< m) of the lower-stored matrix; labels follow
template <class R>
__device__ void sym_swap(R* F, int ld, int m, int p, int q, int* lab) {
  if (p == q) return;
  if (p > q) { const int t = p; p = q; q = t; }
  const int n1 = p, n2 = q - p - 1, n3 = m - q - 1;
  for (int t = threadIdx.x; t < n1 + n2 + n3 + 1; t += blockDim.x) {
    R *x, *y;
    if (t < n1) { x = F + p + static_cast<std::int64_t>(t) * ld; y = F + q + static_cast<std::int64_t>(t) * ld; }
    else if (t < n1 + n2) { const int c = p + 1 + (t - n1); x = F + c + static_cast<std::int64_t>(p) * ld; y = F + q + static_cast<std::int64_t>(c) * ld; }
    else if (t < n1 + n2 + n3) { const int i = q + 1 + (t - n1 - n2); x = F + i + static_cast<std::int64_t>(p) * ld; y = F + i + static_cast<std::int64_t>(q) * ld; }
    else { x = F + p + static_cast<std::int64_t>(p) * ld; y = F + q + static_cast<std::int64_t>(q) * ld; }
    const R v = *x; *x = *y; *y = v;
  }
  if (threadIdx.x == 0 && lab) { const int t = lab[p]; lab[p] = lab[q]; lab[q] = t; }
}

// eliminate a 1x1 (or null) pivot at j: column scaled to l, trailing rows/cols [j+1, m) updated
template <class R>
__device__ void elim1(R* F, int ld, int m, int j, bool null_piv, R* tmp) {
  const R d = F[j + static_cast<std::int64_t>(j) * ld];
  R* cj = F + static_cast<std::int64_t>(j) * ld;
  for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) {
    const R x = cj[i];
    tmp[i] = null_piv ? R(0) : x;
    cj[i] = null_piv ? R(0) : x / d;
  }
  __syncthreads();
  if (!null_piv) {
    const int w = m - j - 1;
    const R inv = R(1) / d;
    for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
      const int i = j + 1 + t % w, c = j + 1 + t / w;
      if (i >= c) F[i + static_cast<std::int64_t>(c) * ld] -= tmp[i] * tmp[c] * inv;
    }
  }
  __syncthreads();
}

// eliminate the 2x2 pivot (j, j+1)
template <class R>
__device__ void elim2(R* F, int ld, int m, int j, R* tmp0, R* tmp1) {
  const R a = F[j + static_cast<std::int64_t>(j) * ld], b = F[j + 1 + static_cast<std::int64_t>(j) * ld];
  const R c = F[j + 1 + static_cast<std::int64_t>(j + 1) * ld];
  const R det = a * c - b * b;
  const R ia = c / det, ib = -b / det, ic = a / det;
  R* c0 = F + static_cast<std::int64_t>(j) * ld;
  R* c1 = F + static_cast<std::int64_t>(j + 1) * ld;
  for (int i = j + 2 + threadIdx.x; i < m; i += blockDim.x) {
    const R x0 = c0[i], x1 = c1[i];
    tmp0[i] = x0;
    tmp1[i] = x1;
    c0[i] = ia * x0 + ib * x1;
    c1[i] = ib * x0 + ic * x1;
  }
  __syncthreads();
  const int w = m - j - 2;
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
    const int i = j + 2 + t % w, cc = j + 2 + t / w;
    if (i >= cc) F[i + static_cast<std::int64_t>(cc) * ld] -= c0[i] * tmp0[cc] + c1[i] * tmp1[cc];
  }
  __syncthreads();
}

// Threshold Bunch-Kaufman on a lower-stored dense matrix in shared memory: candidates [0, nfs),
// rows [0, m). root: pivots may be forced (never fail). Returns the number of eliminated columns
// (positions [e, nfs) failed); pv[t] in {0 null, 1 1x1, 2/3 2x2}; lab follows the swaps.
template <class R>
__device__ int dense_bk(R* F, int ld, int m, int nfs, bool root, double u, double thr, int* lab, signed char* pv,
                        R* tmp0, R* tmp1, StepShared& st) {
  if (threadIdx.x == 0) {
    st.j = 0; st.lim = nfs; st.prog = 0; st.force = 0; st.stop = 0;
    st.neg = st.pos = st.zero = st.two = st.forced = 0;
  }
  __syncthreads();
  while (true) {
    if (threadIdx.x == 0) {
      st.stop = 0;
      if (st.j >= nfs) st.stop = 1;
      else if (st.j >= st.lim) {
        if (st.prog) { st.lim = nfs; st.prog = 0; st.stop = 2; }
        else if (root && !st.force) { st.force = 1; st.lim = nfs; st.stop = 2; }
        else st.stop = 1;
      }
    }
    __syncthreads();
    if (st.stop == 1) break;
    if (st.stop == 2) continue;
    const int j = st.j;
    if (threadIdx.x < 32) decide_pivot(F, ld, m, nfs, j, u, thr, st.force != 0, st);
    __syncthreads();
    const int dec = st.dec, r = st.r;
    if (dec == kFail) {
      sym_swap(F, ld, m, j, st.lim - 1, lab);
      __syncthreads();
      if (threadIdx.x == 0) st.lim -= 1;
      __syncthreads();
      continue;
    }
    if (dec == kOneR) { sym_swap(F, ld, m, j, r, lab); __syncthreads(); }
    if (dec == kTwoR) { sym_swap(F, ld, m, j + 1, r, lab); __syncthreads(); }
    if (dec == kTwoR) {
      if (threadIdx.x == 0) {
        const R a = F[j + static_cast<std::int64_t>(j) * ld], b = F[j + 1 + static_cast<std::int64_t>(j) * ld];
        const R c = F[j + 1 + static_cast<std::int64_t>(j + 1) * ld];
        const R det = a * c - b * b;
        if (det < 0) { st.neg++; st.pos++; } else if (a + c < 0) st.neg += 2; else st.pos += 2;
        st.two++;
        if (st.force) st.forced++;
        pv[j] = 2; pv[j + 1] = 3;
      }
      elim2(F, ld, m, j, tmp0, tmp1);
      if (threadIdx.x == 0) {
        st.j = j + 2; st.prog = 1; st.force = 0;
        if (st.lim < st.j) st.lim = st.j;
        if (st.lim == j + 1) st.lim = j + 2;
      }
    } else {
      const bool nul = dec == kNull;
      if (threadIdx.x == 0) {
        const double d = F[j + static_cast<std::int64_t>(j) * ld];
        if (nul) { st.zero++; pv[j] = 0; }
        else { if (d < 0) st.neg++; else st.pos++; pv[j] = 1; }
        if (st.force) st.forced++;
      }
      elim1(F, ld, m, j, nul, tmp0);
      if (threadIdx.x == 0) {
        st.j = j + 1; st.prog = 1; st.force = 0;
        if (st.lim < st.j) st.lim = st.j;
      }
    }
    __syncthreads();
  }
  __syncthreads();
  return st.j;
}

// Warp maximum of non-negative floats: their bit patterns order like the values, so one integer
// warp reduction replaces a shuffle tree.
__device__ __forceinline__ float warp_maxf(float v) {
  return __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(v)));
}

// One warp: threshold Bunch-Kaufman on the panel's diagonal block (order w <= 32, shared memory,
// ld kNB, all rows candidates). Same acceptance rules as dense_bk; column maxima are reduced in
// single precision (a threshold test needs no more), the argmax for a 2 x 2 partner only when the
// 1 x 1 test fails, one reciprocal per pivot. The update of a step reads the pivot column(s) into
// registers first, so its column read-modify-writes are independent and pipeline (and the routine
// stays a compact loop: it runs once per panel, from a cold instruction cache). Not inlined: as a
// function of its own it is register-allocated apart from the panel kernels' other phases (255
// registers), which measured faster than the inlined loop; the call is once per panel.
// Warp-synchronous: no block barriers. Returns the eliminated count; [e, w) could not be pivoted.
template <class R>
__device__ __noinline__ int warp_block_bk(R* F, int w, bool root, double u, double thr, int* lab, signed char* pv,
                                          StepShared& st, int j0 = 0, int prog0 = 0) {
  const int lane = threadIdx.x & 31;
  constexpr int ld = kNB;
  __shared__ R s_c0[kNB], s_c1[kNB];
  int j = j0, lim = w, prog = prog0, force = 0;
  int neg = 0, pos = 0, zero = 0, two = 0, forced = 0;
  while (j < w) {
    if (j >= lim) {
      if (prog) { lim = w; prog = 0; continue; }
      if (root && !force) { force = 1; lim = w; continue; }
      break;
    }
    const R* cj = F + j * ld;
    const double xj = lane > j && lane < w ? cj[lane] : 0.0;
    const float gcf = warp_maxf(static_cast<float>(fabs(xj)));
    const double gc = static_cast<double>(gcf);
    const double dj = cj[j];
    const double dcc = fabs(dj);
    int dec = kFail, r = -1;
    if (thr >= 0.0 && fmax(dcc, gc) <= thr) dec = kNull;
    else if (dcc > 0.0 && dcc >= u * gc) dec = kOneJ;
    else {
      // partner candidate: argmax over rows (j, w) of |F(i, j)|
      float best = lane > j && lane < w ? static_cast<float>(fabs(xj)) : -1.0f;
      int bi = lane > j && lane < w ? lane : -1;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi >= 0 && (bi < 0 || oi < bi))) { best = ob; bi = oi; }
      }
      r = bi;
      if (force && (r < 0 || best <= 0.0f || dcc >= kAlphaBK * gc)) dec = dcc > 0.0 ? kOneJ : kNull;
      else if (r >= 0 && best > 0.0f) {
        const R* cr = F + r * ld;
        const double xr = lane > j && lane < w && lane != r ? (lane < r ? F[r + lane * ld] : cr[lane]) : 0.0;
        const float gr2f = warp_maxf(static_cast<float>(fabs(xr)));
        const float gc2f = warp_maxf(lane != r ? static_cast<float>(fabs(xj)) : 0.0f);
        const double gr2 = gr2f, gc2 = gc2f;
        const double a = dj, b = cj[r], c = cr[r];
        const double det = pivot_det<R>(a, b, c);
        if (force) dec = det != 0.0 ? kTwoR : (dcc > 0.0 ? kOneJ : kNull);
        else {
          if (det != 0.0) {
            const double ia = fabs(c / det), ib = fabs(b / det), ic = fabs(a / det);
            if (ia * gc2 + ib * gr2 <= 1.0 / u && ib * gc2 + ic * gr2 <= 1.0 / u) dec = kTwoR;
          }
          if (dec == kFail && fabs(c) > 0.0 && fabs(c) >= u * fmax(fabs(b), gr2)) dec = kOneR;
        }
      }
    }
    // swaps (rare)
    int sp = -1, sq = -1;
    if (dec == kFail) { sp = j; sq = lim - 1; }
    else if (dec == kOneR) { sp = j; sq = r; }
    else if (dec == kTwoR) { sp = j + 1; sq = r; }
    if (sp >= 0 && sp != sq) {
      int p = sp < sq ? sp : sq, q = sp < sq ? sq : sp;
      for (int t = lane; t < w + 1; t += 32) {
        R *x = nullptr, *y = nullptr;
        if (t < p) { x = F + p + t * ld; y = F + q + t * ld; }
        else if (t > p && t < q) { x = F + t + p * ld; y = F + q + t * ld; }
        else if (t > q && t < w) { x = F + t + p * ld; y = F + t + q * ld; }
        else if (t == p) { x = F + p + p * ld; y = F + q + q * ld; }
        if (x) { const R v = *x; *x = *y; *y = v; }
      }
      if (lane == 0) { const int tl = lab[p]; lab[p] = lab[q]; lab[q] = tl; }
      __syncwarp();
    }
    if (dec == kFail) { lim -= 1; continue; }
    const int i = lane;
    if (dec == kTwoR) {
      const R a = F[j + j * ld], b = F[j + 1 + j * ld], c = F[j + 1 + (j + 1) * ld];
      const R det = a * c - b * b;
      const R idet = R(1) / det;
      const R ia = c * idet, ib = -b * idet, ic = a * idet;
      const R x0 = (i >= j + 2 && i < w) ? F[i + j * ld] : R(0);
      const R x1 = (i >= j + 2 && i < w) ? F[i + (j + 1) * ld] : R(0);
      const R l0 = ia * x0 + ib * x1, l1 = ib * x0 + ic * x1;
      // the pivot columns go through shared memory into registers first, so that the column
      // updates below are independent of each other (no store can alias a later load)
      s_c0[i] = x0;
      s_c1[i] = x1;
      __syncwarp();
      R y0[kNB], y1[kNB];
#pragma unroll
      for (int c2 = 0; c2 < kNB; ++c2) { y0[c2] = s_c0[c2]; y1[c2] = s_c1[c2]; }
#pragma unroll
      for (int c2 = 0; c2 < kNB; ++c2)
        if (c2 >= j + 2 && i >= c2 && i < w) F[i + c2 * ld] -= l0 * y0[c2] + l1 * y1[c2];
      __syncwarp();
      if (i >= j + 2 && i < w) { F[i + j * ld] = l0; F[i + (j + 1) * ld] = l1; }
      if (lane == 0) { pv[j] = 2; pv[j + 1] = 3; }
      if (det < 0) { neg++; pos++; } else if (a + c < 0) neg += 2; else pos += 2;
      two++;
      if (force) forced++;
      j += 2;
    } else {
      const bool nul = dec == kNull;
      const R d = F[j + j * ld];
      const R inv = nul ? R(0) : R(1) / d;
      const R x = (i > j && i < w) ? F[i + j * ld] : R(0);
      const R xs = x * inv;
      s_c0[i] = x;
      __syncwarp();
      if (!nul) {
        R y[kNB];
#pragma unroll
        for (int c2 = 0; c2 < kNB; ++c2) y[c2] = s_c0[c2];
#pragma unroll
        for (int c2 = 0; c2 < kNB; ++c2)
          if (c2 > j && i >= c2 && i < w) F[i + c2 * ld] -= xs * y[c2];
      }
      __syncwarp();
      if (i > j && i < w) F[i + j * ld] = xs;
      if (lane == 0) pv[j] = nul ? 0 : 1;
      if (nul) zero++;
      else if (d < 0) neg++;
      else pos++;
      if (force) forced++;
      j += 1;
    }
    __syncwarp();
    prog = 1;
    force = 0;
    if (lim < j) lim = j;
  }
  if (lane == 0) { st.neg += neg; st.pos += pos; st.zero += zero; st.two += two; st.forced += forced; }
  return j;
}

}  // namespace

// ---------------------------------------------------------------------- small fronts (smem)

template <int MAXM, class R>
__global__ void __launch_bounds__(256) k_front_small(const std::int32_t* list, const SnDev* sn, R* panels,
                                                      R* cb, signed char* piv_out, std::int32_t* pidx_out,
                                                      FactorParams prm, FactorCounters* cnt, std::int32_t* failed) {
  extern __shared__ __align__(16) unsigned char small_dyn[];
  R* F = reinterpret_cast<R*>(small_dyn);
  __shared__ R tmp0[MAXM], tmp1[MAXM];
  __shared__ int lab[MAXM];
  __shared__ signed char pv[MAXM];
  __shared__ StepShared st;
  const SnDev d = sn[list[blockIdx.x]];
  const int m = d.m, k = d.k, ld = m, c = m - k;
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int i = t % m, j = t / m;
    if (i < j) continue;
    F[t] = j < k ? panels[d.panel_off + static_cast<std::int64_t>(j) * m + i]
                 : cb[d.cb_off + static_cast<std::int64_t>(j - k) * c + (i - k)];
  }
  for (int t = threadIdx.x; t < m; t += blockDim.x) lab[t] = t;
  __syncthreads();
  const double thr = null_threshold(prm);
  const int e = dense_bk(F, ld, m, k, d.parent < 0, prm.u, thr, lab, pv, tmp0, tmp1, st);
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int i = t % m, j = t / m;
    if (i < j) continue;
    if (j < k) panels[d.panel_off + static_cast<std::int64_t>(j) * m + i] = F[t];
    else cb[d.cb_off + static_cast<std::int64_t>(j - k) * c + (i - k)] = F[t];
  }
  for (int t = threadIdx.x; t < k; t += blockDim.x) {
    pidx_out[d.first + t] = lab[t];
    piv_out[d.first + t] = t < e ? pv[t] : static_cast<signed char>(-1);
  }
  if (threadIdx.x == 0) {
    if (st.neg) atomicAdd(&cnt->neg, static_cast<unsigned long long>(st.neg));
    if (st.pos) atomicAdd(&cnt->pos, static_cast<unsigned long long>(st.pos));
    if (st.zero) atomicAdd(&cnt->zero, static_cast<unsigned long long>(st.zero));
    if (st.two) atomicAdd(&cnt->two_by_two, static_cast<unsigned long long>(st.two));
    if (st.forced) atomicAdd(&cnt->forced, static_cast<unsigned long long>(st.forced));
    if (e < k) {
      const unsigned long long at = atomicAdd(&cnt->failed, static_cast<unsigned long long>(k - e));
      for (int t = e; t < k; ++t)
        if (at + (t - e) < static_cast<unsigned long long>(prm.failed_cap)) failed[at + (t - e)] = d.first + lab[t];
    }
  }
}

// ------------------------------------------------------------- larger fronts: a-posteriori pivoting
//
// One front is processed by nr CTAs (nr = 1 for the one-CTA-per-front kernel; nr >= 1 per front in the
// cooperative kernel, where every step is separated by a grid-wide barrier). The pivoting state of a
// front lives in its global scratch (AppCtrl + block + labels + column maxima + backup), written by
// the front's rank-0 CTA and read by all its CTAs after the barrier.

namespace {

template <class R>
struct FrontView {
  R* panel;  // m x k, ld m
  R* cbb;    // (m-k)^2, ld m-k
  int m, k;
  __device__ R* col(int c) const {
    return c < k ? panel + static_cast<std::int64_t>(c) * m : cbb + static_cast<std::int64_t>(c - k) * (m - k) - k;
  }
  __device__ R& at(int i, int c) const { return col(c)[i]; }
};

struct AppCtrl {
  int p, lim, prog, force, stop, w, eb, q;
  int neg, pos, zero, two, forced, finished, fb, bar;  // fb: first pivot whose trailing update is pending;
                                                       // bar: arrivals at the front's barrier
};

// The fields of the control block that a panel step reads, copied by every CTA of the front right
// after a barrier: rank 0 may already change the control block for the next panel while slower
// CTAs still work on this one.
struct StepView {
  int p, w, lim, fb, eb, force, stop;
};

// The scratch of a front is laid out in units of doubles whatever the factor type R; the R-typed
// arrays (B, Borig, backup) occupy the first sizeof(R) / 8 of their double-sized regions.
template <class R>
struct AppFront {
  FrontView<R> f;
  int first;
  bool root;
  AppCtrl* ctrl;
  double* slots;   // two sets of the per-panel arrays below, used by alternate panels
  R* B;            // factored diagonal block, kNB x kNB col-major
  R* Borig;        // the block before factorization
  int* lab;        // block permutation
  signed char* pv; // block pivot types
  unsigned long long* cmax;
  unsigned long long* rmax;
  R* backup;       // kNB columns of m rows
  std::int32_t* plab;
  signed char* ppv;
};

// point the per-panel arrays at set `slot` (0 or 1)
template <class R>
__device__ __forceinline__ void set_slot(AppFront<R>& F, int slot) {
  double* s = F.slots + slot * kAppSlotDoubles;
  F.B = reinterpret_cast<R*>(s);
  s += kNB * kNB;
  F.Borig = reinterpret_cast<R*>(s);
  s += kNB * kNB;
  F.lab = reinterpret_cast<int*>(s);
  s += kNB / 2;
  F.pv = reinterpret_cast<signed char*>(s);
  s += kNB / 8;
  F.cmax = reinterpret_cast<unsigned long long*>(s);
  s += kNB;
  F.rmax = reinterpret_cast<unsigned long long*>(s);
}

__device__ __forceinline__ StepView step_view(const AppCtrl* c) {
  StepView v;
  v.p = __ldcg(&c->p);
  v.w = __ldcg(&c->w);
  v.lim = __ldcg(&c->lim);
  v.fb = __ldcg(&c->fb);
  v.eb = __ldcg(&c->eb);
  v.force = __ldcg(&c->force);
  v.stop = __ldcg(&c->stop);
  return v;
}

template <class R>
__device__ AppFront<R> make_front(const SnDev& d, R* panels, R* cb, double* scratch, signed char* piv_out,
                                  std::int32_t* pidx_out) {
  AppFront<R> F;
  F.f = FrontView<R>{panels + d.panel_off, d.cb_off >= 0 ? cb + d.cb_off : nullptr, d.m, d.k};
  F.first = d.first;
  F.root = d.parent < 0;
  double* s = scratch + d.scratch_off;
  F.ctrl = reinterpret_cast<AppCtrl*>(s);
  s += kAppCtrlDoubles;
  F.slots = s;
  s += 2 * kAppSlotDoubles;
  F.backup = reinterpret_cast<R*>(s);
  F.plab = pidx_out + d.first;
  F.ppv = piv_out + d.first;
  set_slot(F, 0);
  return F;
}

// symmetric swap of fully-summed positions a, b (< k) of the front in global memory
template <class R>
__device__ void front_swap(const FrontView<R>& f, int a, int b, std::int32_t* lab) {
  if (a == b) return;
  if (a > b) { const int t = a; a = b; b = t; }
  const int n1 = a, n2 = b - a - 1, n3 = f.m - b - 1;
  for (int t = threadIdx.x; t < n1 + n2 + n3 + 1; t += blockDim.x) {
    R *x, *y;
    if (t < n1) { x = &f.at(a, t); y = &f.at(b, t); }
    else if (t < n1 + n2) { const int c = a + 1 + (t - n1); x = &f.at(c, a); y = &f.at(b, c); }
    else if (t < n1 + n2 + n3) { const int i = b + 1 + (t - n1 - n2); x = &f.at(i, a); y = &f.at(i, b); }
    else { x = &f.at(a, a); y = &f.at(b, b); }
    const R v = *x; *x = *y; *y = v;
  }
  if (threadIdx.x == 0) { const std::int32_t t = lab[a]; lab[a] = lab[b]; lab[b] = t; }
}

// Init (all ranks split the label work; rank 0 the control block).
template <class R>
__device__ void app_init(AppFront<R>& F, int rank, int nr) {
  const int k = F.f.k;
  for (int t = rank * blockDim.x + threadIdx.x; t < k; t += nr * blockDim.x) { F.plab[t] = t; F.ppv[t] = -1; }
  if (rank == 0 && threadIdx.x == 0) {
    AppCtrl c{};
    c.lim = k;
    *F.ctrl = c;
  }
}

// Rank 0: decide what the next panel is (stop = 1: front finished), and factorize its diagonal block
// with block-restricted threshold Bunch-Kaufman; permute the L rows of the block; publish to scratch.
template <class R>
__device__ void app_control_and_block(AppFront<R>& F, const FactorParams& prm, double thr, R* Bs, R* tmp0,
                                      R* tmp1, int* slab, signed char* spv, StepShared& bst, int* shared_stop,
                                      FactorCounters* cnt, std::int32_t* failed, int* level_done) {
  AppCtrl* c = F.ctrl;
  const int k = F.f.k;
  if (threadIdx.x == 0) {
    int stop = 1;
    if (!c->finished) {
      while (true) {
        if (c->p >= k) { stop = 1; break; }
        if (c->p >= c->lim) {
          if (c->prog) { c->lim = k; c->prog = 0; continue; }
          if (F.root && !c->force) { c->force = 1; c->lim = k; continue; }
          stop = 1;
          break;
        }
        stop = 0;
        c->w = min(kNB, c->lim - c->p);
        break;
      }
    }
    c->stop = stop;
    *shared_stop = stop;
    if (stop && !c->finished) {
      c->finished = 1;
      const int e = c->p;
      if (c->neg) atomicAdd(&cnt->neg, static_cast<unsigned long long>(c->neg));
      if (c->pos) atomicAdd(&cnt->pos, static_cast<unsigned long long>(c->pos));
      if (c->zero) atomicAdd(&cnt->zero, static_cast<unsigned long long>(c->zero));
      if (c->two) atomicAdd(&cnt->two_by_two, static_cast<unsigned long long>(c->two));
      if (c->forced) atomicAdd(&cnt->forced, static_cast<unsigned long long>(c->forced));
      if (e < k) {
        const unsigned long long at = atomicAdd(&cnt->failed, static_cast<unsigned long long>(k - e));
        for (int t = e; t < k; ++t)
          if (at + (t - e) < static_cast<unsigned long long>(prm.failed_cap)) failed[at + (t - e)] = F.first + F.plab[t];
      }
      if (level_done) atomicAdd(level_done, 1);
    }
  }
  __syncthreads();
  if (*shared_stop) return;
  const int p = c->p, w = c->w;
  const bool force = c->force != 0;
  if (force && p + 1 < k) {
    // A root front that made no progress over all its remaining columns: Bunch-Kaufman's choice
    // for column p without threshold, with the partner searched among all remaining fully-summed
    // rows (not only the block's), is brought next to p before the block is factorized.
    __shared__ double s_bv[32], s_gc[32];
    __shared__ int s_bi[32], s_r;
    double bv = -1.0, gc = 0.0;
    int bi = -1;
    for (int i = p + 1 + threadIdx.x; i < F.f.m; i += blockDim.x) {
      const double v = fabs(F.f.at(i, p));
      gc = fmax(gc, v);
      if (i < k && v > bv) { bv = v; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      gc = fmax(gc, __shfl_xor_sync(0xffffffffu, gc, o));
      if (ov > bv || (ov == bv && oi >= 0 && (bi < 0 || oi < bi))) { bv = ov; bi = oi; }
    }
    if ((threadIdx.x & 31) == 0) { s_bv[threadIdx.x >> 5] = bv; s_bi[threadIdx.x >> 5] = bi; s_gc[threadIdx.x >> 5] = gc; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = -1.0, g = 0.0;
      int r = -1;
      for (int q = 0; q < static_cast<int>(blockDim.x >> 5); ++q) {
        g = fmax(g, s_gc[q]);
        if (s_bv[q] > b || (s_bv[q] == b && s_bi[q] >= 0 && (r < 0 || s_bi[q] < r))) { b = s_bv[q]; r = s_bi[q]; }
      }
      const double dcc = fabs(F.f.at(p, p));
      s_r = (r < 0 || b <= 0.0 || dcc >= kAlphaBK * g) ? -1 : r;
    }
    __syncthreads();
    const int r = s_r;
    if (r > p + 1) front_swap(F.f, p + 1, r, F.plab);
    __syncthreads();
  }
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
    const int i = t % w, j = t / w;
    if (i >= j) {
      const double v = F.f.at(p + i, p + j);
      Bs[i + j * kNB] = v;
      F.Borig[i + j * kNB] = v;
    }
  }
  for (int t = threadIdx.x; t < w; t += blockDim.x) slab[t] = t;
  if (threadIdx.x == 0) { bst.neg = bst.pos = bst.zero = bst.two = bst.forced = 0; bst.eb = 0; }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int e = warp_block_bk(Bs, w, force, prm.u, thr, slab, spv, bst);
    if (threadIdx.x == 0) bst.eb = e;
  }
  __syncthreads();
  const int eb = bst.eb;
  if (__syncthreads_or(threadIdx.x < w && slab[threadIdx.x] != static_cast<int>(threadIdx.x))) {
    // the block's rows were swapped: its pivot labels follow
    int old = 0;
    if (threadIdx.x < w) old = F.plab[p + slab[threadIdx.x]];
    __syncthreads();
    if (threadIdx.x < w) F.plab[p + threadIdx.x] = old;
  }
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
    const int i = t % w, j = t / w;
    if (i >= j) F.f.at(p + i, p + j) = Bs[i + j * kNB];
  }
  for (int t = threadIdx.x; t < kNB * kNB; t += blockDim.x) F.B[t] = Bs[t];
  for (int t = threadIdx.x; t < kNB; t += blockDim.x) {
    F.lab[t] = slab[t];
    F.pv[t] = spv[t];
    F.cmax[t] = 0ull;
    F.rmax[t] = 0ull;
  }
  if (threadIdx.x == 0) c->eb = eb;
}

// All ranks: rows [p+w, m) solved against the block (L21 = F21 P L11^-T D^-1), backup, column maxima.
// The block's strict lower part with the 2x2 couplings masked (they belong to D) is staged in Ls
// (shared). The rows of a rank go through shared memory in chunks of kRowChunk: all threads load
// the chunk (coalesced, batches of loads in flight at once) and write the backup; one thread per row
// runs the substitution fully unrolled in registers and applies D^-1 through per-column coefficients
// (no branch on the pivot type, every store after the last load); a warp per four columns then
// writes the L values back (coalesced) and reduces the column maxima.
template <class R>
__device__ void app_rows(AppFront<R>& F, const StepView& v, int rank, int nr, R* Bs, int* slab, signed char* spv,
                         unsigned long long* scm, unsigned long long* srm, R* Lm) {
  const int p = v.p, w = v.w, eb = v.eb, m = F.f.m;
  for (int t = threadIdx.x; t < kNB * kNB; t += blockDim.x) Bs[t] = __ldcg(&F.B[t]);
  for (int t = threadIdx.x; t < kNB; t += blockDim.x) {
    slab[t] = __ldcg(&F.lab[t]);
    spv[t] = __ldcg(&F.pv[t]);
    scm[t] = 0ull;
    srm[t] = 0ull;
  }
  __syncthreads();
  // Lm[t * kNB + s] = L11(t, s) for s < min(t, eb), zero otherwise (row-major for broadcast reads)
  for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x) {
    const int t = e / kNB, s = e % kNB;
    R x = R(0);
    if (t < w && s < t && s < eb && !(spv[s] == 2 && s + 1 == t)) x = Bs[t + s * kNB];
    Lm[e] = x;
  }
  // D^-1 as three coefficients per column: out(t) = k0 y(t-1) + k1 y(t) + k2 y(t+1); ksel says
  // which value the column maximum takes: 0 |out|, 1 |y| (null pivot, l = 0), 2 none (t >= eb)
  R* k0 = Lm + kNB * kNB;
  R* k1 = k0 + kNB;
  R* k2 = k1 + kNB;
  int* ksel = reinterpret_cast<int*>(k2 + kNB);
  R* Y = Lm + kRowStage;  // kNB columns of kRowChunk rows
  for (int t = threadIdx.x; t < kNB; t += blockDim.x) {
    R a0 = R(0), a1 = R(1), a2 = R(0);
    int sel = 2;
    if (t < eb) {
      const signed char ty = spv[t];
      sel = 0;
      if (ty == 0) { a1 = R(0); sel = 1; }
      else if (ty == 1) a1 = R(1) / Bs[t + t * kNB];
      else {
        const int f0 = ty == 2 ? t : t - 1;
        const R a = Bs[f0 + f0 * kNB], b = Bs[f0 + 1 + f0 * kNB], cc = Bs[f0 + 1 + (f0 + 1) * kNB];
        const R idet = R(1) / (a * cc - b * b);
        // first of the pair: l = (c y_t - b y_{t+1}) / det; second: l = (a y_t - b y_{t-1}) / det
        if (ty == 2) { a1 = cc * idet; a2 = -b * idet; }
        else { a0 = -b * idet; a1 = a * idet; }
      }
    }
    k0[t] = a0;
    k1[t] = a1;
    k2[t] = a2;
    ksel[t] = sel;
  }
  // did the block factorization swap any of its rows? (rarely: then the permutation below moves data)
  const bool permuted = __syncthreads_or(threadIdx.x < w && slab[threadIdx.x] != static_cast<int>(threadIdx.x)) != 0;
  // permute the L rows p..p+w-1 of the eliminated columns c < p (a thread owns a column; the
  // columns are split into contiguous chunks over the ranks)
  const int cchunk = (p + nr - 1) / nr;
  const int cend = permuted ? min(p, (rank + 1) * cchunk) : 0;
  for (int cc = rank * cchunk + threadIdx.x; cc < cend; cc += blockDim.x) {
    R x[kNB];
    R* colp = F.f.col(cc) + p;
#pragma unroll
    for (int a = 0; a < kNB; ++a) x[a] = a < w ? colp[slab[a]] : R(0);
#pragma unroll
    for (int a = 0; a < kNB; ++a)
      if (a < w) colp[a] = x[a];
  }
  const int rtotal = m - (p + w);
  const int rchunk = (rtotal + nr - 1) / nr;
  const int rbeg = p + w + rank * rchunk, rend = min(m, rbeg + rchunk);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // warp `warp` writes back and reduces the maxima of columns 4 warp .. 4 warp + 3 (eight warps)
  static_assert(kAppThreads / 32 * 4 == kNB, "the write-back pass takes four columns per warp");
  constexpr int kStageBatch = 8;
  // column maxima in FP32 (rounding is monotone: the maximum of the rounded values is the rounded
  // maximum), reduced over the warp with one integer max on the bit patterns of the non-negative floats
  float cm[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int c0 = rbeg; c0 < rend; c0 += kRowChunk) {
    const int nrow = min(kRowChunk, rend - c0);
    const int total = w * nrow;
    __syncthreads();
    // stage: element e = (column t, row r), column-major, consecutive threads on consecutive rows;
    // a batch of loads is issued before any store (the stores could alias later loads)
    for (int e0 = threadIdx.x; e0 < total; e0 += kStageBatch * kAppThreads) {
      R x[kStageBatch];
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const int e = e0 + u * kAppThreads;
        const int t = e / nrow, r = e - t * nrow;
        x[u] = e < total ? F.f.at(c0 + r, p + slab[t]) : R(0);
      }
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const int e = e0 + u * kAppThreads;
        if (e < total) {
          const int t = e / nrow, r = e - t * nrow;
          F.backup[static_cast<std::int64_t>(t) * m + c0 + r] = x[u];
          Y[t * kRowChunk + r] = x[u];
        }
      }
    }
    __syncthreads();
    // one thread per row: substitution and D^-1 in registers, then the row back to shared memory
    // (the l values; |y| of a null pivot column, whose l is zero, for its maximum)
    for (int r = threadIdx.x; r < nrow; r += kAppThreads) {
      R y[kNB];
#pragma unroll
      for (int t = 0; t < kNB; ++t) y[t] = t < w ? Y[t * kRowChunk + r] : R(0);
#pragma unroll
      for (int t = 1; t < kNB; ++t) {
        R acc = y[t];
#pragma unroll
        for (int s2 = 0; s2 < t; ++s2) acc = fma(-y[s2], Lm[t * kNB + s2], acc);
        y[t] = acc;
      }
      R prev = R(0);
#pragma unroll
      for (int t = 0; t < kNB; ++t) {
        const R yn = t + 1 < kNB ? y[t + 1 < kNB ? t + 1 : t] : R(0);
        const R out = fma(k0[t], prev, fma(k2[t], yn, k1[t] * y[t]));
        prev = y[t];
        y[t] = ksel[t] == 1 ? y[t] : out;
        // the coefficients are read eight columns at a time (hoisting all of them would spill)
        if ((t & 7) == 7) asm volatile("" ::: "memory");
      }
#pragma unroll
      for (int t = 0; t < kNB; ++t)
        if (t < w) Y[t * kRowChunk + r] = y[t];
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int t = 4 * warp + c;
      if (t < w) {
        const int sel = ksel[t];
        R* colp = F.f.col(p + t) + c0;
        // a batch of shared-memory reads before the global stores (which could alias them)
        for (int r0 = lane; r0 < nrow; r0 += 32 * kStageBatch) {
          R x[kStageBatch];
#pragma unroll
          for (int u = 0; u < kStageBatch; ++u) {
            const int r = r0 + 32 * u;
            x[u] = r < nrow ? Y[t * kRowChunk + r] : R(0);
          }
#pragma unroll
          for (int u = 0; u < kStageBatch; ++u) {
            const int r = r0 + 32 * u;
            if (r < nrow) colp[r] = sel == 1 ? R(0) : x[u];
            if (sel != 2) cm[c] = fmaxf(cm[c], static_cast<float>(fabs(x[u])));
          }
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float x = warp_maxf(cm[c]);
    const int t = 4 * warp + c;
    // the column maximum of |l| (|y| for a null pivot), rounded up by 1e-7 to stay conservative;
    // the accept step reads the maxima of all ranks
    if (lane == 0 && t < w && x > 0.0f) {
      const double ad = static_cast<double>(x) * (1.0 + 1e-7);
      const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(ad));
      atomicMax(&F.cmax[t], bits);
      atomicMax(&F.rmax[t], bits);
    }
  }
  (void)scm;
  (void)srm;
}

// All ranks: the accepted prefix q (identical in every CTA); rank 0 books the inertia. The small
// per-panel arrays are staged in shared memory first (one parallel load) so that warp 0's tests
// below touch no global memory. Bs / spv already hold the panel's block and pivot types (app_rows).
template <class R>
__device__ int app_accept(AppFront<R>& F, const StepView& v, int rank, double thr, double inv_u, int* sq,
                          const R* Bs, const signed char* spv, unsigned long long* scm,
                          unsigned long long* srm) {
  const int eb = v.eb;
  const int p = v.p;
  const bool force = v.force != 0;
  for (int t = threadIdx.x; t < kNB; t += blockDim.x) {
    scm[t] = __ldcg(&F.cmax[t]);
    srm[t] = __ldcg(&F.rmax[t]);
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    // warp 0: lane t tests the pivot that starts at t (the second of a 2x2 pair starts none); the
    // accepted prefix ends at the first failing start. A forced step accepts its first pivot
    // without the threshold; the block's later pivots were chosen from the block alone and pass the
    // a-posteriori tests like any other.
    const int t = threadIdx.x;
    const signed char ty = t < eb ? spv[t] : static_cast<signed char>(3);
    const bool start = t < eb && ty != 3;
    bool fail = false;
    if (start && !(force && t == 0)) {
      const double cm = __longlong_as_double(static_cast<long long>(scm[t]));
      if (ty == 0) fail = __longlong_as_double(static_cast<long long>(srm[t])) > thr;
      else if (ty == 1) fail = cm > inv_u;
      else {
        const double cm2 = t + 1 < kNB ? __longlong_as_double(static_cast<long long>(scm[t + 1])) : 0.0;
        fail = fmax(cm, cm2) > inv_u;
      }
    }
    const unsigned fails = __ballot_sync(0xffffffffu, fail);
    const unsigned over = __ballot_sync(0xffffffffu, start && ty != 0 && ty != 1 && t + 1 >= eb);
    const int q = fails ? __ffs(fails) - 1 : (over ? eb + 1 : eb);
    if (t == 0) *sq = q;
    if (rank == 0) {
      // inertia of the accepted pivots: lane t books the pivot that starts at t
      int neg = 0, pos = 0, zero = 0, two = 0;
      if (start && t < q) {
        if (ty == 0) zero = 1;
        else if (ty == 1) { if (Bs[t + t * kNB] < 0) neg = 1; else pos = 1; }
        else if (ty == 2) {
          const R a = Bs[t + t * kNB], b = Bs[t + 1 + t * kNB], cc = Bs[t + 1 + (t + 1) * kNB];
          const R det = a * cc - b * b;
          if (det < 0) { neg = 1; pos = 1; } else if (a + cc < 0) neg = 2; else pos = 2;
          two = 1;
        }
      }
      neg = __reduce_add_sync(0xffffffffu, neg);
      pos = __reduce_add_sync(0xffffffffu, pos);
      zero = __reduce_add_sync(0xffffffffu, zero);
      two = __reduce_add_sync(0xffffffffu, two);
      if (t == 0) {
        AppCtrl* cw = F.ctrl;
        cw->q = q;
        cw->neg += neg;
        cw->pos += pos;
        cw->zero += zero;
        cw->two += two;
        if (force && q > 0) cw->forced += spv[0] == 2 ? 2 : 1;
      }
    }
  }
  __syncthreads();
  const int q = *sq;
  if (rank == 0)
    for (int t = threadIdx.x; t < q; t += blockDim.x) F.ppv[p + t] = spv[t];
  return q;
}

// All ranks: restore the rejected block columns [q, w) from the backup / original block.
template <class R>
__device__ void app_restore(AppFront<R>& F, const StepView& v, int rank, int nr, int q) {
  const int p = v.p, w = v.w, m = F.f.m;
  const int rtotal = m - (p + w);
  const int rchunk = (rtotal + nr - 1) / nr;
  const int rbeg = p + w + rank * rchunk, rend = min(m, rbeg + rchunk);
  for (int i = rbeg + threadIdx.x; i < rend; i += blockDim.x)
    for (int t = q; t < w; ++t) F.f.at(i, p + t) = F.backup[static_cast<std::int64_t>(t) * m + i];
  if (rank == 0) {
    for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
      const int a = t % w, b = t / w;
      if (b >= q && a >= b) {
        const int la = F.lab[a], lb = F.lab[b];
        F.f.at(p + a, p + b) = la >= lb ? F.Borig[la + lb * kNB] : F.Borig[lb + la * kNB];
      }
    }
  }
}

__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// Blocked step. The pivots [fb, p + q) eliminated since the last full update are pending: their
// Schur update has reached only the panels factorized since. After a panel the pending update goes
// either to the whole trailing matrix (a flush: the panel rejected columns, the candidate range
// ends, or kKB pivots would be pending after the next panel) or to the next panel's columns only.
// A column is therefore up to date when its panel is factorized, and every other trailing column
// receives the pending pivots in one rank-(<= kKB) update instead of one update per panel.
__device__ __forceinline__ bool app_flushes(int p, int w, int q, int lim, int fb) {
  return q < w || p + q >= lim || p + q + kNB - fb > kKB;
}

// All ranks: C(i, c) -= sum_{s in [fb, p+q)} L(i, s) W(c, s), W = L D, over the lower triangle
// c <= i < m of the columns c in [p+q, col_hi): all trailing columns when the step flushes, else the
// next panel's. Rejected columns [p+q, p+w) of a flushing panel already hold the updates of
// [fb, p) (they were part of the panel) and take only those of [p, p+q). W is formed while staging
// from L and the pivots' D (1x1: d; 2x2 [a b; b c]: W(c, s) = a L(c, s) + b L(c, s+1) and
// W(c, s+1) = b L(c, s) + c L(c, s+1)); null pivots have L = 0.
//
// The update runs on the FP64 tensor cores (mma.sync m8n8k4, D = A B + C with A 8 x 4, B 4 x 8) by
// 64 x 64 tiles of C dealt round-robin to the ranks: the tile's rows of L and its columns' rows of
// L (<= kKB pivots) are copied asynchronously (cp.async, zero-filled outside the front) into shared
// memory, column-major with stride kUpdLd = 4 (mod 16), so that the copies of consecutive rows are
// contiguous and every fragment read of a half-warp hits 32 distinct banks; D is then applied to the
// second copy in place. Warp w (of 8) computes rows 16 (w % 4) .. +16 and columns 32 (w / 4) .. +32
// of the tile as 2 x 4 blocks of 8 x 8. A thread's fragment element (g, t) is row g = lane / 4,
// column t = lane % 4 of A; row t, column g of B; row g, columns 2t, 2t + 1 of C.
// FP32 factors (the operator factorization of the mixed-precision path) keep the same staging and
// the same output ownership per thread, and accumulate with FP32 FMAs (there is no FP32 tensor
// instruction with full FP32 operands; the FP64 refinement of every solve absorbs FP32 rounding).
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

//
// With look-ahead (la: the panel was accepted whole and the next one follows directly), rank 0 takes
// only tile 0, which holds the next panel's diagonal block, so that it can factorize that block
// while the other ranks finish the remaining tiles.
template <class R>
__device__ void app_update(AppFront<R>& F, const StepView& v, int rank, int nr, int q, bool la, R* Ls, R* Ws,
                           R* ca, R* cb, int* cd, const R* Bs, const signed char* spv) {
  const int p = v.p, w = v.w, lim = v.lim, fb = v.fb, m = F.f.m;
  const int from = p + q;
  const int K = from - fb;
  const int rows = m - from;
  if (rows <= 0 || K <= 0) return;
  const bool flush = app_flushes(p, w, q, lim, fb);
  const int col_hi = flush ? m : min(m, from + min(kNB, lim - from));
  const int rej_hi = flush && q < w ? p + w : 0;  // columns below this take only the pivots >= p
  // staging coefficients of the pending pivots: W(c, fb+s) = ca[s] L(c, fb+s) + cb[s] L(c, fb+s+cd[s])
  // (the panel's own pivots from the block in shared memory: rank 0 books their types in global
  // memory while the other ranks may already be here)
  for (int s = threadIdx.x; s < K; s += blockDim.x) {
    const int j = fb + s;
    R x = R(0), y = R(0);
    int d = 0;
    if (j >= p) {
      const int t = j - p;
      const signed char ty = spv[t];
      if (ty == 1) x = Bs[t + t * kNB];
      else if (ty == 2) { x = Bs[t + t * kNB]; y = Bs[t + 1 + t * kNB]; d = 1; }
      else if (ty == 3) { x = Bs[t + t * kNB]; y = Bs[t + (t - 1) * kNB]; d = -1; }
    } else {
      const signed char ty = __ldcg(&F.ppv[j]);
      if (ty == 1) x = __ldcg(&F.f.at(j, j));
      else if (ty == 2) { x = __ldcg(&F.f.at(j, j)); y = __ldcg(&F.f.at(j + 1, j)); d = 1; }
      else if (ty == 3) { x = __ldcg(&F.f.at(j, j)); y = __ldcg(&F.f.at(j, j - 1)); d = -1; }
    }
    ca[s] = x;
    cb[s] = y;
    cd[s] = d;
  }
  const int nt = (rows + kTile - 1) / kTile;
  const int nct = (col_hi - from + kTile - 1) / kTile;
  const int ntiles = nct * nt - nct * (nct - 1) / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int rbase = (warp & 3) * 16, cbase = (warp >> 2) * 32;
  const int Kpad = (K + 3) & ~3;
  // tiles of this rank: round-robin, or with look-ahead tile 0 for rank 0 and the rest over ranks 1..
  const bool split = la && nr > 1;
  const int tfirst = split ? (rank == 0 ? 0 : rank) : rank;
  const int tstep = split ? (rank == 0 ? ntiles : nr - 1) : nr;
  for (int tile = tfirst; tile < ntiles; tile += tstep) {
    int ti, tj;
    if (nct == nt) {
      ti = static_cast<int>((sqrt(8.0 * tile + 1.0) - 1.0) * 0.5);
      while ((ti + 1) * (ti + 2) / 2 <= tile) ++ti;
      while (ti * (ti + 1) / 2 > tile) --ti;
      tj = tile - ti * (ti + 1) / 2;
    } else {
      int rest = tile;
      tj = 0;
      while (rest >= nt - tj) { rest -= nt - tj; ++tj; }
      ti = tj + rest;
    }
    const int i0 = from + ti * kTile, j0 = from + tj * kTile;
    __syncthreads();
    {
      // thread: tile row r, pivots s = sg, sg + 4, ...: all copies in flight at once
      const int r = threadIdx.x & (kTile - 1), sg = threadIdx.x >> 6;
      const int i = i0 + r, cc = j0 + r;
      const int li = i < m ? i : from, lc = cc < m ? cc : from;
      const bool lb = i < m, wb = cc < col_hi;
#pragma unroll 8
      for (int s = sg; s < Kpad; s += kAppThreads / kTile) {
        const bool in = s < K;
        const R* lj = F.f.col(fb + (in ? s : 0));
        cp_async_elem(&Ls[s * kUpdLd + r], lj + li, in && lb);
        cp_async_elem(&Ws[s * kUpdLd + r], lj + lc, in && wb);
      }
    }
    // prefetch this thread's C entries (rows rbase + 8a + g, columns cbase + 8b + 2 t4 + e)
    R* colp[4][2];
    R cv[2][4][2];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int cc = j0 + cbase + 8 * b + 2 * t4 + e;
        colp[b][e] = cc < col_hi ? F.f.col(cc) : nullptr;
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          const int i = i0 + rbase + 8 * a + g;
          cv[a][b][e] = (colp[b][e] && i < m && cc <= i) ? colp[b][e][i] : R(0);
        }
      }
    cp_async_wait_all();
    __syncthreads();
    // W = L D in place (a 2x2 pair by its first column), zero for the rejected columns' old pivots
    for (int t = threadIdx.x; t < K * kTile; t += blockDim.x) {
      const int s = t / kTile, r = t % kTile;
      const int d = cd[s];
      if (d < 0) continue;
      const bool masked = j0 + r < rej_hi && fb + s < p;
      R* w0 = &Ws[s * kUpdLd + r];
      if (d == 0) {
        *w0 = masked ? R(0) : ca[s] * *w0;
      } else {
        R* w1 = w0 + kUpdLd;
        const R x0 = *w0, x1 = *w1;
        *w0 = masked ? R(0) : fma(ca[s], x0, cb[s] * x1);
        *w1 = masked ? R(0) : fma(cb[s + 1], x0, ca[s + 1] * x1);
      }
    }
    __syncthreads();
    // warps whose 32 columns all lie at or beyond col_hi (the second half of a panel's tile) or
    // whose 16 rows all lie above their first column have nothing to update
    const bool idle = j0 + cbase >= col_hi || i0 + rbase + 15 < j0 + cbase;
    if (idle) continue;
    R acc[2][4][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) { acc[a][b][0] = R(0); acc[a][b][1] = R(0); }
    if constexpr (sizeof(R) == 8) {
#pragma unroll 2
      for (int s0 = 0; s0 < Kpad; s0 += 4) {
        double af[2], bf[4];
#pragma unroll
        for (int a = 0; a < 2; ++a) af[a] = Ls[(s0 + t4) * kUpdLd + rbase + 8 * a + g];
#pragma unroll
        for (int b = 0; b < 4; ++b) bf[b] = Ws[(s0 + t4) * kUpdLd + cbase + 8 * b + g];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) dmma_m8n8k4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
      }
    } else {
      // FP32: the thread's own 2 x 8 outputs by rank-1 steps (two L values, four W pairs per pivot)
#pragma unroll 4
      for (int s = 0; s < K; ++s) {
        const R* ls = Ls + s * kUpdLd + rbase + g;
        const R* ws = Ws + s * kUpdLd + cbase + 2 * t4;
        const R l0 = ls[0], l1 = ls[8];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const auto w2 = load_pair(ws + 8 * b);
          acc[0][b][0] = fma(l0, w2.x, acc[0][b][0]);
          acc[0][b][1] = fma(l0, w2.y, acc[0][b][1]);
          acc[1][b][0] = fma(l1, w2.x, acc[1][b][0]);
          acc[1][b][1] = fma(l1, w2.y, acc[1][b][1]);
        }
      }
    }
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int cc = j0 + cbase + 8 * b + 2 * t4 + e;
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          const int i = i0 + rbase + 8 * a + g;
          if (colp[b][e] && i < m && cc <= i) colp[b][e][i] = cv[a][b][e] - acc[a][b][e];
        }
      }
  }
}

// Rank 0: advance past the accepted pivots; move rejected columns behind the candidates.
template <class R>
__device__ void app_advance(AppFront<R>& F, int q) {
  AppCtrl* c = F.ctrl;
  const int p = c->p, w = c->w;
  const int np = p + q, r = w - q;
  const int lim = c->lim;
  const bool flushed = app_flushes(p, w, q, lim, c->fb);
  if (r > 0 && np + r < lim) {
    for (int t = 0; t < r; ++t) {
      front_swap(F.f, np + t, lim - r + t, F.plab);
      __syncthreads();
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    c->p = np;
    if (flushed) c->fb = np;
    if (q > 0) { c->prog = 1; c->force = 0; }
    if (r > 0) c->lim = np + r < lim ? lim - r : np;
  }
  __syncthreads();
}

template <class R>
struct AppSmem {
  R Bs[kNB * kNB];
  R tmp0[kNB], tmp1[kNB];
  int slab[kNB];
  signed char spv[kNB];
  unsigned long long scm[kNB], srm[kNB];
  StepShared bst;
  R ca[kKB], cb[kKB];
  int cd[kKB];
  int stop, q, ok;
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier of the nr CTAs of one front (all co-resident: cooperative launch). Arrivals count up in
// the front's control block; a CTA waits until the count reaches the next multiple of nr. The wait
// gives up after kBarrierTimeoutNs (or when another front has given up), books the timeout in the
// counters and returns false, so that a stuck front ends the kernel instead of hanging it.
constexpr unsigned long long kBarrierTimeoutNs = 5ull * 1000 * 1000 * 1000;

__device__ bool front_barrier(int* bar, int nr, unsigned long long* timeouts, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    if (nr > 1) {
      // arrival with release semantics (the CTA's writes, ordered before it by the block barrier,
      // become visible to every rank that acquires the count) and acquire for the later reads
      int old;
      asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(bar) : "memory");
      const int target = (old / nr + 1) * nr;
      unsigned long long t0 = 0;
      for (unsigned it = 0;; ++it) {
        int arrived;
        asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(arrived) : "l"(bar) : "memory");
        if (arrived >= target) break;
        if ((it & 63u) == 63u) {
          if (*reinterpret_cast<volatile unsigned long long*>(timeouts) != 0ull) { ok = 0; break; }
          const unsigned long long t = global_ns();
          if (t0 == 0) t0 = t;
          else if (t - t0 > kBarrierTimeoutNs) { atomicAdd(timeouts, 1ull); ok = 0; break; }
          __nanosleep(64);
        }
      }
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// The panel loop of one front, run by its nr CTAs (rank 0 .. nr-1). A step is
//   [control: rank 0 advances past the previous panel and factorizes the next block] barrier
//   rows (all) barrier  accept (all, identical)  [restore (all) barrier]  update (all) barrier
// and when a panel is accepted whole and the next one follows directly (look-ahead), rank 0
// advances and factorizes the next block right after its update tile, so that the control phase
// and its barrier are skipped. Alternate panels use alternate per-panel arrays, so the next
// block's arrays never overlap the ones slower CTAs still read.
template <bool kCoop, class R>
__device__ void app_front(AppFront<R>& F, int rank, int nr, const FactorParams& prm, FactorCounters* cnt,
                          std::int32_t* failed, int* level_done, AppSmem<R>& sm, R* Ls, R* Ws) {
  const double thr = null_threshold(prm);
  const double inv_u = 1.0 / prm.u;
  int* bar = &F.ctrl->bar;
  auto sync = [&]() -> bool {
    if (kCoop) return front_barrier(bar, nr, &cnt->sync_timeouts, &sm.ok);
    __syncthreads();
    return true;
  };
  bool la = false;
  int j = 0, qprev = 0;
  while (true) {
    if (!la) {
      if (rank == 0) {
        if (j > 0) app_advance(F, qprev);
        set_slot(F, j & 1);
        app_control_and_block(F, prm, thr, sm.Bs, sm.tmp0, sm.tmp1, sm.slab, sm.spv, sm.bst, &sm.stop, cnt, failed,
                              level_done);
      }
      if (!sync()) break;
    }
    set_slot(F, j & 1);
    const StepView v = step_view(F.ctrl);
    if (v.stop) break;
    app_rows(F, v, rank, nr, sm.Bs, sm.slab, sm.spv, sm.scm, sm.srm, Ls);
    if (!sync()) break;
    const int q = app_accept(F, v, rank, thr, inv_u, &sm.q, sm.Bs, sm.spv, sm.scm, sm.srm);
    if (q < v.w) {
      app_restore(F, v, rank, nr, q);
      if (!sync()) break;
    }
    la = q == v.w && v.p + v.w < v.lim;
    app_update(F, v, rank, nr, q, la, Ls, Ws, sm.ca, sm.cb, sm.cd, sm.Bs, sm.spv);
    if (la && rank == 0) {
      __syncthreads();
      app_advance(F, q);
      set_slot(F, (j + 1) & 1);
      app_control_and_block(F, prm, thr, sm.Bs, sm.tmp0, sm.tmp1, sm.slab, sm.spv, sm.bst, &sm.stop, cnt, failed,
                            level_done);
    }
    if (!sync()) break;
    qprev = q;
    ++j;
  }
}

}  // namespace

// One CTA per front (nr = 1), fronts listed in `list`.
template <class R>
__global__ void __launch_bounds__(kAppThreads) k_front_app(const std::int32_t* list, const SnDev* sn, R* panels,
                                                           R* cb, double* scratch, signed char* piv_out,
                                                           std::int32_t* pidx_out, FactorParams prm,
                                                           FactorCounters* cnt, std::int32_t* failed) {
  extern __shared__ __align__(16) unsigned char app_dyn[];
  R* Ls = reinterpret_cast<R*>(app_dyn);
  R* Ws = Ls + kKB * kUpdLd;
  __shared__ AppSmem<R> sm;
  const SnDev d = sn[list[blockIdx.x]];
  AppFront<R> F = make_front(d, panels, cb, scratch, piv_out, pidx_out);
  app_init(F, 0, 1);
  __syncthreads();
  app_front<false>(F, 0, 1, prm, cnt, failed, nullptr, sm, Ls, Ws);
}

// Cooperative: the fronts of a level share the grid; front f owns CTAs [cta_start[f], cta_start[f+1])
// and runs its panel loop with its own barriers, independently of the other fronts.
template <class R>
__global__ void __launch_bounds__(kAppThreads) k_front_coop(const std::int32_t* list, const std::int32_t* cta_start,
                                                            int nfronts, const SnDev* sn, R* panels, R* cb,
                                                            double* scratch, signed char* piv_out,
                                                            std::int32_t* pidx_out, FactorParams prm,
                                                            FactorCounters* cnt, std::int32_t* failed,
                                                            int* level_done) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(16) unsigned char app_dyn[];
  R* Ls = reinterpret_cast<R*>(app_dyn);
  R* Ws = Ls + kKB * kUpdLd;
  __shared__ AppSmem<R> sm;
  int fi = 0;
  while (fi + 1 < nfronts && cta_start[fi + 1] <= static_cast<int>(blockIdx.x)) ++fi;
  const int rank = static_cast<int>(blockIdx.x) - cta_start[fi];
  const int nr = cta_start[fi + 1] - cta_start[fi];
  const SnDev d = sn[list[fi]];
  AppFront<R> F = make_front(d, panels, cb, scratch, piv_out, pidx_out);
  app_init(F, rank, nr);
  grid.sync();  // the control blocks (and their barrier counts) are initialized
  app_front<true>(F, rank, nr, prm, cnt, failed, level_done, sm, Ls, Ws);
}

// ------------------------------------------------------------------------------ launchers

void launch_fill(double* x, std::int64_t n, double v, cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = static_cast<int>(std::min<std::int64_t>((n + 255) / 256, 148 * 16));
  note_launches(1);
  k_fill<<<blocks, 256, 0, s>>>(x, n, v);
}

void launch_zero_u64(unsigned long long* x, std::int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = static_cast<int>(std::min<std::int64_t>((n + 255) / 256, 148 * 16));
  note_launches(1);
  k_zero_u64<<<blocks, 256, 0, s>>>(x, n);
}

void launch_scale_rowmax(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                         const double* b, double alpha, double beta, const double* d, unsigned long long* r,
                         cudaStream_t s) {
  const int blocks = static_cast<int>(std::min<std::int64_t>((nnz + 255) / 256, 148 * 16));
  note_launches(1);
  k_scale_rowmax<<<blocks, 256, 0, s>>>(nnz, row, col, a, b, alpha, beta, d, r);
}

void launch_scale_update(std::int64_t n, double* d, unsigned long long* r, cudaStream_t s) {
  const int blocks = static_cast<int>(std::min<std::int64_t>((n + 255) / 256, 148 * 16));
  note_launches(1);
  k_scale_update<<<blocks, 256, 0, s>>>(n, d, r);
}

template <class R>
void launch_scatter(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                    const double* b, double alpha, double beta, const double* d, const std::int64_t* dest,
                    R* panels, FactorCounters* cnt, cudaStream_t s) {
  const int blocks = static_cast<int>(std::min<std::int64_t>((nnz + 255) / 256, 148 * 16));
  note_launches(1);
  k_scatter<R><<<blocks, 256, 0, s>>>(nnz, row, col, a, b, alpha, beta, d, dest, panels, cnt);
}

void launch_amax(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a, const double* b,
                 double alpha, double beta, const double* d, FactorCounters* cnt, cudaStream_t s) {
  const int blocks = static_cast<int>(std::min<std::int64_t>((nnz + 255) / 256, 148 * 16));
  note_launches(1);
  k_amax<<<blocks, 256, 0, s>>>(nnz, row, col, a, b, alpha, beta, d, cnt);
}

template <class R>
void launch_scatter_list(const std::int64_t* idx, std::int64_t count, const std::int32_t* row, const std::int32_t* col,
                         const double* a, const double* b, double alpha, double beta, const double* d,
                         const std::int64_t* dest, R* panels, cudaStream_t s) {
  if (count <= 0) return;
  const int blocks = static_cast<int>(std::min<std::int64_t>((count + 255) / 256, 148 * 16));
  note_launches(1);
  k_scatter_list<R><<<blocks, 256, 0, s>>>(idx, count, row, col, a, b, alpha, beta, d, dest, panels);
}

template <class R>
void launch_zero_cb(const std::int32_t* list, int nlist, int chunks, const SnDev* sn, R* cb, cudaStream_t s) {
  if (nlist <= 0) return;
  dim3 grid(nlist, chunks);
  note_launches(1);
  k_zero_cb<R><<<grid, 256, 0, s>>>(list, sn, cb);
}

template <class R>
void launch_extend_add(const int2* items, int nitems, const SnDev* sn, const std::int32_t* rmap, R* panels, R* cb,
                       cudaStream_t s) {
  if (nitems <= 0) return;
  note_launches(1);
  k_extend_add<R><<<nitems, 128, 0, s>>>(items, sn, rmap, panels, cb);
}

template <class R>
void launch_front_small(int maxm, const std::int32_t* list, int nlist, const SnDev* sn, R* panels, R* cb,
                        signed char* piv, std::int32_t* pidx, const FactorParams& prm, FactorCounters* cnt,
                        std::int32_t* failed, cudaStream_t s) {
  if (nlist <= 0) return;
  const std::size_t smem = static_cast<std::size_t>(maxm) * maxm * sizeof(R);
  note_launches(1);
  if (maxm <= 32) k_front_small<32, R><<<nlist, 128, smem, s>>>(list, sn, panels, cb, piv, pidx, prm, cnt, failed);
  else k_front_small<kSmallMax, R><<<nlist, 256, smem, s>>>(list, sn, panels, cb, piv, pidx, prm, cnt, failed);
}

template <class R>
constexpr std::size_t app_dyn_bytes() { return static_cast<std::size_t>(kAppDynDoubles) * sizeof(R); }

template <class R>
void launch_front_app(const std::int32_t* list, int nlist, const SnDev* sn, R* panels, R* cb, double* scratch,
                      signed char* piv, std::int32_t* pidx, const FactorParams& prm, FactorCounters* cnt,
                      std::int32_t* failed, cudaStream_t s) {
  if (nlist <= 0) return;
  constexpr std::size_t smem = app_dyn_bytes<R>();
  static std::once_flag configured;
  std::call_once(configured, [&] {
    cudaFuncSetAttribute(k_front_app<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  });
  note_launches(1);
  k_front_app<R><<<nlist, kAppThreads, smem, s>>>(list, sn, panels, cb, scratch, piv, pidx, prm, cnt, failed);
}

namespace {
template <class R>
int coop_max_ctas_of(int device) {
  constexpr std::size_t smem = app_dyn_bytes<R>();
  cudaFuncSetAttribute(k_front_coop<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  int per_sm = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_front_coop<R>, kAppThreads, smem);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return per_sm * sms;
}
}  // namespace

// co-resident CTAs of the cooperative panel kernel, valid for both factor types (one plan serves a
// factorization object of either precision)
int coop_max_ctas(int device) { return std::min(coop_max_ctas_of<double>(device), coop_max_ctas_of<float>(device)); }

template <class R>
cudaError_t launch_front_coop(const std::int32_t* list, const std::int32_t* cta_start, int nfronts, int nctas,
                              const SnDev* sn, R* panels, R* cb, double* scratch, signed char* piv, std::int32_t* pidx,
                              const FactorParams& prm, FactorCounters* cnt, std::int32_t* failed, int* level_done,
                              cudaStream_t s) {
  if (nfronts <= 0) return cudaSuccess;
  constexpr std::size_t smem = app_dyn_bytes<R>();
  FactorParams p = prm;
  void* args[] = {const_cast<std::int32_t**>(&list), const_cast<std::int32_t**>(&cta_start), &nfronts,
                  const_cast<SnDev**>(&sn), &panels, &cb, &scratch, &piv, &pidx, &p, &cnt, &failed, &level_done};
  note_launches(1);
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_front_coop<R>), dim3(nctas), dim3(kAppThreads), args,
                                     smem, s);
}

#define HSG_FACTOR_INSTANTIATE(R)                                                                                     \
  template void launch_scatter<R>(std::int64_t, const std::int32_t*, const std::int32_t*, const double*,             \
                                  const double*, double, double, const double*, const std::int64_t*, R*,              \
                                  FactorCounters*, cudaStream_t);                                                     \
  template void launch_zero_cb<R>(const std::int32_t*, int, int, const SnDev*, R*, cudaStream_t);                     \
  template void launch_scatter_list<R>(const std::int64_t*, std::int64_t, const std::int32_t*, const std::int32_t*,   \
                                       const double*, const double*, double, double, const double*,                  \
                                       const std::int64_t*, R*, cudaStream_t);                                       \
  template void launch_extend_add<R>(const int2*, int, const SnDev*, const std::int32_t*, R*, R*, cudaStream_t);     \
  template void launch_front_small<R>(int, const std::int32_t*, int, const SnDev*, R*, R*, signed char*,              \
                                      std::int32_t*, const FactorParams&, FactorCounters*, std::int32_t*,             \
                                      cudaStream_t);                                                                  \
  template void launch_front_app<R>(const std::int32_t*, int, const SnDev*, R*, R*, double*, signed char*,            \
                                    std::int32_t*, const FactorParams&, FactorCounters*, std::int32_t*, cudaStream_t); \
  template cudaError_t launch_front_coop<R>(const std::int32_t*, const std::int32_t*, int, int, const SnDev*, R*, R*, \
                                            double*, signed char*, std::int32_t*, const FactorParams&,                 \
                                            FactorCounters*, std::int32_t*, int*, cudaStream_t);
HSG_FACTOR_INSTANTIATE(double)
HSG_FACTOR_INSTANTIATE(float)
#undef HSG_FACTOR_INSTANTIATE

}  // namespace hsg
