// Supernodal forward / diagonal / backward solves with nrhs right-hand sides (replaces MUMPS JOB=3,
// hsolve src/factor/mumps_factorization.cpp:459-527; MUMPS dsol_fwd.F / dsol_bwd.F).
//
// The forward sweep runs level by level like the factorization: a front gathers its pivot rows from
// the solution vector and its children's contribution vectors (fixed order, no atomics, so results
// are bitwise reproducible), solves with its unit-lower L11 in blocks of at most 32 columns (never
// splitting a 2x2 pivot), and leaves its contribution -L21 z for the parent. The backward sweep
// runs top-down and only gathers (ancestors' values are final). All right-hand sides of a chunk
// are carried together so that every L entry is read once per chunk.
#include <cooperative_groups.h>
#include <cstdint>

#include "common.hpp"
#include "device.cuh"
#include "solve_kernels.cuh"

namespace hsg {

namespace {

__global__ void k_gather_scale(std::int64_t n, int nrhs, const double* b, std::int64_t ldb, const double* d,
                               const std::int32_t* iperm, double* x) {
  const std::int64_t total = n * nrhs;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t i = t % n, r = t / n;
    x[iperm[i] + r * n] = b[i + r * ldb] * d[i];
  }
}

__global__ void k_scatter_scale(std::int64_t n, int nrhs, double* b, std::int64_t ldb, const double* d,
                                const std::int32_t* iperm, const double* x) {
  const std::int64_t total = n * nrhs;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t i = t % n, r = t / n;
    b[i + r * ldb] = x[iperm[i] + r * n] * d[i];
  }
}

// block partition of the k pivots: at most 32 columns, a 2x2 pivot never split
__device__ __forceinline__ int block_size_at(const signed char* pv, int b, int k) {
  int bs = k - b < 32 ? k - b : 32;
  if (bs == 32 && pv[b + 31] == 2) bs = 31;
  return bs;
}

}  // namespace

// After a factorization: the block partition of every front's pivots (<= 32 columns, 2x2 pivots
// never split) and the inverses of its unit-lower diagonal blocks (2x2 couplings are D, not L, and
// excluded), so that the solves apply each block as one small matrix-vector product instead of a
// chain of dependent pivot steps. One CTA per front; warp w inverts blocks w, w + 8, ...; lane c
// computes column c by forward substitution.
__global__ void __launch_bounds__(256) k_inv_blocks(const SnDev* sn, const double* panels, const signed char* piv,
                                                     std::int32_t* blk, std::int32_t* nblk, double* inv) {
  __shared__ int starts[kMaxBlocksPerFront];
  __shared__ int nb;
  const int s = blockIdx.x;
  const SnDev d = sn[s];
  const int k = d.k, m = d.m;
  const signed char* pv = piv + d.first;
  if (threadIdx.x == 0) {
    int c = 0;
    for (int b = 0; b < k && c < kMaxBlocksPerFront;) {
      starts[c++] = b;
      b += block_size_at(pv, b, k);
    }
    nb = c;
    nblk[s] = c;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb; i += blockDim.x) blk[d.first + i] = starts[i];
  const double* P = panels + d.panel_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int bi = warp; bi < nb; bi += nwarps) {
    const int b = starts[bi];
    const int bs = bi + 1 < nb ? starts[bi + 1] - b : k - b;
    double* out = inv + d.inv_off + static_cast<std::int64_t>(bi) * 1024;
    double x[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) x[i] = 0.0;
    if (lane < bs) {
      x[lane] = 1.0;
      for (int i = lane + 1; i < bs; ++i) {
        double acc = 0.0;
        for (int j = lane; j < i; ++j) {
          if (j + 1 == i && pv[b + j] == 2) continue;  // D coupling of a 2x2 pivot
          acc += P[(b + i) + static_cast<std::int64_t>(b + j) * m] * x[j];
        }
        x[i] = -acc;
      }
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) out[lane * 32 + i] = (lane < bs) ? x[i] : 0.0;
  }
}

// Forward sweep of the listed fronts. t (m x R, row-major) in dynamic shared memory.
__global__ void __launch_bounds__(256) k_solve_fwd(const std::int32_t* list, const SnDev* sn,
                                                    const std::int32_t* child_ptr, const std::int32_t* children,
                                                    const std::int32_t* rmap, const double* panels,
                                                    const signed char* piv, const std::int32_t* pidx,
                                                    const std::int32_t* blk, const std::int32_t* nblk,
                                                    const double* inv, double* x, std::int64_t n, double* vec,
                                                    int nrhs, int R) {
  extern __shared__ double smem[];
  __shared__ double zb[32 * 8];
  const int s = list[blockIdx.x];
  const SnDev d = sn[s];
  const int m = d.m, k = d.k, c = m - k;
  double* t = smem;
  int* invp = reinterpret_cast<int*>(smem + static_cast<std::int64_t>(m) * R);
  const double* P = panels + d.panel_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* bst = blk + d.first;
  const int nb = nblk[s];
  const double* Linv = inv + d.inv_off;
  for (int i = threadIdx.x; i < k; i += blockDim.x) invp[pl[i]] = i;
  for (int r0 = 0; r0 < nrhs; r0 += R) {
    const int rr = nrhs - r0 < R ? nrhs - r0 : R;
    __syncthreads();
    for (int idx = threadIdx.x; idx < m * R; idx += blockDim.x) {
      const int i = idx / R, r = idx % R;
      double v = 0.0;
      if (i < k && r < rr) v = x[d.first + pl[i] + (r0 + r) * n];
      t[idx] = v;
    }
    __syncthreads();
    for (int q = child_ptr[s]; q < child_ptr[s + 1]; ++q) {
      const SnDev cd = sn[children[q]];
      const int mc = cd.m - cd.k;
      const std::int32_t* rm = rmap + cd.rmap_off;
      const double* cv = vec + cd.vec_off * nrhs;
      for (int a = threadIdx.x; a < mc; a += blockDim.x) {
        const int pos = rm[a];
        const int row = pos < k ? invp[pos] : pos;
        for (int r = 0; r < rr; ++r) t[row * R + r] += cv[a + static_cast<std::int64_t>(r0 + r) * mc];
      }
      __syncthreads();
    }
    for (int bi = 0; bi < nb; ++bi) {
      const int b = bst[bi];
      const int be = bi + 1 < nb ? bst[bi + 1] : k;
      const int bs = be - b;
      const double* Li = Linv + static_cast<std::int64_t>(bi) * 1024;
      // z_blk = Linv t_blk   (thread (i, r))
      {
        const int i = threadIdx.x % 32, r = threadIdx.x / 32;
        if (i < bs && r < rr) {
          double acc = 0.0;
          for (int cc = 0; cc <= i; ++cc) acc += Li[cc * 32 + i] * t[(b + cc) * R + r];
          zb[i * 8 + r] = acc;
        }
      }
      __syncthreads();
      {
        const int i = threadIdx.x % 32, r = threadIdx.x / 32;
        if (i < bs && r < rr) t[(b + i) * R + r] = zb[i * 8 + r];
      }
      // rows below: t_i -= L[i, blk] z_blk
      for (int i = be + threadIdx.x; i < m; i += blockDim.x) {
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j < bs; ++j) {
          const double l = P[i + static_cast<std::int64_t>(b + j) * m];
#pragma unroll
          for (int r = 0; r < 8; ++r)
            if (r < rr) acc[r] += l * zb[j * 8 + r];
        }
#pragma unroll
        for (int r = 0; r < 8; ++r)
          if (r < rr) t[i * R + r] -= acc[r];
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < k; i += blockDim.x)
      for (int r = 0; r < rr; ++r) x[d.first + pl[i] + (r0 + r) * n] = t[i * R + r];
    double* v = vec + d.vec_off * nrhs;
    for (int a = threadIdx.x; a < c; a += blockDim.x)
      for (int r = 0; r < rr; ++r) v[a + static_cast<std::int64_t>(r0 + r) * c] = t[(k + a) * R + r];
  }
}

// Diagonal solve D y = z, one CTA per front.
__global__ void k_solve_diag(const SnDev* sn, const double* panels, const signed char* piv, const std::int32_t* pidx,
                             double* x, std::int64_t n, int nrhs) {
  const SnDev d = sn[blockIdx.x];
  const double* P = panels + d.panel_off;
  for (int j = threadIdx.x; j < d.k; j += blockDim.x) {
    const signed char ty = piv[d.first + j];
    if (ty == 3) continue;
    const std::int64_t g0 = d.first + pidx[d.first + j];
    if (ty == 0 || ty < 0) {
      for (int r = 0; r < nrhs; ++r) x[g0 + r * n] = 0.0;
    } else if (ty == 1) {
      const double dj = P[j + static_cast<std::int64_t>(j) * d.m];
      for (int r = 0; r < nrhs; ++r) x[g0 + r * n] /= dj;
    } else {
      const std::int64_t g1 = d.first + pidx[d.first + j + 1];
      const double a = P[j + static_cast<std::int64_t>(j) * d.m], b = P[j + 1 + static_cast<std::int64_t>(j) * d.m];
      const double c = P[j + 1 + static_cast<std::int64_t>(j + 1) * d.m];
      const double det = a * c - b * b;
      for (int r = 0; r < nrhs; ++r) {
        const double y0 = x[g0 + r * n], y1 = x[g1 + r * n];
        x[g0 + r * n] = (c * y0 - b * y1) / det;
        x[g1 + r * n] = (-b * y0 + a * y1) / det;
      }
    }
  }
}

// Backward sweep of the listed fronts (ancestors done): right-looking over the blocks, last first.
__global__ void __launch_bounds__(256) k_solve_bwd(const std::int32_t* list, const SnDev* sn, const std::int32_t* rows,
                                                    const double* panels, const std::int32_t* pidx,
                                                    const std::int32_t* blk, const std::int32_t* nblk,
                                                    const double* inv, double* x, std::int64_t n, int nrhs, int R) {
  extern __shared__ double smem[];
  __shared__ double zb[32 * 8];
  const int s = list[blockIdx.x];
  const SnDev d = sn[s];
  const int m = d.m, k = d.k;
  double* t = smem;
  const double* P = panels + d.panel_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* rw = rows + d.rows_off;
  const std::int32_t* bst = blk + d.first;
  const int nb = nblk[s];
  const double* Linv = inv + d.inv_off;
  for (int r0 = 0; r0 < nrhs; r0 += R) {
    const int rr = nrhs - r0 < R ? nrhs - r0 : R;
    __syncthreads();
    for (int idx = threadIdx.x; idx < m * R; idx += blockDim.x) {
      const int i = idx / R, r = idx % R;
      double v = 0.0;
      if (r < rr) v = i < k ? x[d.first + pl[i] + (r0 + r) * n] : x[rw[i] + (r0 + r) * n];
      t[idx] = v;
    }
    __syncthreads();
    // t_j -= sum_{i >= k} L[i, j] t_i  (thread per column; the column is contiguous)
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      const double* Lj = P + static_cast<std::int64_t>(j) * m;
      for (int i = k; i < m; ++i) {
        const double l = Lj[i];
#pragma unroll
        for (int r = 0; r < 8; ++r)
          if (r < rr) acc[r] += l * t[i * R + r];
      }
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < rr) t[j * R + r] -= acc[r];
    }
    __syncthreads();
    for (int bi = nb - 1; bi >= 0; --bi) {
      const int b = bst[bi];
      const int be = bi + 1 < nb ? bst[bi + 1] : k;
      const int bs = be - b;
      const double* Li = Linv + static_cast<std::int64_t>(bi) * 1024;
      // x_blk = Linv^T t_blk  (thread (c, r))
      {
        const int cc = threadIdx.x % 32, r = threadIdx.x / 32;
        if (cc < bs && r < rr) {
          double acc = 0.0;
          for (int i = cc; i < bs; ++i) acc += Li[cc * 32 + i] * t[(b + i) * R + r];
          zb[cc * 8 + r] = acc;
        }
      }
      __syncthreads();
      {
        const int cc = threadIdx.x % 32, r = threadIdx.x / 32;
        if (cc < bs && r < rr) t[(b + cc) * R + r] = zb[cc * 8 + r];
      }
      // earlier pivots: t_j -= sum_{i in blk} L[i, j] x_i  (thread per column j < b)
      for (int j = threadIdx.x; j < b; j += blockDim.x) {
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const double* Lj = P + static_cast<std::int64_t>(j) * m + b;
        for (int i = 0; i < bs; ++i) {
          const double l = Lj[i];
#pragma unroll
          for (int r = 0; r < 8; ++r)
            if (r < rr) acc[r] += l * zb[i * 8 + r];
        }
#pragma unroll
        for (int r = 0; r < 8; ++r)
          if (r < rr) t[j * R + r] -= acc[r];
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < k; i += blockDim.x)
      for (int r = 0; r < rr; ++r) x[d.first + pl[i] + (r0 + r) * n] = t[i * R + r];
  }
}

// ---------------------------------------------------------------- cooperative sweeps (few large fronts)
//
// The fronts of a level share the grid (front f owns CTAs [cta_start[f], cta_start[f+1])); the
// front's right-hand sides live in a global work vector t (m rows x 8 columns, column-major with
// leading dimension m). Each block step of <= 32 pivots is one grid barrier: every CTA of the front
// recomputes the block's 32 x 32 product from t (loaded past L1, since other CTAs wrote it) and
// updates its share of the rows (forward) or columns (backward) that depend on it.

namespace {

__device__ __forceinline__ int front_of(const std::int32_t* cta_start, int nfronts) {
  int f = 0;
  while (f + 1 < nfronts && cta_start[f + 1] <= static_cast<int>(blockIdx.x)) ++f;
  return f;
}

}  // namespace

__global__ void __launch_bounds__(256) k_solve_fwd_coop(const std::int32_t* list, const std::int32_t* cta_start,
                                                         int nfronts, int max_steps, const SnDev* sn,
                                                         const std::int32_t* child_ptr,
                                                         const std::int32_t* children, const std::int32_t* rmap,
                                                         const double* panels, const std::int32_t* pidx,
                                                         const std::int32_t* blk, const std::int32_t* nblk,
                                                         const double* inv, double* x, std::int64_t n, double* vec,
                                                         int nrhs, double* work, const std::int64_t* work_off) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ double zb[32 * 8];
  const int f = front_of(cta_start, nfronts);
  const int rank = static_cast<int>(blockIdx.x) - cta_start[f];
  const int nr = cta_start[f + 1] - cta_start[f];
  const int s = list[f];
  const SnDev d = sn[s];
  const int m = d.m, k = d.k, c = m - k;
  double* t = work + work_off[f];  // t[r * m + i]
  const double* P = panels + d.panel_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* bst = blk + d.first;
  const int nb = nblk[s];
  const double* Linv = inv + d.inv_off;
  const int gt = rank * blockDim.x + threadIdx.x, gs = nr * blockDim.x;
  // gather: pivot rows from x, zero elsewhere; rank 0 then adds the children's contributions
  int* invp = reinterpret_cast<int*>(t + static_cast<std::int64_t>(8) * m);
  for (int i = gt; i < m; i += gs)
    for (int r = 0; r < nrhs; ++r) t[r * m + i] = i < k ? x[d.first + pl[i] + static_cast<std::int64_t>(r) * n] : 0.0;
  for (int i = gt; i < k; i += gs) invp[pl[i]] = i;
  grid.sync();
  if (rank == 0) {
    for (int q = child_ptr[s]; q < child_ptr[s + 1]; ++q) {
      const SnDev cd = sn[children[q]];
      const int mc = cd.m - cd.k;
      const std::int32_t* rm = rmap + cd.rmap_off;
      const double* cv = vec + cd.vec_off * nrhs;
      for (int a = threadIdx.x; a < mc; a += blockDim.x) {
        const int pos = rm[a];
        const int row = pos < k ? __ldcg(&invp[pos]) : pos;
        for (int r = 0; r < nrhs; ++r) t[r * m + row] = __ldcg(&t[r * m + row]) + cv[a + static_cast<std::int64_t>(r) * mc];
      }
      __syncthreads();
    }
  }
  grid.sync();
  for (int step = 0; step < max_steps; ++step) {
    if (step < nb) {
      const int b = bst[step];
      const int be = step + 1 < nb ? bst[step + 1] : k;
      const int bs = be - b;
      const double* Li = Linv + static_cast<std::int64_t>(step) * 1024;
      {
        const int i = threadIdx.x % 32, r = threadIdx.x / 32;
        if (i < bs && r < nrhs) {
          double acc = 0.0;
          for (int cc = 0; cc <= i; ++cc) acc += Li[cc * 32 + i] * __ldcg(&t[r * m + b + cc]);
          zb[i * 8 + r] = acc;
        }
      }
      __syncthreads();
      if (rank == 0) {
        const int i = threadIdx.x % 32, r = threadIdx.x / 32;
        if (i < bs && r < nrhs) x[d.first + pl[b + i] + static_cast<std::int64_t>(r) * n] = zb[i * 8 + r];
      }
      for (int i = be + gt; i < m; i += gs) {
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const double* Li0 = P + i + static_cast<std::int64_t>(b) * m;
#pragma unroll 8
        for (int j = 0; j < bs; ++j) {
          const double l = Li0[static_cast<std::int64_t>(j) * m];
#pragma unroll
          for (int r = 0; r < 8; ++r) acc[r] = fma(l, zb[j * 8 + r], acc[r]);
        }
        for (int r = 0; r < nrhs; ++r) t[r * m + i] -= acc[r];
      }
    }
    grid.sync();
  }
  double* v = vec + d.vec_off * nrhs;
  for (int a = gt; a < c; a += gs)
    for (int r = 0; r < nrhs; ++r) v[a + static_cast<std::int64_t>(r) * c] = __ldcg(&t[r * m + k + a]);
}

__global__ void __launch_bounds__(256) k_solve_bwd_coop(const std::int32_t* list, const std::int32_t* cta_start,
                                                         int nfronts, int max_steps, const SnDev* sn,
                                                         const std::int32_t* rows, const double* panels,
                                                         const std::int32_t* pidx, const std::int32_t* blk,
                                                         const std::int32_t* nblk, const double* inv, double* x,
                                                         std::int64_t n, int nrhs, double* work,
                                                         const std::int64_t* work_off) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ double zb[32 * 8];
  const int f = front_of(cta_start, nfronts);
  const int rank = static_cast<int>(blockIdx.x) - cta_start[f];
  const int nr = cta_start[f + 1] - cta_start[f];
  const int s = list[f];
  const SnDev d = sn[s];
  const int m = d.m, k = d.k;
  double* t = work + work_off[f];
  const double* P = panels + d.panel_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* rw = rows + d.rows_off;
  const std::int32_t* bst = blk + d.first;
  const int nb = nblk[s];
  const double* Linv = inv + d.inv_off;
  const int gt = rank * blockDim.x + threadIdx.x, gs = nr * blockDim.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = rank * (blockDim.x >> 5) + warp, gws = nr * (blockDim.x >> 5);
  for (int i = gt; i < m; i += gs)
    for (int r = 0; r < nrhs; ++r)
      t[r * m + i] = i < k ? x[d.first + pl[i] + static_cast<std::int64_t>(r) * n] : x[rw[i] + static_cast<std::int64_t>(r) * n];
  grid.sync();
  // contributions of the contribution-block rows: warp per pivot column, lanes over rows
  for (int j = gw; j < k; j += gws) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const double* Lj = P + static_cast<std::int64_t>(j) * m;
    for (int i = k + lane; i < m; i += 32) {
      const double l = Lj[i];
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < nrhs) acc[r] = fma(l, __ldcg(&t[r * m + i]), acc[r]);
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      if (r >= nrhs) break;
      const double sum = warp_sum(acc[r]);
      if (lane == 0) t[r * m + j] -= sum;
    }
  }
  grid.sync();
  for (int step = 0; step < max_steps; ++step) {
    const int bi = nb - 1 - step;
    if (bi >= 0) {
      const int b = bst[bi];
      const int be = bi + 1 < nb ? bst[bi + 1] : k;
      const int bs = be - b;
      const double* Li = Linv + static_cast<std::int64_t>(bi) * 1024;
      {
        const int cc = threadIdx.x % 32, r = threadIdx.x / 32;
        if (cc < bs && r < nrhs) {
          double acc = 0.0;
          for (int i = cc; i < bs; ++i) acc += Li[cc * 32 + i] * __ldcg(&t[r * m + b + i]);
          zb[cc * 8 + r] = acc;
        }
      }
      __syncthreads();
      if (rank == 0) {
        const int cc = threadIdx.x % 32, r = threadIdx.x / 32;
        if (cc < bs && r < nrhs) x[d.first + pl[b + cc] + static_cast<std::int64_t>(r) * n] = zb[cc * 8 + r];
      }
      // earlier pivots j < b: warp per column, lanes over the block's rows (contiguous in the column)
      for (int j = gw; j < b; j += gws) {
        const double l = lane < bs ? P[b + lane + static_cast<std::int64_t>(j) * m] : 0.0;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          if (r >= nrhs) break;
          const double sum = warp_sum(l * zb[(lane < bs ? lane : 0) * 8 + r]);
          if (lane == 0) t[r * m + j] -= sum;
        }
      }
    }
    grid.sync();
  }
}

void launch_gather_scale(std::int64_t n, int nrhs, const double* b, std::int64_t ldb, const double* d,
                         const std::int32_t* iperm, double* x, cudaStream_t s) {
  const std::int64_t total = n * nrhs;
  const int blocks = static_cast<int>(std::min<std::int64_t>((total + 255) / 256, 148 * 16));
  note_launches(1);
  k_gather_scale<<<blocks, 256, 0, s>>>(n, nrhs, b, ldb, d, iperm, x);
}

void launch_scatter_scale(std::int64_t n, int nrhs, double* b, std::int64_t ldb, const double* d,
                          const std::int32_t* iperm, const double* x, cudaStream_t s) {
  const std::int64_t total = n * nrhs;
  const int blocks = static_cast<int>(std::min<std::int64_t>((total + 255) / 256, 148 * 16));
  note_launches(1);
  k_scatter_scale<<<blocks, 256, 0, s>>>(n, nrhs, b, ldb, d, iperm, x);
}

static std::size_t solve_smem(int maxm, int R) {
  return static_cast<std::size_t>(maxm) * R * sizeof(double) + static_cast<std::size_t>(maxm) * sizeof(int);
}

int solve_rhs_chunk(int maxm, int nrhs) {
  int R = nrhs < 8 ? nrhs : 8;  // the kernels carry at most 8 right-hand sides
  while (R > 1 && solve_smem(maxm, R) > kSolveSmemMax) --R;
  return R < 1 ? 1 : R;
}

void launch_inv_blocks(int ns, const SnDev* sn, const double* panels, const signed char* piv, std::int32_t* blk,
                       std::int32_t* nblk, double* inv, cudaStream_t s) {
  if (ns <= 0) return;
  note_launches(1);
  k_inv_blocks<<<ns, 256, 0, s>>>(sn, panels, piv, blk, nblk, inv);
}

void launch_solve_fwd(const std::int32_t* list, int nlist, int maxm, const SnDev* sn, const std::int32_t* child_ptr,
                      const std::int32_t* children, const std::int32_t* rmap, const double* panels,
                      const signed char* piv, const std::int32_t* pidx, const std::int32_t* blk,
                      const std::int32_t* nblk, const double* inv, double* x, std::int64_t n, double* vec, int nrhs,
                      cudaStream_t s) {
  if (nlist <= 0) return;
  const int R = solve_rhs_chunk(maxm, nrhs);
  const std::size_t smem = solve_smem(maxm, R);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_solve_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSolveSmemMax));
    configured = true;
  }
  note_launches(1);
  k_solve_fwd<<<nlist, 256, smem, s>>>(list, sn, child_ptr, children, rmap, panels, piv, pidx, blk, nblk, inv, x, n,
                                       vec, nrhs, R);
}

void launch_solve_diag(int ns, const SnDev* sn, const double* panels, const signed char* piv,
                       const std::int32_t* pidx, double* x, std::int64_t n, int nrhs, cudaStream_t s) {
  if (ns <= 0) return;
  note_launches(1);
  k_solve_diag<<<ns, 128, 0, s>>>(sn, panels, piv, pidx, x, n, nrhs);
}

void launch_solve_bwd(const std::int32_t* list, int nlist, int maxm, const SnDev* sn, const std::int32_t* rows,
                      const double* panels, const std::int32_t* pidx, const std::int32_t* blk,
                      const std::int32_t* nblk, const double* inv, double* x, std::int64_t n, int nrhs,
                      cudaStream_t s) {
  if (nlist <= 0) return;
  const int R = solve_rhs_chunk(maxm, nrhs);
  const std::size_t smem = solve_smem(maxm, R);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_solve_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSolveSmemMax));
    configured = true;
  }
  note_launches(1);
  k_solve_bwd<<<nlist, 256, smem, s>>>(list, sn, rows, panels, pidx, blk, nblk, inv, x, n, nrhs, R);
}

int solve_coop_max_ctas(int device) {
  int a = 0, b = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_solve_fwd_coop, 256, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_solve_bwd_coop, 256, 0);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return (a < b ? a : b) * sms;
}

cudaError_t launch_solve_fwd_coop(const std::int32_t* list, const std::int32_t* cta_start, int nfronts, int nctas,
                                  int max_steps, const SnDev* sn, const std::int32_t* child_ptr,
                                  const std::int32_t* children, const std::int32_t* rmap, const double* panels,
                                  const std::int32_t* pidx, const std::int32_t* blk, const std::int32_t* nblk,
                                  const double* inv, double* x, std::int64_t n, double* vec, int nrhs, double* work,
                                  const std::int64_t* work_off, cudaStream_t s) {
  void* args[] = {&list, &cta_start, &nfronts, &max_steps, &sn, &child_ptr, &children, &rmap, &panels, &pidx, &blk,
                  &nblk, &inv, &x, &n, &vec, &nrhs, &work, &work_off};
  note_launches(1);
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_solve_fwd_coop), dim3(nctas), dim3(256), args, 0, s);
}

cudaError_t launch_solve_bwd_coop(const std::int32_t* list, const std::int32_t* cta_start, int nfronts, int nctas,
                                  int max_steps, const SnDev* sn, const std::int32_t* rows, const double* panels,
                                  const std::int32_t* pidx, const std::int32_t* blk, const std::int32_t* nblk,
                                  const double* inv, double* x, std::int64_t n, int nrhs, double* work,
                                  const std::int64_t* work_off, cudaStream_t s) {
  void* args[] = {&list, &cta_start, &nfronts, &max_steps, &sn, &rows, &panels, &pidx, &blk, &nblk, &inv, &x, &n,
                  &nrhs, &work, &work_off};
  note_launches(1);
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_solve_bwd_coop), dim3(nctas), dim3(256), args, 0, s);
}

}  // namespace hsg
