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
#include <mutex>

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
template <class F>
__global__ void __launch_bounds__(256) k_inv_blocks(const SnDev* sn, const F* panels, const signed char* piv,
                                                     std::int32_t* blk, std::int32_t* nblk, F* inv) {
  __shared__ int starts[kMaxBlocksPerFront];
  __shared__ int nb;
  const int s = blockIdx.x;
  const SnDev d = sn[s];
  if (d.w_off >= 0) return;  // large fronts are solved through their super-block operator
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
  const F* P = panels + d.panel_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int bi = warp; bi < nb; bi += nwarps) {
    const int b = starts[bi];
    const int bs = bi + 1 < nb ? starts[bi + 1] - b : k - b;
    F* out = inv + d.inv_off + static_cast<std::int64_t>(bi) * 1024;
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
    for (int i = 0; i < 32; ++i) out[lane * 32 + i] = static_cast<F>((lane < bs) ? x[i] : 0.0);
  }
}

// Forward sweep of the listed fronts. t (m x R, row-major) in dynamic shared memory.
template <class F>
__global__ void __launch_bounds__(256) k_solve_fwd(const std::int32_t* list, const SnDev* sn,
                                                    const std::int32_t* child_ptr, const std::int32_t* children,
                                                    const std::int32_t* rmap, const F* panels,
                                                    const signed char* piv, const std::int32_t* pidx,
                                                    const std::int32_t* blk, const std::int32_t* nblk,
                                                    const F* inv, double* x, std::int64_t n, double* vec,
                                                    int nrhs, int R) {
  extern __shared__ double smem[];
  __shared__ double zb[32 * 8];
  const int s = list[blockIdx.x];
  const SnDev d = sn[s];
  const int m = d.m, k = d.k, c = m - k;
  double* t = smem;
  int* invp = reinterpret_cast<int*>(smem + static_cast<std::int64_t>(m) * R);
  const F* P = panels + d.panel_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* bst = blk + d.first;
  const int nb = nblk[s];
  const F* Linv = inv + d.inv_off;
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
      const F* Li = Linv + static_cast<std::int64_t>(bi) * 1024;
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
template <class F>
__global__ void k_solve_diag(const SnDev* sn, const F* panels, const signed char* piv, const std::int32_t* pidx,
                             double* x, std::int64_t n, int nrhs) {
  const SnDev d = sn[blockIdx.x];
  const F* P = panels + d.panel_off;
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

// Diagonal solve D y = z over all pivots at once (one thread per pivot position p): dpos[p] is the
// panel index of D(p, p), pfirst[p] the first global column of p's front.
template <class F>
__global__ void k_solve_diag_flat(std::int64_t npiv, const std::int64_t* dpos, const std::int32_t* pfirst,
                                  const F* panels, const signed char* piv, const std::int32_t* pidx, double* x,
                                  std::int64_t n, int nrhs) {
  const std::int64_t p = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= npiv) return;
  const signed char ty = piv[p];
  if (ty == 3) return;
  const std::int64_t g0 = pfirst[p] + pidx[p];
  if (ty <= 0) {
    for (int r = 0; r < nrhs; ++r) x[g0 + r * n] = 0.0;
  } else if (ty == 1) {
    const double dj = panels[dpos[p]];
    for (int r = 0; r < nrhs; ++r) x[g0 + r * n] /= dj;
  } else {
    const std::int64_t g1 = pfirst[p] + pidx[p + 1];
    const double a = panels[dpos[p]], b = panels[dpos[p] + 1], c = panels[dpos[p + 1]];
    const double det = a * c - b * b;
    for (int r = 0; r < nrhs; ++r) {
      const double y0 = x[g0 + r * n], y1 = x[g1 + r * n];
      x[g0 + r * n] = (c * y0 - b * y1) / det;
      x[g1 + r * n] = (-b * y0 + a * y1) / det;
    }
  }
}

// Backward sweep of the listed fronts (ancestors done): right-looking over the blocks, last first.
template <class F>
__global__ void __launch_bounds__(256) k_solve_bwd(const std::int32_t* list, const SnDev* sn, const std::int32_t* rows,
                                                    const F* panels, const std::int32_t* pidx,
                                                    const std::int32_t* blk, const std::int32_t* nblk,
                                                    const F* inv, double* x, std::int64_t n, int nrhs, int R) {
  extern __shared__ double smem[];
  __shared__ double zb[32 * 8];
  const int s = list[blockIdx.x];
  const SnDev d = sn[s];
  const int m = d.m, k = d.k;
  double* t = smem;
  const F* P = panels + d.panel_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* rw = rows + d.rows_off;
  const std::int32_t* bst = blk + d.first;
  const int nb = nblk[s];
  const F* Linv = inv + d.inv_off;
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
      const F* Lj = P + static_cast<std::int64_t>(j) * m;
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
      const F* Li = Linv + static_cast<std::int64_t>(bi) * 1024;
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
        const F* Lj = P + static_cast<std::int64_t>(j) * m + b;
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
// The large fronts of the top levels are solved by super-blocks of kSB = 128 pivots. For a
// super-block B = [b, b + bs) of a front with unit lower panel L (m x k, the 2 x 2 pivots'
// coupling entries read as zero), the solve uses
//     W[B, B]     = L_BB^{-1}                 (lower triangular, zero above the diagonal)
//     W[i, B]     = L[i, B] L_BB^{-1},  i >= b + bs,
// stored like the panel (column-major, ld m) in a separate buffer and built once per factorization
// before its first solve. Then the forward sweep L z = t is, super-block by super-block,
//     z_B = W[B, B] t_B,     t_i -= W[i, B] t_B  (i below B),
// and the backward sweep L^T x = t is, from the last super-block to the first,
//     x_B = s_B,             s_j -= W[B, j]^T x_B  (every earlier pivot j),
// with s_j initialised to (W[A, A]^T t_A)_j - W[CB rows, j]^T x_CB for j in super-block A. Every
// step of both sweeps is one grid barrier and one read of the W entries it needs; each row (forward)
// or column (backward) is owned by one thread group per step, so no atomics are used and the sums
// are formed in a fixed order.

namespace {

__device__ __forceinline__ int front_of(const std::int32_t* cta_start, int nfronts) {
  int f = 0;
  while (f + 1 < nfronts && cta_start[f + 1] <= static_cast<int>(blockIdx.x)) ++f;
  return f;
}

}  // namespace

// W[B, B] = L_BB^{-1} for one super-block per CTA: row-by-row substitution X[i, c] =
// -sum_{c <= j < i} L[i, j] X[j, c] on packed triangles in shared memory (two threads per column).
template <class F>
__global__ void __launch_bounds__(256) k_sb_inverse(const int2* sbl, const SnDev* sn, const F* panels,
                                                     const signed char* piv, F* W) {
  extern __shared__ double sm[];
  double* Lp = sm;                                // strictly lower rows, row i at i(i-1)/2
  double* Xp = sm + kSB * (kSB - 1) / 2;          // lower rows incl. diagonal, row i at i(i+1)/2
  double* part = Xp + kSB * (kSB + 1) / 2;        // second-half partial sums
  const int2 e = sbl[blockIdx.x];
  const SnDev d = sn[e.x];
  const int m = d.m;
  const int b = e.y * kSB, bs = min(kSB, d.k - b);
  const F* P = panels + d.panel_off;
  const signed char* pv = piv + d.first;
  for (int idx = threadIdx.x; idx < bs * bs; idx += blockDim.x) {
    const int j = idx / bs, i = idx % bs;
    if (i > j) Lp[i * (i - 1) / 2 + j] = (j + 1 == i && pv[b + j] == 2) ? 0.0 : P[(b + i) + static_cast<std::int64_t>(b + j) * m];
  }
  __syncthreads();
  const int c = threadIdx.x & (kSB - 1), h = threadIdx.x / kSB;
  for (int i = 0; i < bs; ++i) {
    double acc = 0.0;
    const double* Li = Lp + i * (i - 1) / 2;
    for (int j = h; j < i; j += 2)
      if (j >= c) acc = fma(Li[j], Xp[j * (j + 1) / 2 + c], acc);
    if (h == 1) part[c] = acc;
    __syncthreads();
    if (h == 0 && c <= i) Xp[i * (i + 1) / 2 + c] = c == i ? 1.0 : -(acc + part[c]);
    __syncthreads();
  }
  F* Wd = W + d.w_off + b + static_cast<std::int64_t>(b) * m;
  for (int idx = threadIdx.x; idx < bs * bs; idx += blockDim.x) {
    const int cc = idx / bs, i = idx % bs;
    Wd[i + static_cast<std::int64_t>(cc) * m] = static_cast<F>(i >= cc ? Xp[i * (i + 1) / 2 + cc] : 0.0);
  }
}

// W[r0 : r0 + 64, B] = L[r0 : r0 + 64, B] W[B, B] for one 64-row tile below a super-block per CTA.
template <class F>
__global__ void __launch_bounds__(256) k_sb_apply(const int4* tiles, const SnDev* sn, const F* panels,
                                                   const signed char* piv, F* W) {
  __shared__ double Ls[32][64];
  __shared__ double Xs[32][kSB];
  const int4 e = tiles[blockIdx.x];
  const SnDev d = sn[e.x];
  const int m = d.m;
  const int b = e.y * kSB, bs = min(kSB, d.k - b), r0 = e.z;
  const F* P = panels + d.panel_off;
  const signed char* pv = piv + d.first;
  F* Wf = W + d.w_off;
  const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;  // rows tr + 16 q, columns tc * 8 + p
  double acc[4][8];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int p = 0; p < 8; ++p) acc[q][p] = 0.0;
  for (int j0 = 0; j0 < bs; j0 += 32) {
    for (int idx = threadIdx.x; idx < 32 * 64; idx += blockDim.x) {
      const int jj = idx / 64, row = idx % 64, i = r0 + row, j = j0 + jj;
      // a 2 x 2 pivot split by the super-block boundary: its coupling entry is D, not L
      const bool coupling = i == b + j + 1 && pv[b + j] == 2;
      Ls[jj][row] = (i < m && j < bs && !coupling) ? P[i + static_cast<std::int64_t>(b + j) * m] : 0.0;
    }
    for (int idx = threadIdx.x; idx < 32 * kSB; idx += blockDim.x) {
      const int cc = idx / 32, jj = idx % 32, j = j0 + jj;
      Xs[jj][cc] = (j < bs && cc < bs) ? Wf[(b + j) + static_cast<std::int64_t>(b + cc) * m] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int jj = 0; jj < 32; ++jj) {
      double a[4], x[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) a[q] = Ls[jj][tr + 16 * q];
#pragma unroll
      for (int p = 0; p < 8; ++p) x[p] = Xs[jj][tc * 8 + p];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int p = 0; p < 8; ++p) acc[q][p] = fma(a[q], x[p], acc[q][p]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = r0 + tr + 16 * q;
    if (i >= m) continue;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int cc = tc * 8 + p;
      if (cc < bs) Wf[i + static_cast<std::int64_t>(b + cc) * m] = static_cast<F>(acc[q][p]);
    }
  }
}

// The sweeps below synchronise their CTAs through per-front publication counters instead of grid
// barriers: every 32-row group (forward) or 32-column chunk (backward) of a front has one owner CTA
// for the whole sweep (group G, chunk c: CTA G mod nr, c mod nr). An owner that finishes the values
// of the next super-block writes them, fences, and adds 1 to the front's counter; a CTA starts a
// super-block step once the counter shows all of that super-block's groups. The waits are bounded:
// a wait that runs out sets *err and the sweep goes on with whatever it reads (the host reports it).

namespace {

constexpr long long kSweepSpinLimit = 1LL << 22;

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// all threads: wait until *cnt >= target (thread 0 polls)
__device__ __forceinline__ void wait_published(const int* cnt, int target, int* err) {
  if (threadIdx.x == 0 && target > 0) {
    long long it = 0;
    while (ld_acquire(cnt) < target) {
      if (++it > kSweepSpinLimit) { atomicExch(err, 1); break; }
      __nanosleep(32);
    }
  }
  __syncthreads();
}

// all threads, after their writes: make them visible, then count one publication
__device__ __forceinline__ void publish(int* cnt) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(cnt, 1);
}

__device__ __forceinline__ int sb_groups(int q, int k) {
  const int bs = min(kSB, k - q * kSB);
  return (bs + 31) / 32;
}

}  // namespace

// Forward sweep of the level's large fronts (front f owns CTAs [cta_start[f], cta_start[f+1])).
// Each CTA first assembles the right-hand sides of its row groups: the pivot rows' entries of x plus
// the children's contribution vectors, listed per front position in child order (cptr / cent).
// In super-block step q the owner of row group G >= 4q forms the group's 32 rows of W[:, B] t_B:
// its 8 warps split the super-block's columns (16 each, lane = row) and add their partial sums in
// shared memory in warp order. Rows of B give z_B (written to x), rows below update t; the CB rows
// write their final values to the front's contribution vector in the last step.
template <class F>
__global__ void __launch_bounds__(256, 2) k_solve_fwd_coop(const std::int32_t* list, const std::int32_t* cta_start,
                                                            int nfronts, const SnDev* sn, const std::int32_t* cptr,
                                                            const ContribEntry* cent, const F* W,
                                                            const std::int32_t* pidx, double* x, std::int64_t n,
                                                            double* vec, int nrhs, double* work,
                                                            const std::int64_t* work_off, int* cnts, int* err) {
  __shared__ double tb[kSB * 8];
  __shared__ double red[8][32][9];
  const int f = front_of(cta_start, nfronts);
  const int rank = static_cast<int>(blockIdx.x) - cta_start[f];
  const int nr = cta_start[f + 1] - cta_start[f];
  const int s = list[f];
  const SnDev d = sn[s];
  const int m = d.m, k = d.k, c = m - k;
  double* t = work + work_off[f];  // t[r * m + i]
  int* cnt = cnts + f;
  const F* Wf = W + d.w_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* cp = cptr + d.cptr_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = threadIdx.x >> 3, rr = threadIdx.x & 7;
  double* v = vec + d.vec_off * nrhs;
  const int nsb = (k + kSB - 1) / kSB;
  const int ngt = (m + 31) / 32;
  // assemble the owned row groups; the groups of super-block 0 are published
  for (int G = rank; G < ngt; G += nr) {
    const int i = G * 32 + row;
    if (i < m && rr < nrhs) {
      const int pos = i < k ? pl[i] : i;
      double val = i < k ? x[d.first + pos + static_cast<std::int64_t>(rr) * n] : 0.0;
      for (int e = cp[pos]; e < cp[pos + 1]; ++e) {
        const ContribEntry ce = cent[e];
        val += vec[ce.vec_off * nrhs + ce.a + static_cast<std::int64_t>(rr) * ce.mc];
      }
      t[rr * m + i] = val;
    }
    if (G < sb_groups(0, k)) publish(cnt);
  }
  int target = 0;
  for (int q = 0; q < nsb; ++q) {
    const int b = q * kSB, be = min(b + kSB, k), bs = be - b;
    target += sb_groups(q, k);
    int G = rank;
    if (G < b / 32) G += ((b / 32 - G + nr - 1) / nr) * nr;
    if (G >= ngt) break;  // no rows left for this CTA
    const bool last = q + 1 == nsb;
    const int nb0 = (q + 1) * (kSB / 32), nb1 = last ? nb0 : nb0 + sb_groups(q + 1, k);
    // prefetch the first group's W entries and the old values it updates (no dependence on the wait)
    const int j0 = warp * 16;
    double wv[16];
    {
      const int i = G * 32 + lane;
#pragma unroll
      for (int jj = 0; jj < 16; ++jj)
        wv[jj] = (i < m && j0 + jj < bs) ? Wf[i + static_cast<std::int64_t>(b + j0 + jj) * m] : 0.0;
    }
    double told = 0.0;
    int plz = 0;
    {
      const int ii = G * 32 + row;
      if (ii >= be && ii < m && rr < nrhs) told = __ldcg(&t[rr * m + ii]);
      if (ii < be) plz = pl[ii];
    }
    wait_published(cnt, target, err);
    for (int idx = threadIdx.x; idx < kSB * 8; idx += blockDim.x) {
      const int j = idx >> 3, r = idx & 7;
      tb[idx] = (j < bs && r < nrhs) ? __ldcg(&t[r * m + b + j]) : 0.0;
    }
    __syncthreads();
    for (bool first = true; G < ngt; G += nr, first = false) {
      const int i = G * 32 + lane;
      if (!first) {
#pragma unroll
        for (int jj = 0; jj < 16; ++jj)
          wv[jj] = (i < m && j0 + jj < bs) ? Wf[i + static_cast<std::int64_t>(b + j0 + jj) * m] : 0.0;
        const int ii = G * 32 + row;
        told = (ii >= be && ii < m && rr < nrhs) ? __ldcg(&t[rr * m + ii]) : 0.0;
        plz = ii < be ? pl[ii] : 0;
      }
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int jj = 0; jj < 16; ++jj)
#pragma unroll
        for (int r = 0; r < 8; ++r) acc[r] = fma(wv[jj], tb[(j0 + jj) * 8 + r], acc[r]);
#pragma unroll
      for (int r = 0; r < 8; ++r) red[warp][lane][r] = acc[r];
      __syncthreads();
      {
        const int ii = G * 32 + row;
        if (ii < m && rr < nrhs) {
          double val = 0.0;
#pragma unroll
          for (int w = 0; w < 8; ++w) val += red[w][row][rr];
          if (ii < be) {
            x[d.first + plz + static_cast<std::int64_t>(rr) * n] = val;
          } else {
            const double nv = told - val;
            if (last && ii >= k) v[(ii - k) + static_cast<std::int64_t>(rr) * c] = nv;
            else t[rr * m + ii] = nv;
          }
        }
      }
      if (G >= nb0 && G < nb1) publish(cnt);  // rows of the next super-block are final
      else __syncthreads();
    }
  }
}

// Backward sweep of the level's large fronts. Columns are owned by groups of 8 lanes (4 per warp,
// 32 consecutive columns per CTA and round); a group reduces its column's dot products over its
// lanes with shuffles. Super-blocks are processed from the last to the first; the owners of the
// next super-block's columns write x there and publish.
template <class F>
__global__ void __launch_bounds__(256, 2) k_solve_bwd_coop(const std::int32_t* list, const std::int32_t* cta_start,
                                                            int nfronts, const SnDev* sn, const std::int32_t* rows,
                                                            const F* W, const std::int32_t* pidx, double* x,
                                                            std::int64_t n, int nrhs, double* work,
                                                            const std::int64_t* work_off, int* cnts, int* err) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ double xb[kSB * 8];
  const int f = front_of(cta_start, nfronts);
  const int rank = static_cast<int>(blockIdx.x) - cta_start[f];
  const int nr = cta_start[f + 1] - cta_start[f];
  const int s = list[f];
  const SnDev d = sn[s];
  const int m = d.m, k = d.k;
  double* t = work + work_off[f];                              // t[r * m + i]
  double* sv = t + static_cast<std::int64_t>(8) * m;           // sv[r * k + j]
  int* cnt = cnts + f;
  const F* Wf = W + d.w_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* rw = rows + d.rows_off;
  const int gt = rank * blockDim.x + threadIdx.x, gs = nr * blockDim.x;
  const int sub = threadIdx.x & 7, gsub = (threadIdx.x >> 3) & 3;
  const int wbase = rank * 32 + (threadIdx.x >> 5) * 4, ngrp = nr * 32;
  const int nsb = (k + kSB - 1) / kSB;
  for (int i = gt; i < m; i += gs)
    for (int r = 0; r < nrhs; ++r)
      t[r * m + i] = i < k ? x[d.first + pl[i] + static_cast<std::int64_t>(r) * n] : x[rw[i] + static_cast<std::int64_t>(r) * n];
  grid.sync();
  // sv_j = (W[A, A]^T t_A)_j - W[k:m, j]^T t[k:m] for j in super-block A, 128-row chunks of t
  // staged in shared memory (W is zero above the diagonal of W[A, A]); the last super-block's x
  // is final already. Rounds c0 are 32-column chunks, uniform over the CTA.
  const int blast = (nsb - 1) * kSB;
  for (int c0 = rank * 32; c0 < k; c0 += ngrp) {
    const int j = c0 + (threadIdx.x >> 3);
    const int bA = (c0 / kSB) * kSB;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i0 = bA, chunk = 0; i0 < m; ++chunk) {
      const int i1 = chunk == 0 ? min(bA + kSB, k) : min(i0 + kSB, m);
      const double sg = chunk == 0 ? 1.0 : -1.0;
      double wv[16];
      const F* Wj = Wf + i0 + static_cast<std::int64_t>(j) * m;
#pragma unroll
      for (int u = 0; u < 16; ++u) wv[u] = (j < k && i0 + sub + 8 * u < i1) ? sg * Wj[sub + 8 * u] : 0.0;
      __syncthreads();
      for (int idx = threadIdx.x; idx < kSB * 8; idx += blockDim.x) {
        const int r = idx / kSB, i = idx % kSB;
        xb[idx] = (i0 + i < i1 && r < nrhs) ? __ldcg(&t[r * m + i0 + i]) : 0.0;
      }
      __syncthreads();
#pragma unroll
      for (int u = 0; u < 16; ++u)
#pragma unroll
        for (int r = 0; r < 8; ++r) acc[r] = fma(wv[u], xb[r * kSB + sub + 8 * u], acc[r]);
      i0 = chunk == 0 ? k : i1;
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 4);
      acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 2);
      acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 1);
    }
    if (j < k && sub < nrhs) {
      double a = acc[0];
#pragma unroll
      for (int r = 1; r < 8; ++r)
        if (sub == r) a = acc[r];
      sv[sub * k + j] = a;
      if (j >= blast) x[d.first + pl[j] + static_cast<std::int64_t>(sub) * n] = a;
    }
    if (c0 >= blast) publish(cnt);  // this CTA's 32 columns of the last super-block are final
    else __syncthreads();
  }
  int target = 0;
  for (int step = 0; step < nsb; ++step) {
    const int q = nsb - 1 - step;
    const int b = q * kSB, be = min(b + kSB, k), bs = be - b;
    target += sb_groups(q, k);
    if (wbase >= b) break;  // no columns left for this CTA (uniform: b is a multiple of 32)
    const int bprev = b - kSB;  // columns of the next super-block: [bprev, b)
    // the CTA's column chunks below b are updated from the highest down: the next super-block's
    // columns (the highest ones) are finished and published first, so the next step can start
    // while the rest of the update runs (every column has one owner, so nothing else reads it)
    const int top = wbase + ((b - 1 - wbase) / ngrp) * ngrp;  // uniform over the CTA
    // prefetch the first column's W entries and old value
    int j = top + gsub;
    double wv[16];
    {
      const F* Wj = Wf + b + static_cast<std::int64_t>(j) * m;
#pragma unroll
      for (int u = 0; u < 16; ++u) wv[u] = (j < b && sub + 8 * u < bs) ? Wj[sub + 8 * u] : 0.0;
    }
    double sold = (j < b && sub < nrhs) ? __ldcg(&sv[sub * k + j]) : 0.0;
    int plj = (j < b && j >= bprev) ? pl[j] : 0;
    wait_published(cnt, target, err);
    for (int idx = threadIdx.x; idx < kSB * 8; idx += blockDim.x) {
      const int r = idx / kSB, i = idx % kSB;  // xb[r * kSB + i]: conflict-free reads below
      xb[idx] = (i < bs && r < nrhs) ? __ldcg(&sv[r * k + b + i]) : 0.0;
    }
    __syncthreads();
    for (int base = top; base >= wbase; base -= ngrp) {
      j = base + gsub;
      if (base != top) {
        const F* Wj = Wf + b + static_cast<std::int64_t>(j) * m;
#pragma unroll
        for (int u = 0; u < 16; ++u) wv[u] = (j < b && sub + 8 * u < bs) ? Wj[sub + 8 * u] : 0.0;
        sold = (j < b && sub < nrhs) ? __ldcg(&sv[sub * k + j]) : 0.0;
        plj = (j < b && j >= bprev) ? pl[j] : 0;
      }
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int u = 0; u < 16; ++u)
#pragma unroll
        for (int r = 0; r < 8; ++r) acc[r] = fma(wv[u], xb[r * kSB + sub + 8 * u], acc[r]);
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 4);
        acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 2);
        acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 1);
      }
      if (j < b && sub < nrhs) {
        double a = acc[0];
#pragma unroll
        for (int r = 1; r < 8; ++r)
          if (sub == r) a = acc[r];
        const double nv = sold - a;
        sv[sub * k + j] = nv;
        if (j >= bprev) x[d.first + plj + static_cast<std::int64_t>(sub) * n] = nv;
      }
      if (base >= bprev) publish(cnt);  // this CTA's 32 columns of the next super-block are final
      else __syncthreads();
    }
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

template <class F>
void launch_inv_blocks(int ns, const SnDev* sn, const F* panels, const signed char* piv, std::int32_t* blk,
                       std::int32_t* nblk, F* inv, cudaStream_t s) {
  if (ns <= 0) return;
  note_launches(1);
  k_inv_blocks<F><<<ns, 256, 0, s>>>(sn, panels, piv, blk, nblk, inv);
}

template <class F>
void launch_solve_fwd(const std::int32_t* list, int nlist, int maxm, const SnDev* sn, const std::int32_t* child_ptr,
                      const std::int32_t* children, const std::int32_t* rmap, const F* panels,
                      const signed char* piv, const std::int32_t* pidx, const std::int32_t* blk,
                      const std::int32_t* nblk, const F* inv, double* x, std::int64_t n, double* vec, int nrhs,
                      cudaStream_t s) {
  if (nlist <= 0) return;
  const int R = solve_rhs_chunk(maxm, nrhs);
  const std::size_t smem = solve_smem(maxm, R);
  static std::once_flag configured;
  std::call_once(configured, [&] {
    cudaFuncSetAttribute(k_solve_fwd<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSolveSmemMax));
  });
  note_launches(1);
  k_solve_fwd<F><<<nlist, 256, smem, s>>>(list, sn, child_ptr, children, rmap, panels, piv, pidx, blk, nblk, inv, x, n,
                                          vec, nrhs, R);
}

template <class F>
void launch_solve_diag_flat(std::int64_t npiv, const std::int64_t* dpos, const std::int32_t* pfirst, const F* panels,
                            const signed char* piv, const std::int32_t* pidx, double* x, std::int64_t n, int nrhs,
                            cudaStream_t s) {
  if (npiv <= 0) return;
  note_launches(1);
  k_solve_diag_flat<F><<<static_cast<unsigned>((npiv + 255) / 256), 256, 0, s>>>(npiv, dpos, pfirst, panels, piv, pidx,
                                                                                x, n, nrhs);
}

template <class F>
void launch_solve_diag(int ns, const SnDev* sn, const F* panels, const signed char* piv, const std::int32_t* pidx,
                       double* x, std::int64_t n, int nrhs, cudaStream_t s) {
  if (ns <= 0) return;
  note_launches(1);
  k_solve_diag<F><<<ns, 128, 0, s>>>(sn, panels, piv, pidx, x, n, nrhs);
}

template <class F>
void launch_solve_bwd(const std::int32_t* list, int nlist, int maxm, const SnDev* sn, const std::int32_t* rows,
                      const F* panels, const std::int32_t* pidx, const std::int32_t* blk, const std::int32_t* nblk,
                      const F* inv, double* x, std::int64_t n, int nrhs, cudaStream_t s) {
  if (nlist <= 0) return;
  const int R = solve_rhs_chunk(maxm, nrhs);
  const std::size_t smem = solve_smem(maxm, R);
  static std::once_flag configured;
  std::call_once(configured, [&] {
    cudaFuncSetAttribute(k_solve_bwd<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSolveSmemMax));
  });
  note_launches(1);
  k_solve_bwd<F><<<nlist, 256, smem, s>>>(list, sn, rows, panels, pidx, blk, nblk, inv, x, n, nrhs, R);
}

namespace {
template <class F>
int solve_coop_max_of(int device) {
  int a = 0, b = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_solve_fwd_coop<F>, 256, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_solve_bwd_coop<F>, 256, 0);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return (a < b ? a : b) * sms;
}
}  // namespace

// co-resident CTAs of the cooperative sweeps, valid for both factor types
int solve_coop_max_ctas(int device) {
  const int a = solve_coop_max_of<double>(device), b = solve_coop_max_of<float>(device);
  return a < b ? a : b;
}

template <class F>
void launch_sb_build(const int2* sbl, int nsb, const int4* tiles, int ntiles, const SnDev* sn, const F* panels,
                     const signed char* piv, F* W, cudaStream_t s) {
  if (nsb <= 0) return;
  constexpr std::size_t smem = sizeof(double) * (kSB * (kSB - 1) / 2 + kSB * (kSB + 1) / 2 + kSB);
  static std::once_flag configured;
  std::call_once(configured, [&] {
    cudaFuncSetAttribute(k_sb_inverse<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  });
  note_launches(1);
  k_sb_inverse<F><<<nsb, 256, smem, s>>>(sbl, sn, panels, piv, W);
  if (ntiles > 0) {
    note_launches(1);
    k_sb_apply<F><<<ntiles, 256, 0, s>>>(tiles, sn, panels, piv, W);
  }
}

template <class F>
cudaError_t launch_solve_fwd_coop(const std::int32_t* list, const std::int32_t* cta_start, int nfronts, int nctas,
                                  const SnDev* sn, const std::int32_t* cptr, const ContribEntry* cent, const F* W,
                                  const std::int32_t* pidx, double* x, std::int64_t n, double* vec, int nrhs,
                                  double* work, const std::int64_t* work_off, int* cnts, int* err, cudaStream_t s) {
  void* args[] = {&list, &cta_start, &nfronts, &sn, &cptr, &cent, &W, &pidx, &x, &n, &vec, &nrhs, &work, &work_off,
                  &cnts, &err};
  note_launches(1);
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_solve_fwd_coop<F>), dim3(nctas), dim3(256), args, 0, s);
}

template <class F>
cudaError_t launch_solve_bwd_coop(const std::int32_t* list, const std::int32_t* cta_start, int nfronts, int nctas,
                                  const SnDev* sn, const std::int32_t* rows, const F* W, const std::int32_t* pidx,
                                  double* x, std::int64_t n, int nrhs, double* work, const std::int64_t* work_off,
                                  int* cnts, int* err, cudaStream_t s) {
  void* args[] = {&list, &cta_start, &nfronts, &sn, &rows, &W, &pidx, &x, &n, &nrhs, &work, &work_off, &cnts, &err};
  note_launches(1);
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_solve_bwd_coop<F>), dim3(nctas), dim3(256), args, 0, s);
}

#define HSG_SOLVE_INSTANTIATE(F)                                                                                       \
  template void launch_inv_blocks<F>(int, const SnDev*, const F*, const signed char*, std::int32_t*, std::int32_t*,   \
                                     F*, cudaStream_t);                                                                \
  template void launch_solve_fwd<F>(const std::int32_t*, int, int, const SnDev*, const std::int32_t*,                 \
                                    const std::int32_t*, const std::int32_t*, const F*, const signed char*,            \
                                    const std::int32_t*, const std::int32_t*, const std::int32_t*, const F*, double*,  \
                                    std::int64_t, double*, int, cudaStream_t);                                         \
  template void launch_solve_diag_flat<F>(std::int64_t, const std::int64_t*, const std::int32_t*, const F*,          \
                                          const signed char*, const std::int32_t*, double*, std::int64_t, int,        \
                                          cudaStream_t);                                                               \
  template void launch_solve_diag<F>(int, const SnDev*, const F*, const signed char*, const std::int32_t*, double*,   \
                                     std::int64_t, int, cudaStream_t);                                                 \
  template void launch_solve_bwd<F>(const std::int32_t*, int, int, const SnDev*, const std::int32_t*, const F*,      \
                                    const std::int32_t*, const std::int32_t*, const std::int32_t*, const F*, double*,  \
                                    std::int64_t, int, cudaStream_t);                                                  \
  template void launch_sb_build<F>(const int2*, int, const int4*, int, const SnDev*, const F*, const signed char*,    \
                                   F*, cudaStream_t);                                                                  \
  template cudaError_t launch_solve_fwd_coop<F>(const std::int32_t*, const std::int32_t*, int, int, const SnDev*,    \
                                                const std::int32_t*, const ContribEntry*, const F*,                    \
                                                const std::int32_t*, double*, std::int64_t, double*, int, double*,      \
                                                const std::int64_t*, int*, int*, cudaStream_t);                        \
  template cudaError_t launch_solve_bwd_coop<F>(const std::int32_t*, const std::int32_t*, int, int, const SnDev*,    \
                                                const std::int32_t*, const F*, const std::int32_t*, double*,            \
                                                std::int64_t, int, double*, const std::int64_t*, int*, int*,            \
                                                cudaStream_t);
HSG_SOLVE_INSTANTIATE(double)
HSG_SOLVE_INSTANTIATE(float)
#undef HSG_SOLVE_INSTANTIATE

}  // namespace hsg
