// Supernodal forward / diagonal / backward solves with nrhs right-hand sides (replaces MUMPS JOB=3,
// hsolve src/factor/mumps_factorization.cpp:459-527; MUMPS dsol_fwd.F / dsol_bwd.F).
//
// The forward sweep runs level by level like the factorization: a front gathers its pivot rows from
// the solution vector and its children's contribution vectors (fixed order, no atomics, so results
// are bitwise reproducible), solves with its unit-lower L11 in blocks of at most 32 columns (never
// splitting a 2x2 pivot), and leaves its contribution -L21 z for the parent. The backward sweep
// runs top-down and only gathers (ancestors' values are final). All right-hand sides of a chunk
// are carried together so that every L entry is read once per chunk.
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

// Forward sweep of the listed fronts. t (m x R, row-major) in dynamic shared memory.
__global__ void __launch_bounds__(256) k_solve_fwd(const std::int32_t* list, const SnDev* sn,
                                                    const std::int32_t* child_ptr, const std::int32_t* children,
                                                    const std::int32_t* rmap, const double* panels,
                                                    const signed char* piv, const std::int32_t* pidx, double* x,
                                                    std::int64_t n, double* vec, int nrhs, int R) {
  extern __shared__ double smem[];
  const int s = list[blockIdx.x];
  const SnDev d = sn[s];
  const int m = d.m, k = d.k, c = m - k;
  double* t = smem;
  int* invp = reinterpret_cast<int*>(smem + static_cast<std::int64_t>(m) * R);
  const double* P = panels + d.panel_off;
  const signed char* pv = piv + d.first;
  const std::int32_t* pl = pidx + d.first;
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
    // blocked forward substitution
    for (int b = 0; b < k;) {
      const int bs = block_size_at(pv, b, k);
      if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        for (int j = b; j < b + bs; ++j) {
          const signed char ty = pv[j];
          if (ty == 3) continue;
          const double* Lj = P + static_cast<std::int64_t>(j) * m;
          if (ty == 2) {
            const double* Lj1 = Lj + m;
            for (int i = j + 2 + lane; i < b + bs; i += 32)
              for (int r = 0; r < rr; ++r) t[i * R + r] -= Lj[i] * t[j * R + r] + Lj1[i] * t[(j + 1) * R + r];
          } else {
            for (int i = j + 1 + lane; i < b + bs; i += 32)
              for (int r = 0; r < rr; ++r) t[i * R + r] -= Lj[i] * t[j * R + r];
          }
          __syncwarp();
        }
      }
      __syncthreads();
      for (int i = b + bs + threadIdx.x; i < m; i += blockDim.x) {
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = b; j < b + bs; ++j) {
          const double l = P[i + static_cast<std::int64_t>(j) * m];
          for (int r = 0; r < rr && r < 8; ++r) acc[r] += l * t[j * R + r];
        }
        for (int r = 0; r < rr && r < 8; ++r) t[i * R + r] -= acc[r];
      }
      __syncthreads();
      b += bs;
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

// Backward sweep of the listed fronts (ancestors done).
__global__ void __launch_bounds__(256) k_solve_bwd(const std::int32_t* list, const SnDev* sn, const std::int32_t* rows,
                                                    const double* panels, const signed char* piv,
                                                    const std::int32_t* pidx, double* x, std::int64_t n, int nrhs,
                                                    int R) {
  extern __shared__ double smem[];
  __shared__ int blocks[1024];
  __shared__ int nblocks;
  const SnDev d = sn[list[blockIdx.x]];
  const int m = d.m, k = d.k;
  double* t = smem;
  const double* P = panels + d.panel_off;
  const signed char* pv = piv + d.first;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* rw = rows + d.rows_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  if (threadIdx.x == 0) {
    int nb = 0;
    for (int b = 0; b < k;) { const int bs = block_size_at(pv, b, k); if (nb < 1024) blocks[nb++] = b; b += bs; }
    nblocks = nb;
  }
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
    // t_j -= sum_{i >= k} L[i, j] t_i  (warp per column)
    for (int j = warp; j < k; j += nwarps) {
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      const double* Lj = P + static_cast<std::int64_t>(j) * m;
      for (int i = k + lane; i < m; i += 32) {
        const double l = Lj[i];
        for (int r = 0; r < rr && r < 8; ++r) acc[r] += l * t[i * R + r];
      }
      for (int r = 0; r < rr && r < 8; ++r) {
        const double s = warp_sum(acc[r]);
        if (lane == 0) t[j * R + r] -= s;
      }
    }
    __syncthreads();
    for (int bi = nblocks - 1; bi >= 0; --bi) {
      const int b = blocks[bi];
      const int be = bi + 1 < nblocks ? blocks[bi + 1] : k;
      // contributions of the pivots after this block (already solved)
      for (int j = b + warp; j < be; j += nwarps) {
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const double* Lj = P + static_cast<std::int64_t>(j) * m;
        for (int i = be + lane; i < k; i += 32) {
          const double l = Lj[i];
          for (int r = 0; r < rr && r < 8; ++r) acc[r] += l * t[i * R + r];
        }
        for (int r = 0; r < rr && r < 8; ++r) {
          const double s = warp_sum(acc[r]);
          if (lane == 0) t[j * R + r] -= s;
        }
      }
      __syncthreads();
      if (warp == 0) {
        for (int j = be - 1; j >= b; --j) {
          const signed char ty = pv[j];
          if (ty == 2) continue;  // handled with its partner (j + 1)
          const int j0 = ty == 3 ? j - 1 : j;
          for (int jj = j0; jj <= j; ++jj) {
            const double* Lj = P + static_cast<std::int64_t>(jj) * m;
            for (int r = 0; r < rr; ++r) {
              double acc = 0.0;
              for (int i = j + 1 + lane; i < be; i += 32) acc += Lj[i] * t[i * R + r];
              acc = warp_sum(acc);
              if (lane == 0) t[jj * R + r] -= acc;
            }
          }
          __syncwarp();
        }
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < k; i += blockDim.x)
      for (int r = 0; r < rr; ++r) x[d.first + pl[i] + (r0 + r) * n] = t[i * R + r];
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
  int R = nrhs < 8 ? nrhs : 8;
  while (R > 1 && solve_smem(maxm, R) > kSolveSmemMax) --R;
  return R < 1 ? 1 : R;
}

void launch_solve_fwd(const std::int32_t* list, int nlist, int maxm, const SnDev* sn, const std::int32_t* child_ptr,
                      const std::int32_t* children, const std::int32_t* rmap, const double* panels,
                      const signed char* piv, const std::int32_t* pidx, double* x, std::int64_t n, double* vec,
                      int nrhs, cudaStream_t s) {
  if (nlist <= 0) return;
  const int R = solve_rhs_chunk(maxm, nrhs);
  const std::size_t smem = solve_smem(maxm, R);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_solve_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSolveSmemMax));
    configured = true;
  }
  note_launches(1);
  k_solve_fwd<<<nlist, 256, smem, s>>>(list, sn, child_ptr, children, rmap, panels, piv, pidx, x, n, vec, nrhs, R);
}

void launch_solve_diag(int ns, const SnDev* sn, const double* panels, const signed char* piv,
                       const std::int32_t* pidx, double* x, std::int64_t n, int nrhs, cudaStream_t s) {
  if (ns <= 0) return;
  note_launches(1);
  k_solve_diag<<<ns, 128, 0, s>>>(sn, panels, piv, pidx, x, n, nrhs);
}

void launch_solve_bwd(const std::int32_t* list, int nlist, int maxm, const SnDev* sn, const std::int32_t* rows,
                      const double* panels, const signed char* piv, const std::int32_t* pidx, double* x,
                      std::int64_t n, int nrhs, cudaStream_t s) {
  if (nlist <= 0) return;
  const int R = solve_rhs_chunk(maxm, nrhs);
  const std::size_t smem = solve_smem(maxm, R);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_solve_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSolveSmemMax));
    configured = true;
  }
  note_launches(1);
  k_solve_bwd<<<nlist, 256, smem, s>>>(list, sn, rows, panels, piv, pidx, x, n, nrhs, R);
}

}  // namespace hsg
