// HBM-bound kernels of the Krylov loop (sm_100a, FP64):
//  * CSR SpMM  Y = M X  (replaces hsolve's spmm, src/sparse/kernels.cpp:797);
//  * fused shifted residual R = B (X + sigma Y) - A Y with its column norms (shifted_residual,
//    src/sparse/kernels.cpp:850; contract include/hsolve/sparse.hpp:157-174);
//  * tall-skinny Gram G = X^T Y with a fixed-order two-stage reduction (bitwise reproducible), and
//    Y = beta Y + alpha X S for the block Gram-Schmidt / CholQR updates and Ritz vectors
//    (BlockOrthonormalizer, src/eigen/block_ortho.cpp:165,270; orthogonalize_block_cgs2,
//    src/linalg/dense_ops.hpp:180).
#include <cstdint>
#include <mutex>

#include <math_constants.h>

#include "blas_kernels.cuh"
#include "common.hpp"
#include "device.cuh"

namespace hsg {

void cuda_check(cudaError_t e, const char* what);

namespace {

// One warp per row; each lane handles a stride of the row's entries, all p columns at once.
template <int P>
__global__ void k_spmm(std::int64_t n, const std::int64_t* rp, const std::int32_t* ci, const double* v, const double* x,
                       std::int64_t ldx, double* y, std::int64_t ldy, int p, double alpha, double beta) {
  const int lane = threadIdx.x & 31;
  const std::int64_t warp = (blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x) >> 5;
  const std::int64_t nwarps = (static_cast<std::int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (std::int64_t i = warp; i < n; i += nwarps) {
    double acc[P];
#pragma unroll
    for (int r = 0; r < P; ++r) acc[r] = 0.0;
    for (std::int64_t q = rp[i] + lane; q < rp[i + 1]; q += 32) {
      const double a = v[q];
      const std::int64_t j = ci[q];
#pragma unroll
      for (int r = 0; r < P; ++r)
        if (r < p) acc[r] += a * x[j + r * ldx];
    }
#pragma unroll
    for (int r = 0; r < P; ++r) {
      if (r >= p) break;
      const double s = warp_sum(acc[r]);
      if (lane == 0) y[i + r * ldy] = alpha * s + (beta == 0.0 ? 0.0 : beta * y[i + r * ldy]);
    }
  }
}

// Partial Gram sums: CTA b covers rows [b*chunk, (b+1)*chunk); warp w handles columns i = w, w+8,..
// of X; the result part[b][i + c*m] = sum_rows X[row,i] Y[row,c].
__global__ void k_gram_partial(std::int64_t n, int m, int p, const double* x, std::int64_t ldx, const double* y,
                               std::int64_t ldy, std::int64_t chunk, double* part) {
  extern __shared__ double ys[];  // chunk x p
  const std::int64_t r0 = blockIdx.x * chunk;
  const std::int64_t r1 = r0 + chunk < n ? r0 + chunk : n;
  const int rows = static_cast<int>(r1 - r0);
  for (int t = threadIdx.x; t < rows * p; t += blockDim.x) {
    const int rr = t % rows, c = t / rows;
    ys[c * chunk + rr] = y[r0 + rr + c * ldy];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double* out = part + static_cast<std::int64_t>(blockIdx.x) * m * p;
  for (int i = warp; i < m; i += nw) {
    double acc[kMaxBlock];
#pragma unroll
    for (int c = 0; c < kMaxBlock; ++c) acc[c] = 0.0;
    const double* xi = x + static_cast<std::int64_t>(i) * ldx + r0;
    for (int rr = lane; rr < rows; rr += 32) {
      const double xv = xi[rr];
#pragma unroll
      for (int c = 0; c < kMaxBlock; ++c)
        if (c < p) acc[c] += xv * ys[c * chunk + rr];
    }
#pragma unroll
    for (int c = 0; c < kMaxBlock; ++c) {
      if (c >= p) break;
      const double s = warp_sum(acc[c]);
      if (lane == 0) out[i + c * m] = s;
    }
  }
}

// Fixed-order sum of the partials: g[t] = sum_b part[b][t]. A block takes 32 consecutive outputs;
// its 8 thread rows stride over the partials (reads coalesced over the outputs) and their 8 sums are
// added in shared memory in row order, so the result does not depend on the launch.
constexpr int kReduceRows = 8;
__global__ void __launch_bounds__(32 * kReduceRows) k_gram_reduce(int nparts, int mp, const double* part, double* g) {
  __shared__ double acc[kReduceRows][33];
  const int tl = threadIdx.x & 31, row = threadIdx.x >> 5;
  const int t = blockIdx.x * 32 + tl;
  double s = 0.0;
  if (t < mp)
    for (int b = row; b < nparts; b += kReduceRows) s += part[static_cast<std::int64_t>(b) * mp + t];
  acc[row][tl] = s;
  __syncthreads();
  if (row == 0 && t < mp) {
    double v = 0.0;
#pragma unroll
    for (int r = 0; r < kReduceRows; ++r) v += acc[r][tl];
    g[t] = v;
  }
}

// Y[:, c0:c0+q] = beta Y + alpha X S[:, c0:c0+q] (X n x m, S m x q in shared memory), 16 columns a pass.
// y (n x q) = alpha X S + beta y: one thread per row, S staged in shared memory QC columns at a time
// (QC = 8 for the Krylov block width, 16 for wider products).
template <int QC>
__global__ void k_gemm_tall(std::int64_t n, int m, int q, const double* x, std::int64_t ldx, const double* s, int lds,
                            double* y, std::int64_t ldy, double alpha, double beta) {
  extern __shared__ double ss[];  // m x QC
  for (int c0 = 0; c0 < q; c0 += QC) {
    const int qc = q - c0 < QC ? q - c0 : QC;
    __syncthreads();
    for (int t = threadIdx.x; t < m * QC; t += blockDim.x) {
      const int i = t % m, c = t / m;
      ss[c * m + i] = c < qc ? s[i + static_cast<std::int64_t>(c0 + c) * lds] : 0.0;
    }
    __syncthreads();
    for (std::int64_t row = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; row < n;
         row += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
      double acc[QC];
#pragma unroll
      for (int c = 0; c < QC; ++c) acc[c] = 0.0;
#pragma unroll 4
      for (int i = 0; i < m; ++i) {
        const double xv = x[row + static_cast<std::int64_t>(i) * ldx];
#pragma unroll
        for (int c = 0; c < QC; ++c) acc[c] += xv * ss[c * m + i];
      }
#pragma unroll
      for (int c = 0; c < QC; ++c) {
        if (c >= qc) break;
        double* yp = y + row + static_cast<std::int64_t>(c0 + c) * ldy;
        *yp = alpha * acc[c] + (beta == 0.0 ? 0.0 : beta * *yp);
      }
    }
  }
}

__global__ void k_diag_scale(std::int64_t n, int p, const double* d, const double* x, std::int64_t ldx, double* y,
                             std::int64_t ldy) {
  const std::int64_t total = n * p;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t i = t % n, c = t / n;
    y[i + c * ldy] = d[i] * x[i + c * ldx];
  }
}

__global__ void k_copy_cols(std::int64_t n, int p, const double* x, std::int64_t ldx, double* y, std::int64_t ldy) {
  const std::int64_t total = n * p;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t i = t % n, c = t / n;
    y[i + c * ldy] = x[i + c * ldx];
  }
}

// Standard normal entries y(i, c) from a counter-based stream: a SplitMix64 hash of (seed, element
// index) gives two uniforms, Box-Muller turns them into one normal deviate. Deterministic in the
// seed and independent of the launch shape.
__device__ __forceinline__ std::uint64_t splitmix64(std::uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_fill_normal(std::int64_t n, int p, double* y, std::int64_t ldy, std::uint64_t seed) {
  const std::int64_t total = n * p;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::uint64_t h1 = splitmix64(seed ^ (static_cast<std::uint64_t>(t) * 2 + 1));
    const std::uint64_t h2 = splitmix64(h1 ^ 0xD1B54A32D192ED03ull);
    const double u1 = (static_cast<double>(h1 >> 11) + 0.5) * 0x1.0p-53;  // (0, 1)
    const double u2 = static_cast<double>(h2 >> 11) * 0x1.0p-53;          // [0, 1)
    const std::int64_t i = t % n, c = t / n;
    y[i + c * ldy] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
}

// Shifted residual of a shift-invert solve, one warp per row and all P columns at once:
//   r(i, c) = (B w_c)(i) - (A y_c)(i),  w = x + sigma y  (B = null: B = I),
//   s(i, c) = (|B| |w_c|)(i) + (|A| |y_c|)(i),
// and the componentwise backward error omega_c = max_i |r(i, c)| / s(i, c) with 0/0 = 0, r/0 = inf and
// inf for a row whose r or s is not finite (the contract of hsolve's shifted_residual,
// include/hsolve/sparse.hpp:157-174). omega must hold zeros at launch; the maximum is taken by an
// integer atomic max on the bit patterns of non-negative doubles (order independent).
template <int P>
__global__ void k_shifted_residual(std::int64_t n, const std::int64_t* arp, const std::int32_t* aci, const double* av,
                                   const std::int64_t* brp, const std::int32_t* bci, const double* bv, double sigma,
                                   const double* x, std::int64_t ldx, const double* y, std::int64_t ldy, double* r,
                                   std::int64_t ldr, int p, unsigned long long* omega) {
  const int lane = threadIdx.x & 31;
  const std::int64_t warp = (blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x) >> 5;
  const std::int64_t nwarps = (static_cast<std::int64_t>(gridDim.x) * blockDim.x) >> 5;
  double om[P];
#pragma unroll
  for (int c = 0; c < P; ++c) om[c] = 0.0;
  for (std::int64_t i = warp; i < n; i += nwarps) {
    double ra[P], sa[P];
#pragma unroll
    for (int c = 0; c < P; ++c) { ra[c] = 0.0; sa[c] = 0.0; }
    for (std::int64_t q = arp[i] + lane; q < arp[i + 1]; q += 32) {
      const double a = av[q];
      const std::int64_t j = aci[q];
#pragma unroll
      for (int c = 0; c < P; ++c)
        if (c < p) {
          const double yj = y[j + c * ldy];
          ra[c] = fma(-a, yj, ra[c]);
          sa[c] = fma(fabs(a), fabs(yj), sa[c]);
        }
    }
    if (brp) {
      for (std::int64_t q = brp[i] + lane; q < brp[i + 1]; q += 32) {
        const double b = bv[q];
        const std::int64_t j = bci[q];
#pragma unroll
        for (int c = 0; c < P; ++c)
          if (c < p) {
            const double wj = fma(sigma, y[j + c * ldy], x[j + c * ldx]);
            ra[c] = fma(b, wj, ra[c]);
            sa[c] = fma(fabs(b), fabs(wj), sa[c]);
          }
      }
    } else if (lane == 0) {
#pragma unroll
      for (int c = 0; c < P; ++c)
        if (c < p) {
          const double wi = fma(sigma, y[i + c * ldy], x[i + c * ldx]);
          ra[c] += wi;
          sa[c] += fabs(wi);
        }
    }
#pragma unroll
    for (int c = 0; c < P; ++c) {
      if (c >= p) break;
      const double rs = warp_sum(ra[c]);
      const double ss = warp_sum(sa[c]);
      if (lane == 0) {
        if (r) r[i + c * ldr] = rs;
        const double ar = fabs(rs);
        double w;
        if (!isfinite(rs) || !isfinite(ss)) w = CUDART_INF;
        else if (ss > 0.0) w = ar / ss;
        else w = ar > 0.0 ? CUDART_INF : 0.0;
        om[c] = fmax(om[c], w);
      }
    }
  }
  if (omega && lane == 0) {
#pragma unroll
    for (int c = 0; c < P; ++c)
      if (c < p && om[c] > 0.0) atomic_max_nonneg(&omega[c], om[c]);
  }
}

// z = x + y (p columns)
__global__ void k_add_cols(std::int64_t n, int p, const double* x, std::int64_t ldx, const double* y,
                           std::int64_t ldy, double* z, std::int64_t ldz) {
  const std::int64_t total = n * p;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t i = t % n, c = t / n;
    z[i + c * ldz] = x[i + c * ldx] + y[i + c * ldy];
  }
}

// y(:, c) = x(:, c) for the columns with mask bit c set (p <= 32)
__global__ void k_copy_cols_masked(std::int64_t n, int p, unsigned mask, const double* x, std::int64_t ldx, double* y,
                                   std::int64_t ldy) {
  const std::int64_t total = n * p;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t i = t % n, c = t / n;
    if ((mask >> c) & 1u) y[i + c * ldy] = x[i + c * ldx];
  }
}

// bits of a non-negative double array (atomic max slots) -> doubles, in place
__global__ void k_bits_to_double(int p, unsigned long long* w) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < p) reinterpret_cast<double*>(w)[c] = __longlong_as_double(static_cast<long long>(w[c]));
}

// r = a - lam .* b (column c uses lam[c]); y holds r
__global__ void k_residual_cols(std::int64_t n, int p, const double* ax, std::int64_t lda, const double* bx,
                                std::int64_t ldb, const double* lam, double* r, std::int64_t ldr) {
  const std::int64_t total = n * p;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t i = t % n, c = t / n;
    r[i + c * ldr] = ax[i + c * lda] - lam[c] * bx[i + c * ldb];
  }
}

__global__ void k_scale_cols(std::int64_t n, int p, double a, double* y, std::int64_t ldy) {
  const std::int64_t total = n * p;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t i = t % n, c = t / n;
    y[i + c * ldy] *= a;
  }
}

// out[j] = sum_i x[i, j] y[i, j] (one CTA per column, fixed-order tree reduction)
__global__ void k_col_dots(std::int64_t n, const double* x, std::int64_t ldx, const double* y, std::int64_t ldy,
                           double* out) {
  __shared__ double red[32];
  const double* xc = x + static_cast<std::int64_t>(blockIdx.x) * ldx;
  const double* yc = y + static_cast<std::int64_t>(blockIdx.x) * ldy;
  double s = 0.0;
  for (std::int64_t i = threadIdx.x; i < n; i += blockDim.x) s += xc[i] * yc[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) out[blockIdx.x] = t;
  }
}

int grid_for(std::int64_t work, int threads) {
  const std::int64_t b = (work + threads - 1) / threads;
  return static_cast<int>(b < 1 ? 1 : (b > 148 * 32 ? 148 * 32 : b));
}

}  // namespace

void spmm(const CsrDev& M, const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p, double alpha,
          double beta, cudaStream_t s) {
  if (p <= 0 || M.n == 0) return;
  const int threads = 256;
  const int blocks = grid_for(M.n * 32, threads);
  for (int c0 = 0; c0 < p; c0 += 8) {
    const int pc = p - c0 < 8 ? p - c0 : 8;
    const double* xc = x + c0 * ldx;
    double* yc = y + c0 * ldy;
    if (pc == 1) { note_launches(1); k_spmm<1><<<blocks, threads, 0, s>>>(M.n, M.rp, M.ci, M.v, xc, ldx, yc, ldy, pc, alpha, beta); }
    else if (pc <= 2) { note_launches(1); k_spmm<2><<<blocks, threads, 0, s>>>(M.n, M.rp, M.ci, M.v, xc, ldx, yc, ldy, pc, alpha, beta); }
    else if (pc <= 4) { note_launches(1); k_spmm<4><<<blocks, threads, 0, s>>>(M.n, M.rp, M.ci, M.v, xc, ldx, yc, ldy, pc, alpha, beta); }
    else { note_launches(1); k_spmm<8><<<blocks, threads, 0, s>>>(M.n, M.rp, M.ci, M.v, xc, ldx, yc, ldy, pc, alpha, beta); }
  }
}

void gram(std::int64_t n, int m, int p, const double* x, std::int64_t ldx, const double* y, std::int64_t ldy,
          double* g, double* part, std::int64_t part_cap, cudaStream_t s) {
  if (m <= 0 || p <= 0) return;
  // p > kMaxBlock: column chunks of Y
  for (int c0 = 0; c0 < p; c0 += kMaxBlock) {
    const int pc = p - c0 < kMaxBlock ? p - c0 : kMaxBlock;
    std::int64_t chunk = (n + 295) / 296;
    const std::int64_t cap_rows = 6144 / pc;  // Y chunk <= 48 KB of shared memory
    if (chunk > cap_rows) chunk = cap_rows;
    if (chunk < 64) chunk = 64;
    const std::int64_t nparts = (n + chunk - 1) / chunk;
    if (nparts * m * pc > part_cap) return;  // caller sized part_cap with gram_part_size()
    const std::size_t smem = static_cast<std::size_t>(chunk) * pc * sizeof(double);
    note_launches(1);
    k_gram_partial<<<static_cast<int>(nparts), 256, smem, s>>>(n, m, pc, x, ldx, y + c0 * ldy, ldy, chunk, part);
    note_launches(1);
    k_gram_reduce<<<(m * pc + 31) / 32, 32 * kReduceRows, 0, s>>>(static_cast<int>(nparts), m * pc, part,
                                                               g + static_cast<std::int64_t>(c0) * m);
  }
}

void gemm_tall(std::int64_t n, int m, int q, const double* x, std::int64_t ldx, const double* sdev, int lds, double* y,
               std::int64_t ldy, double alpha, double beta, cudaStream_t s) {
  if (q <= 0 || n <= 0) return;
  if (m <= 0) {
    if (beta != 1.0) { note_launches(1); k_scale_cols<<<grid_for(n * q, 256), 256, 0, s>>>(n, q, beta, y, ldy); }
    return;
  }
  static std::once_flag configured;
  std::call_once(configured, [&] {
    cudaFuncSetAttribute(k_gemm_tall<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_gemm_tall<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  });
  note_launches(1);
  if (q <= 8) {
    const std::size_t smem = static_cast<std::size_t>(m) * 8 * sizeof(double);
    k_gemm_tall<8><<<grid_for(n, 256), 256, smem, s>>>(n, m, q, x, ldx, sdev, lds, y, ldy, alpha, beta);
  } else {
    const std::size_t smem = static_cast<std::size_t>(m) * 16 * sizeof(double);
    k_gemm_tall<16><<<grid_for(n, 256), 256, smem, s>>>(n, m, q, x, ldx, sdev, lds, y, ldy, alpha, beta);
  }
}

std::int64_t gram_part_size(std::int64_t n, int m, int p) {
  const int pc = p < kMaxBlock ? p : kMaxBlock;
  std::int64_t chunk = (n + 295) / 296;
  const std::int64_t cap_rows = 6144 / (pc > 0 ? pc : 1);
  if (chunk > cap_rows) chunk = cap_rows;
  if (chunk < 64) chunk = 64;
  return ((n + chunk - 1) / chunk) * static_cast<std::int64_t>(m) * pc;
}

void col_dots(std::int64_t n, int m, const double* x, std::int64_t ldx, const double* y, std::int64_t ldy, double* out,
              cudaStream_t s) {
  if (m <= 0) return;
  note_launches(1);
  k_col_dots<<<m, 512, 0, s>>>(n, x, ldx, y, ldy, out);
}

void scale_cols(std::int64_t n, int p, double a, double* y, std::int64_t ldy, cudaStream_t s) {
  note_launches(1);
  k_scale_cols<<<grid_for(n * p, 256), 256, 0, s>>>(n, p, a, y, ldy);
}

void diag_scale(std::int64_t n, int p, const double* d, const double* x, std::int64_t ldx, double* y,
                std::int64_t ldy, cudaStream_t s) {
  note_launches(1);
  k_diag_scale<<<grid_for(n * p, 256), 256, 0, s>>>(n, p, d, x, ldx, y, ldy);
}

void copy_cols(std::int64_t n, int p, const double* x, std::int64_t ldx, double* y, std::int64_t ldy, cudaStream_t s) {
  note_launches(1);
  k_copy_cols<<<grid_for(n * p, 256), 256, 0, s>>>(n, p, x, ldx, y, ldy);
}

namespace {
// Lanczos recurrence with device-resident coefficients (ab[j]: alpha_j = v_j^T A v_j; ab[kLanczosMax + j]:
// beta_j^2 = ||w_j||^2): w -= alpha_j v_j + beta_{j-1} v_{j-1}
__global__ void k_lanczos_orth(std::int64_t n, double* w, const double* v, const double* vp, const double* ab, int j,
                               int stride) {
  const double alpha = ab[j];
  const double beta = j > 0 ? sqrt(fmax(ab[stride + j - 1], 0.0)) : 0.0;
  for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::int64_t>(gridDim.x) * blockDim.x)
    w[i] -= alpha * v[i] + (j > 0 ? beta * vp[i] : 0.0);
}
// v = w / sqrt(nrm2[0]) (zero when the norm is zero: the Krylov space is invariant)
__global__ void k_scale_by_norm(std::int64_t n, const double* w, double* v, const double* nrm2) {
  const double q = nrm2[0];
  const double f = q > 0.0 ? 1.0 / sqrt(q) : 0.0;
  for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::int64_t>(gridDim.x) * blockDim.x)
    v[i] = w[i] * f;
}
}  // namespace

void lanczos_orth(std::int64_t n, double* w, const double* v, const double* vp, const double* ab, int j, int stride,
                  cudaStream_t s) {
  note_launches(1);
  k_lanczos_orth<<<grid_for(n, 256), 256, 0, s>>>(n, w, v, vp, ab, j, stride);
}

void scale_by_norm(std::int64_t n, const double* w, double* v, const double* nrm2, cudaStream_t s) {
  note_launches(1);
  k_scale_by_norm<<<grid_for(n, 256), 256, 0, s>>>(n, w, v, nrm2);
}

void fill_normal(std::int64_t n, int p, double* y, std::int64_t ldy, std::uint64_t seed, cudaStream_t s) {
  note_launches(1);
  k_fill_normal<<<grid_for(n * p, 256), 256, 0, s>>>(n, p, y, ldy, seed);
}

void shifted_residual(const CsrDev& A, const CsrDev* B, double sigma, const double* x, std::int64_t ldx,
                      const double* y, std::int64_t ldy, double* r, std::int64_t ldr, int p, double* omega,
                      cudaStream_t s) {
  if (p <= 0 || A.n == 0) return;
  const int threads = 256;
  const int blocks = grid_for(A.n * 32, threads);
  if (omega) cuda_check(cudaMemsetAsync(omega, 0, static_cast<std::size_t>(p) * sizeof(double), s), "memset omega");
  for (int c0 = 0; c0 < p; c0 += 8) {
    const int pc = p - c0 < 8 ? p - c0 : 8;
    const double* xc = x + c0 * ldx;
    const double* yc = y + c0 * ldy;
    double* rc = r ? r + c0 * ldr : nullptr;
    unsigned long long* oc = omega ? reinterpret_cast<unsigned long long*>(omega + c0) : nullptr;
    const std::int64_t* brp = B ? B->rp : nullptr;
    const std::int32_t* bci = B ? B->ci : nullptr;
    const double* bvv = B ? B->v : nullptr;
    note_launches(1);
    if (pc == 1)
      k_shifted_residual<1><<<blocks, threads, 0, s>>>(A.n, A.rp, A.ci, A.v, brp, bci, bvv, sigma, xc, ldx, yc, ldy, rc, ldr, pc, oc);
    else if (pc <= 2)
      k_shifted_residual<2><<<blocks, threads, 0, s>>>(A.n, A.rp, A.ci, A.v, brp, bci, bvv, sigma, xc, ldx, yc, ldy, rc, ldr, pc, oc);
    else if (pc <= 4)
      k_shifted_residual<4><<<blocks, threads, 0, s>>>(A.n, A.rp, A.ci, A.v, brp, bci, bvv, sigma, xc, ldx, yc, ldy, rc, ldr, pc, oc);
    else
      k_shifted_residual<8><<<blocks, threads, 0, s>>>(A.n, A.rp, A.ci, A.v, brp, bci, bvv, sigma, xc, ldx, yc, ldy, rc, ldr, pc, oc);
  }
  if (omega) {
    note_launches(1);
    k_bits_to_double<<<(p + 127) / 128, 128, 0, s>>>(p, reinterpret_cast<unsigned long long*>(omega));
  }
}

void add_cols(std::int64_t n, int p, const double* x, std::int64_t ldx, const double* y, std::int64_t ldy, double* z,
              std::int64_t ldz, cudaStream_t s) {
  if (p <= 0 || n <= 0) return;
  note_launches(1);
  k_add_cols<<<grid_for(n * p, 256), 256, 0, s>>>(n, p, x, ldx, y, ldy, z, ldz);
}

void copy_cols_masked(std::int64_t n, int p, unsigned mask, const double* x, std::int64_t ldx, double* y,
                      std::int64_t ldy, cudaStream_t s) {
  if (p <= 0 || n <= 0 || mask == 0u) return;
  note_launches(1);
  k_copy_cols_masked<<<grid_for(n * p, 256), 256, 0, s>>>(n, p, mask, x, ldx, y, ldy);
}

void residual_cols(std::int64_t n, int p, const double* ax, std::int64_t lda, const double* bx, std::int64_t ldb,
                   const double* lam, double* r, std::int64_t ldr, cudaStream_t s) {
  note_launches(1);
  k_residual_cols<<<grid_for(n * p, 256), 256, 0, s>>>(n, p, ax, lda, bx, ldb, lam, r, ldr);
}

}  // namespace hsg
