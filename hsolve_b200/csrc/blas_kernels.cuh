// Launchers of the Krylov-loop kernels (blas_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hsg {

constexpr int kMaxBlock = 8;  // columns a Gram pass carries (the Krylov block width is <= 8)

// Full (both triangles) CSR matrix on the device.
struct CsrDev {
  std::int64_t n = 0;
  const std::int64_t* rp = nullptr;
  const std::int32_t* ci = nullptr;
  const double* v = nullptr;
};

// y = alpha M x + beta y (p columns)
void spmm(const CsrDev& M, const double* x, std::int64_t ldx, double* y, std::int64_t ldy, int p, double alpha,
          double beta, cudaStream_t s);
// g (m x p, ld m) = X^T Y with X n x m, Y n x p; part: workspace of gram_part_size(n, m, p) doubles
void gram(std::int64_t n, int m, int p, const double* x, std::int64_t ldx, const double* y, std::int64_t ldy,
          double* g, double* part, std::int64_t part_cap, cudaStream_t s);
std::int64_t gram_part_size(std::int64_t n, int m, int p);
// y (n x q) = alpha X S + beta y, X n x m, S m x q (device, ld lds)
void gemm_tall(std::int64_t n, int m, int q, const double* x, std::int64_t ldx, const double* sdev, int lds, double* y,
               std::int64_t ldy, double alpha, double beta, cudaStream_t s);
// out[j] = <x_j, y_j> for m columns (device out)
void col_dots(std::int64_t n, int m, const double* x, std::int64_t ldx, const double* y, std::int64_t ldy, double* out,
              cudaStream_t s);
void scale_cols(std::int64_t n, int p, double a, double* y, std::int64_t ldy, cudaStream_t s);
void diag_scale(std::int64_t n, int p, const double* d, const double* x, std::int64_t ldx, double* y,
                std::int64_t ldy, cudaStream_t s);
void copy_cols(std::int64_t n, int p, const double* x, std::int64_t ldx, double* y, std::int64_t ldy, cudaStream_t s);
// standard normal entries from a counter-based stream (deterministic in seed)
void fill_normal(std::int64_t n, int p, double* y, std::int64_t ldy, std::uint64_t seed, cudaStream_t s);
// Lanczos with coefficients on the device: w -= ab[j] v + sqrt(ab[stride + j - 1]) vp (no second
// term for j = 0); v = w / sqrt(nrm2[0]) (zero for a zero norm)
void lanczos_orth(std::int64_t n, double* w, const double* v, const double* vp, const double* ab, int j, int stride,
                  cudaStream_t s);
void scale_by_norm(std::int64_t n, const double* w, double* v, const double* nrm2, cudaStream_t s);
// R = B (X + sigma Y) - A Y (B == null: B = I) for p columns in one sweep over the rows of A and B,
// and omega[c] = max_i |R(i, c)| / (|B| |X + sigma Y| + |A| |Y|)(i, c), the componentwise backward
// error of every column (device array of p doubles, or null). r may be null (omega only).
void shifted_residual(const CsrDev& A, const CsrDev* B, double sigma, const double* x, std::int64_t ldx,
                      const double* y, std::int64_t ldy, double* r, std::int64_t ldr, int p, double* omega,
                      cudaStream_t s);
// z = x + y (p columns)
void add_cols(std::int64_t n, int p, const double* x, std::int64_t ldx, const double* y, std::int64_t ldy, double* z,
              std::int64_t ldz, cudaStream_t s);
// y(:, c) = x(:, c) for every column c < p whose bit is set in mask (p <= 32)
void copy_cols_masked(std::int64_t n, int p, unsigned mask, const double* x, std::int64_t ldx, double* y,
                      std::int64_t ldy, cudaStream_t s);
void residual_cols(std::int64_t n, int p, const double* ax, std::int64_t lda, const double* bx, std::int64_t ldb,
                   const double* lam, double* r, std::int64_t ldr, cudaStream_t s);

}  // namespace hsg
