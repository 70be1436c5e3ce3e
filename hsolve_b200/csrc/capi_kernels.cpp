// C ABI of the sparse kernels on device pointers (include/hsg.h): hs::spmm and
// hs::shifted_residual (include/hsolve/sparse.hpp:140-174) for callers that hold their vectors on
// the GPU. Both run on the legacy default stream and wait for their GPU work before returning.
#include <cmath>

#include <cuda_runtime.h>

#include "blas_kernels.cuh"
#include "common.hpp"
#include "gpu_factor.hpp"
#include "hsg.h"

using namespace hsg;

extern "C" {

int hsg_spmm(int64_t n, const int64_t* a_rowptr, const int32_t* a_col, const double* a_val, const double* x,
             int64_t ldx, double* y, int64_t ldy, int64_t p, double alpha, double beta) {
  return guarded([&] {
    HSG_REQUIRE(n >= 0 && p >= 0, HSG_INVALID_INPUT, "hsg_spmm: negative size");
    if (n == 0 || p == 0) return;
    HSG_REQUIRE(a_rowptr && a_col && a_val && x && y, HSG_INVALID_INPUT, "hsg_spmm: null pointer");
    HSG_REQUIRE(ldx >= n && ldy >= n, HSG_INVALID_INPUT, "hsg_spmm: leading dimension below n");
    HSG_REQUIRE(p <= (int64_t{1} << 30) && std::isfinite(alpha) && std::isfinite(beta), HSG_INVALID_INPUT,
                "hsg_spmm: p or alpha / beta out of range");
    const CsrDev a{n, a_rowptr, a_col, a_val};
    spmm(a, x, ldx, y, ldy, static_cast<int>(p), alpha, beta, cudaStreamLegacy);
    cuda_check(cudaGetLastError(), "hsg_spmm launch");
    cuda_check(cudaStreamSynchronize(cudaStreamLegacy), "hsg_spmm");
  });
}

int hsg_shifted_residual(int64_t n, const int64_t* a_rowptr, const int32_t* a_col, const double* a_val,
                         const int64_t* b_rowptr, const int32_t* b_col, const double* b_val, double sigma,
                         const double* x, int64_t ldx, const double* y, int64_t ldy, double* r, int64_t ldr,
                         int64_t p, double* backward_error) {
  return guarded([&] {
    HSG_REQUIRE(n >= 0 && p >= 0, HSG_INVALID_INPUT, "hsg_shifted_residual: negative size");
    if (n == 0 || p == 0) return;
    HSG_REQUIRE(a_rowptr && a_col && a_val && x && y && (r || backward_error), HSG_INVALID_INPUT,
                "hsg_shifted_residual: null pointer");
    HSG_REQUIRE(!b_rowptr || (b_col && b_val), HSG_INVALID_INPUT, "hsg_shifted_residual: incomplete B");
    HSG_REQUIRE(ldx >= n && ldy >= n && (!r || ldr >= n), HSG_INVALID_INPUT,
                "hsg_shifted_residual: leading dimension below n");
    HSG_REQUIRE(std::isfinite(sigma) && p <= (int64_t{1} << 30), HSG_INVALID_INPUT,
                "hsg_shifted_residual: non-finite sigma or p out of range");
    const CsrDev a{n, a_rowptr, a_col, a_val};
    const CsrDev b{n, b_rowptr, b_col, b_val};
    shifted_residual(a, b_rowptr ? &b : nullptr, sigma, x, ldx, y, ldy, r, ldr, static_cast<int>(p), backward_error,
                     cudaStreamLegacy);
    cuda_check(cudaGetLastError(), "hsg_shifted_residual launch");
    cuda_check(cudaStreamSynchronize(cudaStreamLegacy), "hsg_shifted_residual");
  });
}

}  // extern "C"
