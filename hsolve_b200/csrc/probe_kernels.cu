// FP64 FMA throughput probe: the measured denominator of the factorization roofline (the
// machine-peak file holds HBM and bf16 figures only). Eight independent FMA chains per thread keep
// the FP64 pipes busy; the result is 2 * FMAs / elapsed time.
#include <algorithm>
#include <cuda_runtime.h>

#include "common.hpp"
#include "gpu_factor.hpp"
#include "hsg.h"

namespace hsg {
namespace {
__global__ void k_fma_chains(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) x[c] = threadIdx.x * 1e-3 + c;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < 8; ++c) s += x[c];
  if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains live
}
}  // namespace
}  // namespace hsg

extern "C" int hsg_fp64_peak_probe(int32_t device, double* tflops) {
  using namespace hsg;
  return guarded([&] {
    HSG_REQUIRE(tflops, HSG_INVALID_INPUT, "null output");
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cudaDeviceProp prop{};
    cuda_check(cudaGetDeviceProperties(&prop, device), "props");
    DevBuf<double> out;
    out.alloc(4096);
    const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    note_launches(1);
    k_fma_chains<<<blocks, threads>>>(out.p, iters, 0.999999, 1e-7);  // warm-up
    double best = 0.0;
    for (int rep = 0; rep < 5; ++rep) {
      cuda_check(cudaEventRecord(e0), "event");
      note_launches(1);
      k_fma_chains<<<blocks, threads>>>(out.p, iters, 0.999999, 1e-7);
      cuda_check(cudaEventRecord(e1), "event");
      cuda_check(cudaEventSynchronize(e1), "sync");
      float ms = 0.0f;
      cuda_check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
      const double fl = 2.0 * 8.0 * static_cast<double>(iters) * blocks * threads;
      best = std::max(best, fl / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *tflops = best;
  });
}
