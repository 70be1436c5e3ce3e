// Per-device caching pool behind DevBuf (gpu_factor.hpp).
#include <cstdint>
#include <map>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "common.hpp"
#include "gpu_factor.hpp"

namespace hsg {

namespace {

constexpr int kMaxDevices = 64;

struct Pool {
  std::mutex mu;
  std::multimap<std::size_t, void*> free[kMaxDevices];  // size class -> cached blocks
};

Pool& pool() {
  static Pool* p = new Pool;  // never destroyed: blocks may be released after static destructors ran
  return *p;
}

// smallest size class >= bytes: 256-byte granularity below 64 KiB, else eight classes per octave
std::size_t size_class(std::size_t bytes) {
  if (bytes <= (64u << 10)) return (bytes + 255) / 256 * 256;
  int e = 0;
  while ((std::size_t{1} << (e + 1)) <= bytes) ++e;  // 2^e <= bytes < 2^(e+1)
  const std::size_t step = std::size_t{1} << (e - 3);
  return (bytes + step - 1) / step * step;
}

void release_cached(int device) {
  Pool& P = pool();
  for (auto& kv : P.free[device]) cudaFree(kv.second);
  P.free[device].clear();
}

}  // namespace

void* pool_alloc(std::size_t bytes, std::size_t* cap, int* device) {
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  HSG_REQUIRE(dev >= 0 && dev < kMaxDevices, HSG_INTERNAL, "device " << dev << " out of range");
  const std::size_t c = size_class(bytes);
  Pool& P = pool();
  {
    std::lock_guard<std::mutex> lk(P.mu);
    auto it = P.free[dev].find(c);
    if (it != P.free[dev].end()) {
      void* p = it->second;
      P.free[dev].erase(it);
      *cap = c;
      *device = dev;
      return p;
    }
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, c);
  if (e != cudaSuccess) {
    cudaGetLastError();
    {
      std::lock_guard<std::mutex> lk(P.mu);
      release_cached(dev);
    }
    e = cudaMalloc(&p, c);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    HSG_THROW(HSG_OUT_OF_MEMORY_BUDGET, "cudaMalloc of " << c << " bytes failed: " << cudaGetErrorString(e));
  }
  *cap = c;
  *device = dev;
  return p;
}

void pool_free(void* p, std::size_t cap, int device) {
  if (!p) return;
  Pool& P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  P.free[device].emplace(cap, p);
}

void pool_trim() {
  Pool& P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  int cur = 0;
  cudaGetDevice(&cur);
  for (int d = 0; d < kMaxDevices; ++d) {
    if (P.free[d].empty()) continue;
    cudaSetDevice(d);
    release_cached(d);
  }
  cudaSetDevice(cur);
}

}  // namespace hsg
