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

// A cached block and, when it was released inside a PoolStreamScope, an event recorded on that
// stream at the release: the block may still be read or written by work queued before the event.
struct Block {
  void* p;
  cudaEvent_t ev;
};

struct Pool {
  std::mutex mu;
  std::multimap<std::size_t, Block> free[kMaxDevices];  // size class -> cached blocks
  std::vector<cudaEvent_t> events[kMaxDevices];          // idle events for later releases
};

thread_local cudaStream_t t_stream = nullptr;

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
  for (auto& kv : P.free[device]) {
    if (kv.second.ev) {
      cudaEventSynchronize(kv.second.ev);
      P.events[device].push_back(kv.second.ev);
    }
    cudaFree(kv.second.p);
  }
  P.free[device].clear();
}

// Makes the block usable by the calling thread's work: a stream-ordered wait on the release event
// when the thread has a scope on this device, else a host wait for it.
void settle(Block& b, int dev) {
  if (!b.ev) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (t_stream && cur == dev) cuda_check(cudaStreamWaitEvent(t_stream, b.ev, 0), "pool: wait for the release");
  else cuda_check(cudaEventSynchronize(b.ev), "pool: wait for the release");
  Pool& P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  P.events[dev].push_back(b.ev);
  b.ev = nullptr;
}

}  // namespace

PoolStreamScope::PoolStreamScope(cudaStream_t s) : prev_(t_stream) { t_stream = s; }
PoolStreamScope::~PoolStreamScope() { t_stream = prev_; }

void* pool_alloc(std::size_t bytes, std::size_t* cap, int* device) {
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  HSG_REQUIRE(dev >= 0 && dev < kMaxDevices, HSG_INTERNAL, "device " << dev << " out of range");
  const std::size_t c = size_class(bytes);
  Pool& P = pool();
  {
    Block b{nullptr, nullptr};
    {
      std::lock_guard<std::mutex> lk(P.mu);
      auto it = P.free[dev].find(c);
      if (it != P.free[dev].end()) {
        b = it->second;
        P.free[dev].erase(it);
      }
    }
    if (b.p) {
      settle(b, dev);
      *cap = c;
      *device = dev;
      return b.p;
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
  cudaEvent_t ev = nullptr;
  int cur = -1;
  if (t_stream && cudaGetDevice(&cur) == cudaSuccess && cur == device) {
    {
      std::lock_guard<std::mutex> lk(P.mu);
      if (!P.events[device].empty()) {
        ev = P.events[device].back();
        P.events[device].pop_back();
      }
    }
    if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      ev = nullptr;
    }
    if (ev && cudaEventRecord(ev, t_stream) != cudaSuccess) {
      // no ordering possible: wait for the stream here, so the block is idle when it is cached
      cudaGetLastError();
      cudaStreamSynchronize(t_stream);
      std::lock_guard<std::mutex> lk(P.mu);
      P.events[device].push_back(ev);
      ev = nullptr;
    }
  }
  std::lock_guard<std::mutex> lk(P.mu);
  P.free[device].emplace(cap, Block{p, ev});
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
