// hsg_solve_static: the multi-RHS solve with its work space in a fixed array compiled into the
// library instead of device memory allocated at run time, for callers that must not allocate.
//
// The array g_solve_scratch below is a file-scope __device__ variable: every device that loads the
// library holds its HSG_SOLVE_STATIC_SCRATCH_BYTES until the process exits. In host code its name
// is only a host-side stand-in, never a device address, so the host looks the address up once per
// device (cudaGetSymbolAddress, with that device current) and passes it to the solve kernels as
// a plain pointer. The solve writes every scratch entry it reads (the gathered right-hand sides and
// the children's update vectors), so the array keeps the last call's contents and none of it has to
// be cleared between calls. Calls on one device share the array: calls whose GPU work overlaps race.
#include <algorithm>
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "common.hpp"
#include "gpu_factor.hpp"
#include "hsg.h"

namespace hsg {
GpuFactor& factor_of(hsg_factor* f);
}

namespace {

constexpr std::size_t kScratchDoubles = HSG_SOLVE_STATIC_SCRATCH_BYTES / sizeof(double);
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_solve_scratch[kScratchDoubles];

std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of g_solve_scratch on `device` (looked up on the first call for that device).
double* scratch_on(int device) {
  HSG_REQUIRE(device >= 0 && device < kMaxDevices, HSG_INVALID_INPUT, "hsg_solve_static: device " << device
                                                                          << " out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[device]) {
    int prev = -1;
    hsg::cuda_check(cudaGetDevice(&prev), "cudaGetDevice");
    if (prev != device) hsg::cuda_check(cudaSetDevice(device), "cudaSetDevice");
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_solve_scratch);
    if (prev != device) cudaSetDevice(prev);
    HSG_REQUIRE(e == cudaSuccess && p, HSG_INTERNAL,
                "hsg_solve_static: cudaGetSymbolAddress failed on device " << device << ": " << cudaGetErrorString(e));
    g_scratch_addr[device] = static_cast<double*>(p);
  }
  return g_scratch_addr[device];
}

}  // namespace

extern "C" int hsg_solve_static(hsg_factor* f, double* b_device, int64_t nrhs, int64_t ldb) {
  return hsg::guarded([&] {
    hsg::GpuFactor& g = hsg::factor_of(f);
    HSG_REQUIRE(nrhs >= 0, HSG_INVALID_INPUT, "hsg_solve_static: nrhs < 0");
    // the right-hand sides alone (n per column) must fit before the exact size is formed, so that
    // a huge nrhs cannot overflow the 64-bit product below
    const std::int64_t n = std::max<std::int64_t>(1, g.order());
    HSG_REQUIRE(nrhs <= static_cast<std::int64_t>(kScratchDoubles) / n, HSG_INVALID_INPUT,
                "hsg_solve_static: " << nrhs << " right-hand sides of order " << g.order()
                                     << " exceed what the static array holds (" << kScratchDoubles * 8
                                     << " bytes); split the right-hand sides or use hsg_solve");
    const std::size_t need = nrhs > 0 ? g.solve_scratch_doubles(nrhs) : 0;
    HSG_REQUIRE(need <= kScratchDoubles, HSG_INVALID_INPUT,
                "hsg_solve_static: " << nrhs << " right-hand sides of order " << g.order() << " need " << need * 8
                                     << " bytes of scratch, the static array holds " << kScratchDoubles * 8
                                     << "; split the right-hand sides or use hsg_solve");
    if (nrhs == 0) return;
    HSG_REQUIRE(b_device, HSG_INVALID_INPUT, "hsg_solve_static: null right-hand side");
    // b must be device (or managed) memory of the factorization's device: a host pointer or another
    // device's memory would make the solve kernels fault
    cudaPointerAttributes attr{};
    const cudaError_t pe = cudaPointerGetAttributes(&attr, b_device);
    if (pe != cudaSuccess) cudaGetLastError();  // clear the sticky-free error of an unknown pointer
    HSG_REQUIRE(pe == cudaSuccess &&
                    (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) &&
                    attr.device == g.device(),
                HSG_INVALID_INPUT, "hsg_solve_static: b_device is not device memory of device " << g.device());
    g.order_after_legacy_stream();
    g.solve_with_scratch(b_device, nrhs, ldb, scratch_on(g.device()), kScratchDoubles);
  });
}
