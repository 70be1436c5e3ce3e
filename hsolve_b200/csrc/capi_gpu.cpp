// GPU C ABI entry points (include/hsg.h): thin wrappers over GpuFactor.
#include <cmath>
#include <memory>

#include "common.hpp"
#include "gpu_factor.hpp"
#include "hsg.h"

struct hsg_factor {
  std::unique_ptr<hsg::GpuFactor> impl;
};

using namespace hsg;

namespace {
GpuFactor& get(hsg_factor* f) {
  HSG_REQUIRE(f && f->impl, HSG_INVALID_INPUT, "null factorization handle");
  return *f->impl;
}
const GpuFactor& get(const hsg_factor* f) {
  HSG_REQUIRE(f && f->impl, HSG_INVALID_INPUT, "null factorization handle");
  return *f->impl;
}
}  // namespace

namespace hsg {
// The object behind a handle, for entry points defined in other translation units.
GpuFactor& factor_of(hsg_factor* f) { return get(f); }
void clear_analysis_cache();
}  // namespace hsg

extern "C" {

int hsg_create(const hsg_options_t* opt, hsg_factor** out) {
  return guarded([&] {
    HSG_REQUIRE(out, HSG_INVALID_INPUT, "hsg_create: null output");
    *out = nullptr;
    hsg_options_t o;
    hsg_default_options(&o);
    if (opt) o = *opt;
    auto h = std::make_unique<hsg_factor>();
    h->impl = std::make_unique<GpuFactor>(o);
    *out = h.release();
  });
}

int hsg_destroy(hsg_factor* f) {
  return guarded([&] { delete f; });
}

int hsg_analyze(hsg_factor* f, int64_t n, const int64_t* a_rowptr, const int32_t* a_col, const double* a_val,
                const int64_t* b_rowptr, const int32_t* b_col, const double* b_val, double alpha, double beta,
                const int32_t* pivot_order) {
  return guarded([&] {
    HSG_REQUIRE(std::isfinite(alpha) && std::isfinite(beta), HSG_INVALID_INPUT, "analyze: non-finite alpha / beta");
    get(f).analyze(n, a_rowptr, a_col, a_val, b_rowptr, b_col, b_val, pivot_order);
  });
}

int hsg_estimate(const hsg_factor* f, hsg_estimate_t* out) {
  return guarded([&] {
    HSG_REQUIRE(out, HSG_INVALID_INPUT, "hsg_estimate: null output");
    *out = get(f).estimate();
  });
}

int hsg_factorize(hsg_factor* f, double alpha, double beta, hsg_inertia_t* out) {
  return guarded([&] {
    GpuFactor& g = get(f);
    const hsg_inertia_t in = g.factorize(alpha, beta, g.detection());
    if (out) *out = in;
  });
}

int hsg_count(hsg_factor* f, double alpha, double beta, int32_t detection, hsg_inertia_t* out) {
  return guarded([&] {
    GpuFactor& g = get(f);
    const hsg_inertia_t in = g.count(alpha, beta, detection != 0);
    if (out) *out = in;
  });
}

int hsg_solve(hsg_factor* f, double* b, int64_t nrhs, int64_t ldb, int32_t b_on_device) {
  return guarded([&] {
    GpuFactor& g = get(f);
    if (b_on_device) g.order_after_legacy_stream();
    g.solve(b, nrhs, ldb, b_on_device != 0);
  });
}

int hsg_inertia(const hsg_factor* f, hsg_inertia_t* out) {
  return guarded([&] {
    HSG_REQUIRE(out, HSG_INVALID_INPUT, "hsg_inertia: null output");
    *out = get(f).inertia();
  });
}

int hsg_release(hsg_factor* f, int32_t* released) {
  return guarded([&] {
    GpuFactor& g = get(f);
    const bool had = g.inertia().valid != 0;
    g.release();
    if (released) *released = had ? 1 : 0;
  });
}

int hsg_set_null_pivot_detection(hsg_factor* f, int32_t on) {
  return guarded([&] { get(f).set_detection(on != 0); });
}

int hsg_pivot_order(const hsg_factor* f, int32_t* out) {
  return guarded([&] {
    HSG_REQUIRE(out, HSG_INVALID_INPUT, "hsg_pivot_order: null output");
    get(f).pivot_order(out);
  });
}

int hsg_clear_analysis_cache(void) {
  return guarded([] { clear_analysis_cache(); });
}

int64_t hsg_order(const hsg_factor* f) {
  if (!f || !f->impl) return -1;
  return f->impl->order();
}

}  // extern "C"
