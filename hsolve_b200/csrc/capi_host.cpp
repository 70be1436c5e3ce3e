// Host-only C ABI entry points (no GPU needed): status strings, ordering, symbolic statistics.
#include <atomic>
#include <cmath>
#include <string>
#include <vector>

#include "common.hpp"
#include "hsg.h"
#include "symbolic.hpp"

namespace hsg {
namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
}  // namespace
void set_last_error(const std::string& msg) { g_last_error = msg; }
void note_launches(long long count) { g_launches.fetch_add(count, std::memory_order_relaxed); }
}  // namespace hsg

using namespace hsg;

extern "C" {

const char* hsg_status_string(int status) {
  switch (status) {
    case HSG_OK: return "ok";
    case HSG_INVALID_INPUT: return "invalid_input";
    case HSG_IO: return "io";
    case HSG_NOT_HERMITIAN: return "not_hermitian";
    case HSG_UNSUPPORTED: return "unsupported";
    case HSG_FACTORIZATION_FAILED: return "factorization_failed";
    case HSG_SINGULAR: return "singular";
    case HSG_OUT_OF_MEMORY_BUDGET: return "out_of_memory_budget";
    case HSG_NOT_CONVERGED: return "not_converged";
    case HSG_INTERNAL: return "internal";
    default: return "unknown";
  }
}

const char* hsg_last_error(void) { return g_last_error.c_str(); }

int64_t hsg_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

void hsg_default_options(hsg_options_t* opt) {
  if (!opt) return;
  opt->precision = 0;
  opt->null_pivot_tol = 1e-8;
  opt->single_null_pivot_tol = 1e-4;
  opt->pivot_threshold = 0.01;
  opt->device = 0;
  opt->ordering_seed = 2026;
  opt->scaling = 1;
}

int hsg_compute_ordering(int64_t n, const int64_t* rowptr, const int32_t* col, uint64_t seed, int32_t* out) {
  return guarded([&] {
    HSG_REQUIRE(n >= 0 && rowptr && col && out, HSG_INVALID_INPUT, "hsg_compute_ordering: null argument");
    Adjacency g = adjacency_from_upper(n, rowptr, col);
    OrderingOptions o;
    o.seed = seed;
    const std::vector<std::int32_t> order = nested_dissection(g, o);
    for (int64_t i = 0; i < n; ++i) out[order[i]] = static_cast<int32_t>(i + 1);
  });
}

int hsg_symbolic_stats(int64_t n, const int64_t* rowptr, const int32_t* col, const int32_t* pivot_order,
                       int32_t amalgamate, hsg_estimate_t* out) {
  return guarded([&] {
    HSG_REQUIRE(n > 0 && rowptr && col && out, HSG_INVALID_INPUT, "hsg_symbolic_stats: bad argument");
    std::vector<std::int32_t> order;
    if (pivot_order) {
      order.assign(n, -1);
      for (int64_t v = 0; v < n; ++v) {
        const int64_t p = pivot_order[v] - 1;
        HSG_REQUIRE(p >= 0 && p < n && order[p] < 0, HSG_INVALID_INPUT, "pivot order is not a permutation");
        order[p] = static_cast<std::int32_t>(v);
      }
    }
    SymbolicOptions so;
    so.amalgamate = amalgamate != 0;
    Symbolic s = analyze_pattern(n, rowptr, col, pivot_order ? order.data() : nullptr, so);
    out->factor_entries = s.factor_entries;
    out->nnz_l = s.nnz_l;
    out->flops = s.flops;
    out->device_mb = 8.0 * (s.factor_entries + s.cb_arena) / 1e6;
    out->supernodes = s.ns;
    out->levels = s.nlevels;
    out->max_front = s.max_front;
    out->ordering_s = s.ordering_seconds;
    out->analyze_s = s.ordering_seconds + s.symbolic_seconds;
  });
}

}  // extern "C"
