// Host-only C ABI entry points (no GPU needed): status strings, ordering, symbolic statistics.
#include <atomic>
#include <cmath>
#include <algorithm>
#include <string>
#include <thread>
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

int hsg_csr_inspect(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val, int32_t* flags,
                    int64_t* counts, double* defect, double* sym) {
  return guarded([&] {
    HSG_REQUIRE(n >= 0 && rowptr && flags && counts && defect, HSG_INVALID_INPUT, "hsg_csr_inspect: null argument");
    const int64_t nnz = rowptr[n];
    HSG_REQUIRE(nnz == 0 || (col && val), HSG_INVALID_INPUT, "hsg_csr_inspect: null arrays");
    // rows split over threads; every partial result is combined in thread order
    const int nt = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>({8, std::thread::hardware_concurrency() ? static_cast<int64_t>(std::thread::hardware_concurrency()) : 1, n / 4096 + 1})));
    struct Part {
      bool sorted = true, zero = false, symmetric = true;
      int64_t up = 0, lo = 0;
      double d2 = 0.0, m2 = 0.0;
    };
    std::vector<Part> parts(nt);
    // pass 1: order, zeros, triangle counts
    auto pass1 = [&](int t) {
      Part& q = parts[t];
      for (int64_t i = n * t / nt; i < n * (t + 1) / nt; ++i)
        for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) {
          const int64_t j = col[e];
          if (j < 0 || j >= n) { q.sorted = false; continue; }
          if (e > rowptr[i] && col[e - 1] >= j) q.sorted = false;
          if (val[e] == 0.0) q.zero = true;
          if (j > i) ++q.up;
          else if (j < i) ++q.lo;
        }
    };
    auto run = [&](auto&& f) {
      std::vector<std::thread> th;
      for (int t = 1; t < nt; ++t) th.emplace_back(f, t);
      f(0);
      for (auto& x : th) x.join();
    };
    run(pass1);
    bool sorted = true, zero = false;
    int64_t up = 0, lo = 0;
    for (const Part& q : parts) { sorted = sorted && q.sorted; zero = zero || q.zero; up += q.up; lo += q.lo; }
    flags[0] = sorted ? 1 : 0;
    flags[1] = zero ? 1 : 0;
    counts[0] = up;
    counts[1] = lo;
    flags[2] = 0;
    *defect = 0.0;
    if (!sorted) return;
    // pass 2 (sorted rows): the transposed entry of every (i, j) by binary search in row j
    auto pass2 = [&](int t) {
      Part& q = parts[t];
      for (int64_t i = n * t / nt; i < n * (t + 1) / nt; ++i)
        for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) {
          const int64_t j = col[e];
          const int32_t* b = col + rowptr[j];
          const int32_t* en = col + rowptr[j + 1];
          const int32_t* f = std::lower_bound(b, en, static_cast<int32_t>(i));
          const double v = val[e];
          q.m2 += v * v;
          if (f == en || *f != i) { q.symmetric = false; continue; }
          const double vt = val[rowptr[j] + (f - b)];
          q.d2 += (v - vt) * (v - vt);
          if (sym) sym[e] = 0.5 * (v + vt);
        }
    };
    run(pass2);
    bool symmetric = true;
    double d2 = 0.0, m2 = 0.0;
    for (const Part& q : parts) { symmetric = symmetric && q.symmetric; d2 += q.d2; m2 += q.m2; }
    flags[2] = symmetric ? 1 : 0;
    *defect = m2 > 0.0 ? std::sqrt(d2) / std::sqrt(m2) : 0.0;
  });
}

}  // extern "C"
