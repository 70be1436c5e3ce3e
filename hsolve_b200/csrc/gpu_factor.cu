// GpuFactor: analysis, numeric factorization driver and solves on the device (see gpu_factor.hpp).
#include "gpu_factor.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <mutex>
#include <memory>
#include <list>

#include "factor_kernels.cuh"
#include "solve_kernels.cuh"

namespace hsg {

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) HSG_THROW(HSG_INTERNAL, "CUDA error in " << what << ": " << cudaGetErrorString(e));
}

namespace {

// Process-wide cache of nested-dissection analyses keyed by the union pattern and the ordering
// seed (a hit is confirmed by comparing the whole pattern): repeated solves on one sparsity
// pattern (new values, new shifts, new Bloch wavevectors) skip the ordering and the symbolic
// factorization. It holds the analysis as computed, before any delayed-pivot re-plan.
// Beside each analysis it keeps the front plan built from it on each device (FrontPlan), so that a
// new factorization object on a known pattern neither builds nor uploads a plan.
struct AnalysisEntry {
  std::uint64_t key;
  std::uint64_t seed;
  std::vector<std::int64_t> rp;
  std::vector<std::int32_t> ci;
  std::shared_ptr<const Symbolic> sym;
  std::vector<std::shared_ptr<const FrontPlan>> plans;  // at most one per device
};

constexpr std::size_t kAnalysisCacheEntries = 8;
// panel entries per CTA of a solve sweep (fewer, busier CTAs: their waits hold fewer SMs from
// concurrent requests)
constexpr double kSolveEntriesPerCta = 32768.0;
// most parts a backward chunk's contribution-row tiles are cut into (owner + helpers)
constexpr int kSolveParts = 4;
std::mutex g_analysis_mu;
std::list<AnalysisEntry> g_analysis_cache;  // most recently used first

std::uint64_t pattern_key(const std::vector<std::int64_t>& rp, const std::vector<std::int32_t>& ci, std::uint64_t seed) {
  std::uint64_t h = 0xcbf29ce484222325ull ^ seed;
  auto mix = [&](std::uint64_t v) {
    h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
  };
  mix(rp.size());
  for (std::int64_t v : rp) mix(static_cast<std::uint64_t>(v));
  for (std::int32_t v : ci) mix(static_cast<std::uint32_t>(v));
  return h;
}

// The analysis of the pattern (rp, ci) from the cache, or computed and cached; `hit` tells which,
// and `plan` receives the cached front plan of `device` (null if none).
std::shared_ptr<const Symbolic> cached_analysis(std::int64_t n, const std::vector<std::int64_t>& rp,
                                                const std::vector<std::int32_t>& ci, const SymbolicOptions& so,
                                                int device, std::shared_ptr<const FrontPlan>& plan, bool& hit) {
  const std::uint64_t key = pattern_key(rp, ci, so.ordering.seed);
  plan.reset();
  hit = false;
  {
    std::lock_guard<std::mutex> lk(g_analysis_mu);
    for (auto it = g_analysis_cache.begin(); it != g_analysis_cache.end(); ++it) {
      if (it->key == key && it->seed == so.ordering.seed && it->rp == rp && it->ci == ci) {
        g_analysis_cache.splice(g_analysis_cache.begin(), g_analysis_cache, it);
        const AnalysisEntry& e = g_analysis_cache.front();
        for (const auto& pl : e.plans)
          if (pl->device == device) plan = pl;
        hit = true;
        return e.sym;
      }
    }
  }
  auto s = std::make_shared<const Symbolic>(analyze_pattern(n, rp.data(), ci.data(), nullptr, so));
  std::lock_guard<std::mutex> lk(g_analysis_mu);
  g_analysis_cache.push_front(AnalysisEntry{key, so.ordering.seed, rp, ci, s, {}});
  if (g_analysis_cache.size() > kAnalysisCacheEntries) g_analysis_cache.pop_back();
  return s;
}

// Keeps `plan` (built from the cached analysis `origin`) with that cache entry, if it still holds
// `origin`.
void remember_plan(const std::shared_ptr<const Symbolic>& origin, const std::shared_ptr<const FrontPlan>& plan) {
  std::lock_guard<std::mutex> lk(g_analysis_mu);
  for (auto& e : g_analysis_cache)
    if (e.sym == origin) {
      for (auto& pl : e.plans)
        if (pl->device == plan->device) {
          pl = plan;
          return;
        }
      e.plans.push_back(plan);
      return;
    }
}

// A factorization that had to move delayed pivots to their parent fronts leaves its analysis with
// those pivots moved; that structure is valid for any values on the pattern, so the cached entry
// takes it and later analyses of the pattern start without those re-plans.
void learn_delays(const std::vector<std::int64_t>& rp, const std::vector<std::int32_t>& ci, std::uint64_t seed,
                  const Symbolic& sym) {
  const std::uint64_t key = pattern_key(rp, ci, seed);
  std::lock_guard<std::mutex> lk(g_analysis_mu);
  for (auto& e : g_analysis_cache)
    if (e.key == key && e.seed == seed && e.rp == rp && e.ci == ci) {
      if (sym.delayed_moves > e.sym->delayed_moves) {
        e.sym = std::make_shared<const Symbolic>(sym);
        e.plans.clear();  // they belong to the structure before the moves
      }
      return;
    }
}

}  // namespace

void clear_analysis_cache() {
  std::lock_guard<std::mutex> lk(g_analysis_mu);
  g_analysis_cache.clear();
}

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cuda_check(cudaSetDevice(dev), "cudaSetDevice");
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Union of the upper patterns of A and B (B == null: identity), diagonal always present.
void merge_upper(std::int64_t n, const std::int64_t* arp, const std::int32_t* aci, const double* av,
                 const std::int64_t* brp, const std::int32_t* bci, const double* bv, std::vector<std::int64_t>& rp,
                 std::vector<std::int32_t>& ci, std::vector<double>& a, std::vector<double>& b) {
  rp.assign(n + 1, 0);
  ci.clear();
  a.clear();
  b.clear();
  std::vector<std::pair<std::int32_t, std::pair<double, double>>> row;
  for (std::int64_t i = 0; i < n; ++i) {
    row.clear();
    row.push_back({static_cast<std::int32_t>(i), {0.0, 0.0}});
    for (std::int64_t p = arp[i]; p < arp[i + 1]; ++p) {
      HSG_REQUIRE(aci[p] >= i && aci[p] < n, HSG_INVALID_INPUT, "A: entry (" << i << ", " << aci[p] << ") outside the upper triangle");
      HSG_REQUIRE(std::isfinite(av[p]), HSG_INVALID_INPUT, "A: non-finite entry");
      row.push_back({aci[p], {av[p], 0.0}});
    }
    if (brp) {
      for (std::int64_t p = brp[i]; p < brp[i + 1]; ++p) {
        HSG_REQUIRE(bci[p] >= i && bci[p] < n, HSG_INVALID_INPUT, "B: entry (" << i << ", " << bci[p] << ") outside the upper triangle");
        HSG_REQUIRE(std::isfinite(bv[p]), HSG_INVALID_INPUT, "B: non-finite entry");
        row.push_back({bci[p], {0.0, bv[p]}});
      }
    } else {
      row.push_back({static_cast<std::int32_t>(i), {0.0, 1.0}});
    }
    std::sort(row.begin(), row.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    for (std::size_t q = 0; q < row.size();) {
      std::size_t e = q;
      double sa = 0.0, sb = 0.0;
      while (e < row.size() && row[e].first == row[q].first) { sa += row[e].second.first; sb += row[e].second.second; ++e; }
      ci.push_back(row[q].first);
      a.push_back(sa);
      b.push_back(sb);
      q = e;
    }
    rp[i + 1] = static_cast<std::int64_t>(ci.size());
  }
}

}  // namespace

GpuFactor::GpuFactor(const hsg_options_t& opt) : opt_(opt) {
  int count = 0;
  cuda_check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
  HSG_REQUIRE(opt_.device >= 0 && opt_.device < count, HSG_INVALID_INPUT, "no CUDA device " << opt_.device);
  HSG_REQUIRE(opt_.precision == 0 || opt_.precision == 1, HSG_INVALID_INPUT, "precision must be 0 (double) or 1 (single)");
  HSG_REQUIRE(opt_.precision == 0 || (opt_.single_null_pivot_tol > 0.0 && opt_.single_null_pivot_tol < 1.0),
              HSG_INVALID_INPUT, "single_null_pivot_tol outside (0, 1)");
  HSG_REQUIRE(opt_.pivot_threshold > 0.0 && opt_.pivot_threshold <= 0.5, HSG_INVALID_INPUT, "pivot threshold outside (0, 0.5]");
  HSG_REQUIRE(opt_.null_pivot_tol > 0.0 && opt_.null_pivot_tol < 1.0, HSG_INVALID_INPUT, "null_pivot_tol outside (0, 1)");
  DeviceGuard g(opt_.device);
  cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  cuda_check(cudaEventCreate(&ev0_), "cudaEventCreate");
  cuda_check(cudaEventCreate(&ev1_), "cudaEventCreate");
  cuda_check(cudaEventCreateWithFlags(&ev_in_, cudaEventDisableTiming), "cudaEventCreate");
}

void GpuFactor::order_after_legacy_stream() { order_after(cudaStreamLegacy); }

void GpuFactor::order_after(cudaStream_t other) {
  if (other == stream_) return;
  DeviceGuard g(opt_.device);
  cuda_check(cudaEventRecord(ev_in_, other), "event on the producing stream");
  cuda_check(cudaStreamWaitEvent(stream_, ev_in_, 0), "wait for the producing stream");
}

GpuFactor::~GpuFactor() {
  DeviceGuard g(opt_.device);
  if (stream_) {
    cudaStreamSynchronize(stream_);
    clear_sweep_graphs();
    cudaStreamDestroy(stream_);
  }
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (ev_in_) cudaEventDestroy(ev_in_);
}

void GpuFactor::analyze(std::int64_t n, const std::int64_t* a_rp, const std::int32_t* a_ci, const double* a_v,
                        const std::int64_t* b_rp, const std::int32_t* b_ci, const double* b_v,
                        const std::int32_t* order) {
  HSG_REQUIRE(n > 0 && a_rp && a_ci && a_v, HSG_INVALID_INPUT, "analyze: empty pencil or null pointer");
  HSG_REQUIRE(n < (std::int64_t(1) << 31) - 1, HSG_UNSUPPORTED, "order above the 32-bit index range");
  HSG_REQUIRE(!b_rp || (b_ci && b_v), HSG_INVALID_INPUT, "analyze: incomplete B");
  DeviceGuard g(opt_.device);
  PoolStreamScope scope(stream_);
  analysed_ = false;
  factored_ = false;
  std::vector<double> av, bv;
  merge_upper(n, a_rp, a_ci, a_v, b_rp, b_ci, b_v, rp_, ci_, av, bv);
  n_ = n;
  nnz_ = rp_[n];
  std::vector<std::int32_t> perm;
  if (order) {
    perm.assign(n, -1);
    for (std::int64_t v = 0; v < n; ++v) {
      const std::int64_t p = static_cast<std::int64_t>(order[v]) - 1;
      HSG_REQUIRE(p >= 0 && p < n && perm[p] < 0, HSG_INVALID_INPUT, "pivot order is not a permutation of 1..n");
      perm[p] = static_cast<std::int32_t>(v);
    }
  }
  SymbolicOptions so;
  so.ordering.seed = opt_.ordering_seed;
  std::shared_ptr<const FrontPlan> known_plan;
  if (order) {
    sym_ = analyze_pattern(n, rp_.data(), ci_.data(), perm.data(), so);
    sym_origin_.reset();
  } else {
    bool hit = false;
    sym_origin_ = cached_analysis(n, rp_, ci_, so, opt_.device, known_plan, hit);
    sym_ = *sym_origin_;
    if (hit) {
      sym_.ordering_seconds = 0.0;
      sym_.symbolic_seconds = 0.0;
    }
  }
  cached_analysis_ = order == nullptr;
  row_.resize(nnz_);
  for (std::int64_t i = 0; i < n; ++i)
    for (std::int64_t p = rp_[i]; p < rp_[i + 1]; ++p) row_[p] = static_cast<std::int32_t>(i);
  d_a_.upload(av, stream_);
  d_b_.upload(bv, stream_);
  d_scale_.alloc(n);
  d_r_.alloc(n);
  d_cnt_.alloc(1);
  d_failed_.alloc(static_cast<std::size_t>(n));
  d_piv_.alloc(n);
  d_pidx_.alloc(n);
  if (known_plan) {
    plan_ = known_plan;
  } else {
    plan_ = make_plan();
    // the uploads ran on this object's stream: complete them before another object (on another
    // stream, possibly another thread) can take the plan from the cache
    cuda_check(cudaStreamSynchronize(stream_), "plan upload");
    if (sym_origin_) remember_plan(sym_origin_, plan_);
  }
  alloc_work();
  cuda_check(cudaStreamSynchronize(stream_), "analyze");
  inertia_ = hsg_inertia_t{-1, -1, -1, 0, 0, 0, 0, 0};
  analysed_ = true;
}

void GpuFactor::analyze_like(const GpuFactor& src) {
  HSG_REQUIRE(src.analysed_, HSG_INTERNAL, "analyze_like: source not analysed");
  HSG_REQUIRE(src.opt_.device == opt_.device, HSG_INVALID_INPUT, "analyze_like: different devices");
  DeviceGuard g(opt_.device);
  PoolStreamScope scope(stream_);
  analysed_ = false;
  factored_ = false;
  n_ = src.n_;
  nnz_ = src.nnz_;
  rp_ = src.rp_;
  ci_ = src.ci_;
  row_ = src.row_;
  sym_ = src.sym_;
  sym_origin_ = src.sym_origin_;
  plan_ = src.plan_;  // shared: the plan is immutable
  cached_analysis_ = src.cached_analysis_;
  {
    std::lock_guard<std::mutex> lk(src.capture_mu_);
    cuda_check(cudaStreamSynchronize(src.stream_), "analyze_like: source");
  }
  d_a_.alloc(src.d_a_.n);
  d_b_.alloc(std::max<std::size_t>(1, src.d_b_.n));
  cuda_check(cudaMemcpyAsync(d_a_.p, src.d_a_.p, src.d_a_.n * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "copy");
  if (src.d_b_.n) cuda_check(cudaMemcpyAsync(d_b_.p, src.d_b_.p, src.d_b_.n * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "copy");
  d_scale_.alloc(n_);
  d_r_.alloc(n_);
  d_cnt_.alloc(1);
  d_failed_.alloc(static_cast<std::size_t>(n_));
  d_piv_.alloc(n_);
  d_pidx_.alloc(n_);
  alloc_work();
  cuda_check(cudaStreamSynchronize(stream_), "analyze_like");
  inertia_ = hsg_inertia_t{-1, -1, -1, 0, 0, 0, 0, 0};
  analysed_ = true;
}

std::shared_ptr<FrontPlan> GpuFactor::make_plan() {
  const Symbolic& S = sym_;
  auto plan = std::make_shared<FrontPlan>();
  FrontPlan& P = *plan;
  P.device = opt_.device;
  P.row.upload(row_, stream_);
  P.col.upload(ci_, stream_);
  const std::int32_t ns = S.ns;
  std::vector<SnDev> sn(ns);
  std::int64_t vec = 0;
  for (std::int32_t s = 0; s < ns; ++s) {
    SnDev& d = sn[s];
    d.first = S.first[s];
    d.k = S.k_of(s);
    d.m = S.m_of(s);
    d.parent = S.parent[s];
    d.panel_off = S.panel_off[s];
    d.cb_off = d.m > d.k ? S.cb_off[s] : -1;
    d.rows_off = S.rowptr[s];
    d.rmap_off = S.rmap_off[s];
    d.vec_off = vec;
    vec += d.m - d.k;
    d.scratch_off = 0;
    d.w_off = -1;
    d.cptr_off = -1;
  }
  P.vec_total = vec;
  {
    // per pivot: panel index of its diagonal entry and its front's first column
    std::vector<std::int64_t> dpos(n_);
    std::vector<std::int32_t> pfirst(n_);
    for (std::int32_t q = 0; q < ns; ++q)
      for (int j = 0; j < sn[q].k; ++j) {
        dpos[sn[q].first + j] = sn[q].panel_off + j + static_cast<std::int64_t>(j) * sn[q].m;
        pfirst[sn[q].first + j] = sn[q].first;
      }
    P.dpos.upload(dpos, stream_);
    P.pfirst.upload(pfirst, stream_);
  }
  if (coop_max_ == 0) coop_max_ = coop_max_ctas(opt_.device);
  if (solve_coop_max_ == 0) solve_coop_max_ = solve_coop_max_ctas(opt_.device);
  std::vector<SolveTask> tasks;
  std::int32_t hcnt_total = 0;  // backward helper counters: one per 32-column chunk of every front
  std::int64_t work_max = 0;
  std::vector<int2> sbl;
  std::vector<int4> tiles;
  std::int64_t w_total = 0;
  std::vector<std::int32_t> cptr;
  std::vector<ContribEntry> cent;
  std::vector<std::int32_t> lists;
  std::vector<int2> items;
  P.levels.assign(S.nlevels, LevelPlan{});
  std::int64_t scratch_max = 0;
  for (std::int32_t l = 0; l < S.nlevels; ++l) {
    LevelPlan& L = P.levels[l];
    std::vector<std::int32_t> zero, s32, s64, app, all;
    std::int64_t maxcb = 0, scratch = 0;
    int maxm = 0;
    for (std::int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
      const std::int32_t s = S.level_sn[q];
      const int m = sn[s].m, k = sn[s].k;
      all.push_back(s);
      maxm = std::max(maxm, m);
      if (m > k) { zero.push_back(s); maxcb = std::max<std::int64_t>(maxcb, static_cast<std::int64_t>(m - k) * (m - k)); }
      if (m <= 32) s32.push_back(s);
      else if (m <= kSmallMax) s64.push_back(s);
      else {
        app.push_back(s);
        sn[s].scratch_off = scratch;
        scratch += app_scratch_doubles(m);
      }
    }
    scratch_max = std::max(scratch_max, scratch);
    auto put = [&](const std::vector<std::int32_t>& v, std::int64_t& off, int& cnt) {
      off = static_cast<std::int64_t>(lists.size());
      cnt = static_cast<int>(v.size());
      lists.insert(lists.end(), v.begin(), v.end());
    };
    put(zero, L.zero_off, L.zero_n);
    put(s32, L.s32_off, L.s32_n);
    put(s64, L.s64_off, L.s64_n);
    put(app, L.app_off, L.app_n);
    put(all, L.all_off, L.all_n);
    // solve sweeps: every front gets its children's contribution lists and a solve operator, and
    // CTAs by its panel size (about kSolveEntriesPerCta entries each, at most one per 32-row group
    // forward and one per 32-column chunk backward); a level whose CTAs would exceed the
    // co-resident bound shares what fits by panel size, or runs one CTA per front
    {
      std::int64_t wofs = 0;
      std::vector<std::int64_t> fwofs(all.size());
      std::vector<std::int32_t> hoff(all.size());
      for (std::size_t q = 0; q < all.size(); ++q) {
        const std::int32_t sq = all[q];
        SnDev& dw = sn[sq];
        fwofs[q] = wofs;
        // forward t (8 m); backward s and the entry values (16 k) and the helpers' partial sums
        wofs += std::max<std::int64_t>(8 * static_cast<std::int64_t>(dw.m),
                                       16 * static_cast<std::int64_t>(dw.k) +
                                           256 * static_cast<std::int64_t>((dw.k + 31) / 32) * (kSolveParts - 1));
        hoff[q] = hcnt_total;
        hcnt_total += (dw.k + 31) / 32;
        dw.cptr_off = static_cast<std::int64_t>(cptr.size());
        std::vector<std::int32_t> num(dw.m + 1, 0);
        for (std::int32_t e = S.child_ptr[sq]; e < S.child_ptr[sq + 1]; ++e) {
          const std::int32_t ch = S.children[e];
          const int mc = sn[ch].m - sn[ch].k;
          for (int a = 0; a < mc; ++a) num[S.rmap[S.rmap_off[ch] + a] + 1]++;
        }
        for (int i = 0; i < dw.m; ++i) num[i + 1] += num[i];
        const std::int32_t base = static_cast<std::int32_t>(cent.size());
        for (int i = 0; i <= dw.m; ++i) cptr.push_back(base + num[i]);
        cent.resize(cent.size() + num[dw.m]);
        std::vector<std::int32_t> fill(num.begin(), num.end() - 1);
        for (std::int32_t e = S.child_ptr[sq]; e < S.child_ptr[sq + 1]; ++e) {
          const std::int32_t ch = S.children[e];
          const int mc = sn[ch].m - sn[ch].k;
          for (int a = 0; a < mc; ++a) {
            ContribEntry ce;
            ce.vec_off = sn[ch].vec_off;
            ce.a = a;
            ce.mc = mc;
            cent[base + fill[S.rmap[S.rmap_off[ch] + a]]++] = ce;
          }
        }
        dw.w_off = w_total;
        w_total += static_cast<std::int64_t>(dw.m) * dw.k;
        for (int b = 0, qb = 0; b < dw.k; b += kSB, ++qb) {
          sbl.push_back(make_int2(sq, qb));
          const int be = std::min(b + kSB, dw.k);
          for (int r0 = be; r0 < dw.m; r0 += 64) tiles.push_back(make_int4(sq, qb, r0, 0));
        }
      }
      work_max = std::max(work_max, wofs);
      auto plan_tasks = [&](bool bwd, int budget, std::int64_t& off, int& ctas, bool& coop) {
        auto cap = [&](const SnDev& dd) { return std::max(1, ((bwd ? dd.k : dd.m) + 31) / 32); };
        std::vector<int> nr(all.size());
        double wsum = 0.0;
        int total = 0;
        for (std::size_t q = 0; q < all.size(); ++q) {
          const SnDev& dd = sn[all[q]];
          const double w = static_cast<double>(dd.m) * dd.k;
          wsum += w;
          nr[q] = static_cast<int>(std::min<double>(cap(dd), std::max(1.0, std::ceil(w / kSolveEntriesPerCta))));
          total += nr[q];
        }
        if (total > budget) {
          const int spare = budget - static_cast<int>(all.size());
          for (std::size_t q = 0; q < all.size(); ++q) {
            const SnDev& dd = sn[all[q]];
            const double w = static_cast<double>(dd.m) * dd.k;
            nr[q] = spare > 0 && wsum > 0.0 ? std::min(cap(dd), 1 + static_cast<int>(std::floor(spare * w / wsum))) : 1;
          }
        }
        // backward helpers: where the level's CTAs fit the co-resident bound with room to spare, the
        // contribution-row tiles of each chunk of the widest fronts are cut into up to kSolveParts
        // parts (about 16 tiles per CTA), parts 1.. on helper CTAs
        std::vector<int> parts(all.size(), 1);
        int used = 0;
        for (int v : nr) used += v;
        if (bwd && used <= budget) {
          int spare = budget - used;
          std::vector<std::size_t> by(all.size());
          std::iota(by.begin(), by.end(), std::size_t{0});
          std::stable_sort(by.begin(), by.end(), [&](std::size_t x, std::size_t y) {
            return sn[all[x]].m - sn[all[x]].k > sn[all[y]].m - sn[all[y]].k;
          });
          for (std::size_t q : by) {
            const SnDev& dd = sn[all[q]];
            const int nch = (dd.k + 31) / 32, t2 = (dd.m - dd.k + 31) / 32;
            if (nch == 0 || spare < nch) continue;
            int want = std::min({kSolveParts, std::max(1, (t2 + 4 + 15) / 16), std::max(1, t2)});
            want = std::min(want, 1 + spare / nch);
            parts[q] = want;
            spare -= nch * (want - 1);
          }
        }
        off = static_cast<std::int64_t>(tasks.size());
        coop = false;
        for (std::size_t q = 0; q < all.size(); ++q) {
          const int nch = (sn[all[q]].k + 31) / 32;
          const int helpers = bwd ? nch * (parts[q] - 1) : 0;
          for (int r = 0; r < nr[q] + helpers; ++r)
            tasks.push_back(SolveTask{all[q], r, nr[q], bwd ? parts[q] : 1, bwd ? hoff[q] : 0, 0, fwofs[q]});
          coop = coop || nr[q] > 1 || helpers > 0;
        }
        ctas = static_cast<int>(static_cast<std::int64_t>(tasks.size()) - off);
      };
      L.tiny = !all.empty();
      for (std::int32_t sq : all) L.tiny = L.tiny && sn[sq].m <= kTinyRows && sn[sq].k <= 32;
      for (int c = 0; c < kSweepChunks; ++c) {
        // a launch of c + 1 chunks runs (c + 1) CTAs per task: the co-resident bound is shared
        const int budget = solve_coop_max_ / (c + 1);
        plan_tasks(false, budget, L.fwd_task_off[c], L.fwd_ctas[c], L.fwd_coop[c]);
        plan_tasks(true, budget, L.bwd_task_off[c], L.bwd_ctas[c], L.bwd_coop[c]);
      }
    }
    // cooperative launch when the level's panel fronts fit the co-resident grid; CTAs apportioned
    // by m^2, for the whole device and for the shared budget (a third of it, used while several
    // shifts are factorized at once)
    const int shared_max = std::max(1, coop_max_ / kSharedParts);
    if (!app.empty() && static_cast<int>(app.size()) <= coop_max_) {
      int mmax = 0;
      for (std::int32_t s : app) mmax = std::max(mmax, sn[s].m);
      if (mmax >= kCoopMinFront) {
        auto plan_ctas = [&](int budget, std::int64_t& off, int& ctas) {
          std::vector<double> wts(app.size());
          double wsum = 0.0;
          for (std::size_t q = 0; q < app.size(); ++q) {
            const double m = sn[app[q]].m;
            wts[q] = m * m;
            wsum += wts[q];
          }
          std::vector<int> nr(app.size());
          int total = 0;
          for (std::size_t q = 0; q < app.size(); ++q) {
            // about 16 tiles of 64 x 64 per CTA at the first panel: fewer CTAs wait at the front's
            // barriers, which leaves SMs to concurrent requests (served throughput +11 % on the
            // n = 1e5 box against 8 tiles, one request 2 % slower)
            const double want = std::ceil(wts[q] / (2.0 * 64 * 64 * 16));
            nr[q] = static_cast<int>(std::max(1.0, std::min<double>(want, budget)));
            total += nr[q];
          }
          if (total > budget) {
            const int spare = budget - static_cast<int>(app.size());
            total = 0;
            for (std::size_t q = 0; q < app.size(); ++q) {
              nr[q] = 1 + static_cast<int>(std::floor(spare * wts[q] / wsum));
              total += nr[q];
            }
          }
          std::vector<std::int32_t> starts(app.size() + 1, 0);
          for (std::size_t q = 0; q < app.size(); ++q) starts[q + 1] = starts[q] + nr[q];
          off = static_cast<std::int64_t>(lists.size());
          lists.insert(lists.end(), starts.begin(), starts.end());
          ctas = starts.back();
        };
        L.coop = true;
        plan_ctas(coop_max_, L.cta_off, L.coop_ctas);
        L.coop_shared = static_cast<int>(app.size()) <= shared_max;
        if (L.coop_shared) plan_ctas(shared_max, L.cta_off_shared, L.coop_ctas_shared);
        L.done_slot = P.ncoop++;
      }
    }
    L.maxm = maxm;
    L.zero_chunks = static_cast<int>(std::max<std::int64_t>(1, std::min<std::int64_t>(64, (maxcb + 4095) / 4096)));
    // extend-add items by child rank
    int maxrank = 0;
    for (std::int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
      const std::int32_t s = S.level_sn[q];
      maxrank = std::max(maxrank, S.child_ptr[s + 1] - S.child_ptr[s]);
    }
    for (int r = 0; r < maxrank; ++r) {
      const std::int64_t off = static_cast<std::int64_t>(items.size());
      for (std::int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
        const std::int32_t s = S.level_sn[q];
        if (S.child_ptr[s] + r >= S.child_ptr[s + 1]) continue;
        const std::int32_t c = S.children[S.child_ptr[s] + r];
        const int mc = sn[c].m - sn[c].k;
        for (int b0 = 0; b0 < mc; b0 += kExtendAddCols) items.push_back(make_int2(c, b0));
      }
      const int cnt = static_cast<int>(items.size() - off);
      if (cnt) L.ea.push_back({off, cnt});
    }
  }
  std::vector<std::int32_t> rows(S.rows.begin(), S.rows.end());
  {
    // inertia-only counts: the panels of one level packed at the start of an arena (the next level
    // reuses it), and the pencil's entries grouped by the level of the front they scatter into
    std::vector<SnDev> snc = sn;
    std::vector<std::int32_t> level_of(ns, 0);
    P.arena_entries = 1;
    for (std::int32_t l = 0; l < S.nlevels; ++l) {
      std::int64_t off = 0;
      for (std::int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
        const std::int32_t s = S.level_sn[q];
        level_of[s] = l;
        snc[s].panel_off = off;
        off += static_cast<std::int64_t>(sn[s].m) * sn[s].k;
      }
      P.levels[l].arena_used = off;
      P.arena_entries = std::max(P.arena_entries, off);
    }
    std::vector<std::int64_t> dest_cnt(nnz_), lcount(S.nlevels + 1, 0);
    std::vector<std::int32_t> ent_level(nnz_);
    for (std::int64_t p = 0; p < nnz_; ++p) {
      const std::int64_t dst = S.dest[p];
      const std::int32_t s = static_cast<std::int32_t>(
          std::upper_bound(S.panel_off.begin(), S.panel_off.begin() + ns + 1, dst) - S.panel_off.begin() - 1);
      dest_cnt[p] = dst - S.panel_off[s] + snc[s].panel_off;
      ent_level[p] = level_of[s];
      lcount[level_of[s] + 1]++;
    }
    for (std::int32_t l = 0; l < S.nlevels; ++l) lcount[l + 1] += lcount[l];
    std::vector<std::int64_t> ent_idx(std::max<std::int64_t>(1, nnz_));
    std::vector<std::int64_t> fill(lcount.begin(), lcount.end() - 1);
    for (std::int64_t p = 0; p < nnz_; ++p) ent_idx[fill[ent_level[p]]++] = p;
    for (std::int32_t l = 0; l < S.nlevels; ++l) {
      P.levels[l].ent_off = lcount[l];
      P.levels[l].ent_n = lcount[l + 1] - lcount[l];
    }
    P.sn_cnt.upload(snc, stream_);
    P.dest_cnt.upload(dest_cnt, stream_);
    P.ent_idx.upload(ent_idx, stream_);
  }
  P.sn.upload(sn, stream_);
  P.lists.upload(lists, stream_);
  P.items.upload(items, stream_);
  P.rmap.upload(S.rmap, stream_);
  P.rows.upload(rows, stream_);
  P.child_ptr.upload(S.child_ptr, stream_);
  P.children.upload(S.children, stream_);
  P.iperm.upload(S.iperm, stream_);
  P.dest.upload(S.dest, stream_);
  P.tasks.upload(tasks, stream_);
  P.hcnt_total = hcnt_total;
  P.cptr.upload(cptr, stream_);
  P.cent.upload(cent, stream_);
  P.sbl.upload(sbl, stream_);
  P.tiles.upload(tiles, stream_);
  P.nsbl = static_cast<int>(sbl.size());
  P.ntiles = static_cast<int>(tiles.size());
  P.scratch_max = scratch_max;
  P.work_max = work_max;
  P.w_total = w_total;
  return plan;
}

void GpuFactor::alloc_work() {
  clear_sweep_graphs();  // captured launches name the buffers and the plan being replaced
  const FrontPlan& P = *plan_;
  const std::size_t fe = static_cast<std::size_t>(std::max<std::int64_t>(1, sym_.factor_entries));
  const std::size_t cbe = static_cast<std::size_t>(std::max<std::int64_t>(1, sym_.cb_arena));
  const std::size_t we = static_cast<std::size_t>(std::max<std::int64_t>(1, P.w_total));
  if (single()) {
    d_panels_f_.alloc(fe);
    d_cb_f_.alloc(cbe);
    d_w_f_.alloc(we);
  } else {
    d_panels_.alloc(fe);
    d_cb_.alloc(cbe);
    d_w_.alloc(we);
  }
  d_scratch_.alloc(static_cast<std::size_t>(std::max<std::int64_t>(1, P.scratch_max)));
  d_level_done_.alloc(static_cast<std::size_t>(std::max(1, P.ncoop)));
  d_work_.alloc(static_cast<std::size_t>(std::max<std::int64_t>(1, P.work_max)) * kSweepChunks);
  d_err_.alloc(1);
  d_sweep_cnt_.alloc(static_cast<std::size_t>(3 * std::max(1, sym_.ns) + P.hcnt_total) * kSweepChunks);
  w_ready_ = false;
}

void GpuFactor::build_plan() {
  plan_ = make_plan();
  sym_origin_.reset();
  alloc_work();
}

template <> double* GpuFactor::panels_of<double>() { return d_panels_.p; }
template <> float* GpuFactor::panels_of<float>() { return d_panels_f_.p; }
template <> double* GpuFactor::cb_of<double>() { return d_cb_.p; }
template <> float* GpuFactor::cb_of<float>() { return d_cb_f_.p; }
template <> double* GpuFactor::w_of<double>() { return d_w_.p; }
template <> float* GpuFactor::w_of<float>() { return d_w_f_.p; }

std::size_t GpuFactor::factor_bytes() const {
  const std::size_t el = single() ? sizeof(float) : sizeof(double);
  return el * (d_panels_.n + d_panels_f_.n + d_w_.n + d_w_f_.n);
}

void GpuFactor::run_numeric(double alpha, double beta, bool detection, bool count_only) {
  if (single()) run_numeric_t<float>(alpha, beta, detection, count_only);
  else run_numeric_t<double>(alpha, beta, detection, count_only);
}

template <class R>
void GpuFactor::run_numeric_t(double alpha, double beta, bool detection, bool count_only) {
  cudaStream_t s = stream_;
  R* panels = panels_of<R>();
  R* cb = cb_of<R>();
  const SnDev* sn = plan_->sn.p;
  if (count_only) {
    // the level's panels live in the arena; entries are scattered level by level below
    if constexpr (sizeof(R) == 8) { d_arena_.alloc(static_cast<std::size_t>(plan_->arena_entries)); panels = reinterpret_cast<R*>(d_arena_.p); }
    else { d_arena_f_.alloc(static_cast<std::size_t>(plan_->arena_entries)); panels = reinterpret_cast<R*>(d_arena_f_.p); }
    sn = plan_->sn_cnt.p;
  }
  cuda_check(cudaMemsetAsync(d_cnt_.p, 0, sizeof(FactorCounters), s), "memset counters");
  cuda_check(cudaMemsetAsync(d_level_done_.p, 0, d_level_done_.n * sizeof(int), s), "memset level flags");
  launch_fill(d_scale_.p, n_, 1.0, s);
  if (opt_.scaling) {
    cuda_check(cudaMemsetAsync(d_r_.p, 0, n_ * sizeof(unsigned long long), s), "memset r");
    for (int it = 0; it < 10; ++it) {
      launch_scale_rowmax(nnz_, plan_->row.p, plan_->col.p, d_a_.p, d_b_.p, alpha, beta, d_scale_.p, d_r_.p, s);
      launch_scale_update(n_, d_scale_.p, d_r_.p, s);
    }
  }
  if (count_only) {
    launch_amax(nnz_, plan_->row.p, plan_->col.p, d_a_.p, d_b_.p, alpha, beta, d_scale_.p, d_cnt_.p, s);
  } else {
    cuda_check(cudaMemsetAsync(panels, 0, sym_.factor_entries * sizeof(R), s), "memset panels");
    launch_scatter<R>(nnz_, plan_->row.p, plan_->col.p, d_a_.p, d_b_.p, alpha, beta, d_scale_.p, plan_->dest.p, panels, d_cnt_.p, s);
  }
  FactorParams prm;
  prm.u = opt_.pivot_threshold;
  // null pivots relative to the largest scaled entry: 1e-8 for FP64 factors, 1e-4 for FP32
  // (include/hsolve/factor.hpp:279-283 in hsolve)
  prm.null_tol = detection ? (single() ? opt_.single_null_pivot_tol : opt_.null_pivot_tol) : 0.0;
  prm.cnt = d_cnt_.p;
  prm.failed_cap = static_cast<std::int32_t>(n_);
  const std::int32_t* lists = plan_->lists.p;
  for (const LevelPlan& L : plan_->levels) {
    if (count_only) {
      cuda_check(cudaMemsetAsync(panels, 0, static_cast<std::size_t>(L.arena_used) * sizeof(R), s), "memset arena");
      launch_scatter_list<R>(plan_->ent_idx.p + L.ent_off, L.ent_n, plan_->row.p, plan_->col.p, d_a_.p, d_b_.p, alpha, beta,
                             d_scale_.p, plan_->dest_cnt.p, panels, s);
    }
    launch_zero_cb<R>(lists + L.zero_off, L.zero_n, L.zero_chunks, sn, cb, s);
    for (const auto& ea : L.ea) launch_extend_add<R>(plan_->items.p + ea.first, ea.second, sn, plan_->rmap.p, panels, cb, s);
    launch_front_small<R>(32, lists + L.s32_off, L.s32_n, sn, panels, cb, d_piv_.p, d_pidx_.p, prm, d_cnt_.p, d_failed_.p, s);
    launch_front_small<R>(kSmallMax, lists + L.s64_off, L.s64_n, sn, panels, cb, d_piv_.p, d_pidx_.p, prm, d_cnt_.p, d_failed_.p, s);
    if (shared_ ? L.coop_shared : L.coop) {
      const std::int64_t cta_off = shared_ ? L.cta_off_shared : L.cta_off;
      const int ctas = shared_ ? L.coop_ctas_shared : L.coop_ctas;
      cuda_check(launch_front_coop<R>(lists + L.app_off, lists + cta_off, L.app_n, ctas, sn, panels, cb,
                                      d_scratch_.p, d_piv_.p, d_pidx_.p, prm, d_cnt_.p, d_failed_.p,
                                      d_level_done_.p + L.done_slot, s),
                 "cooperative front launch");
    } else {
      launch_front_app<R>(lists + L.app_off, L.app_n, sn, panels, cb, d_scratch_.p, d_piv_.p, d_pidx_.p, prm, d_cnt_.p, d_failed_.p, s);
    }
  }
  cuda_check(cudaGetLastError(), "factorization launch");
}

template void GpuFactor::run_numeric_t<double>(double, double, bool, bool);
template void GpuFactor::run_numeric_t<float>(double, double, bool, bool);

hsg_inertia_t GpuFactor::factorize(double alpha, double beta, bool detection, bool shared) {
  return run_factorization(alpha, beta, detection, shared, false);
}

hsg_inertia_t GpuFactor::count(double alpha, double beta, bool detection, bool shared) {
  const hsg_inertia_t in = run_factorization(alpha, beta, detection, shared, true);
  factored_ = false;  // no factor was kept
  return in;
}

hsg_inertia_t GpuFactor::run_factorization(double alpha, double beta, bool detection, bool shared, bool count_only) {
  shared_ = shared;
  HSG_REQUIRE(analysed_, HSG_INTERNAL, "factorize before analyze");
  HSG_REQUIRE(std::isfinite(alpha) && std::isfinite(beta), HSG_INVALID_INPUT, "non-finite alpha / beta");
  DeviceGuard g(opt_.device);
  PoolStreamScope scope(stream_);
  factored_ = false;
  w_ready_ = false;
  const auto t0 = std::chrono::steady_clock::now();
  FactorCounters c{};
  int replans = 0;
  std::int64_t delayed = 0;
  for (;;) {
    cuda_check(cudaEventRecord(ev0_, stream_), "event");
    run_numeric(alpha, beta, detection, count_only);
    cuda_check(cudaEventRecord(ev1_, stream_), "event");
    cuda_check(cudaMemcpyAsync(&c, d_cnt_.p, sizeof(c), cudaMemcpyDeviceToHost, stream_), "counters");
    cuda_check(cudaStreamSynchronize(stream_), "factorization");
    {
      float ms = 0.0f;
      cuda_check(cudaEventElapsedTime(&ms, ev0_, ev1_), "event time");
      dstats_.factor_ms += ms;
      dstats_.factorizations += 1;
    }
    HSG_REQUIRE(c.sync_timeouts == 0, HSG_INTERNAL, "factorization: a front barrier timed out");
    if (c.failed == 0) break;
    HSG_REQUIRE(replans < 16, HSG_FACTORIZATION_FAILED, "delayed pivots could not be placed after " << replans << " re-plans");
    const std::int64_t nf = std::min<std::int64_t>(static_cast<std::int64_t>(c.failed), n_);
    std::vector<std::int32_t> failed(nf);
    cuda_check(cudaMemcpy(failed.data(), d_failed_.p, nf * sizeof(std::int32_t), cudaMemcpyDeviceToHost), "failed list");
    const std::int64_t moved = move_delayed(sym_, rp_.data(), ci_.data(), failed);
    HSG_REQUIRE(moved > 0, HSG_FACTORIZATION_FAILED, "pivots failed in root fronts");
    delayed += moved;
    ++replans;
    build_plan();
  }
  inertia_.neg = static_cast<std::int64_t>(c.neg);
  inertia_.zero = static_cast<std::int64_t>(c.zero);
  inertia_.pos = n_ - inertia_.neg - inertia_.zero;
  inertia_.null_pivots = static_cast<std::int64_t>(c.zero);
  inertia_.two_by_two = static_cast<std::int64_t>(c.two_by_two);
  inertia_.delayed_pivots = sym_.delayed_moves;
  inertia_.replans = replans;
  if (replans > 0 && cached_analysis_) learn_delays(rp_, ci_, opt_.ordering_seed, sym_);
  inertia_.valid = c.zero == 0 ? 1 : 0;
  factored_ = inertia_.valid != 0;
  last_factor_s_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  (void)delayed;
  return inertia_;
}

void GpuFactor::solve(double* b, std::int64_t nrhs, std::int64_t ldb, bool on_device) {
  HSG_REQUIRE(factored_, HSG_INTERNAL, "solve without a valid factorization");
  HSG_REQUIRE(nrhs >= 0 && ldb >= n_, HSG_INVALID_INPUT, "solve: nrhs < 0 or ldb < n");
  if (nrhs == 0) return;
  HSG_REQUIRE(b, HSG_INVALID_INPUT, "solve: null right-hand side");
  DeviceGuard g(opt_.device);
  PoolStreamScope scope(stream_);
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t s = stream_;
  const int nr = static_cast<int>(nrhs);
  d_xwork_.alloc(static_cast<std::size_t>(n_) * nr);
  d_vec_.alloc(static_cast<std::size_t>(std::max<std::int64_t>(1, plan_->vec_total)) * nr);
  double* db = b;
  std::int64_t ld = ldb;
  if (!on_device) {
    d_btmp_.alloc(static_cast<std::size_t>(n_) * nr);
    cuda_check(cudaMemcpy2DAsync(d_btmp_.p, n_ * sizeof(double), b, ldb * sizeof(double), n_ * sizeof(double), nr,
                                 cudaMemcpyHostToDevice, s), "H2D rhs");
    db = d_btmp_.p;
    ld = n_;
  }
  cuda_check(cudaMemsetAsync(d_err_.p, 0, sizeof(int), s), "reset solve status");
  cuda_check(cudaEventRecord(ev0_, s), "event");
  build_solve_operator();
  launch_gather_scale(n_, nr, db, ld, d_scale_.p, plan_->iperm.p, d_xwork_.p, s);
  run_sweeps(d_xwork_.p, d_vec_.p, nr, true);
  launch_scatter_scale(n_, nr, db, ld, d_scale_.p, plan_->iperm.p, d_xwork_.p, s);
  cuda_check(cudaEventRecord(ev1_, s), "event");
  cuda_check(cudaGetLastError(), "solve launch");
  if (!on_device) {
    cuda_check(cudaMemcpy2DAsync(b, ldb * sizeof(double), d_btmp_.p, n_ * sizeof(double), n_ * sizeof(double), nr,
                                 cudaMemcpyDeviceToHost, s), "D2H rhs");
  }
  int err = 0;
  cuda_check(cudaMemcpyAsync(&err, d_err_.p, sizeof(int), cudaMemcpyDeviceToHost, s), "solve status");
  cuda_check(cudaStreamSynchronize(s), "solve");
  HSG_REQUIRE(err == 0, HSG_INTERNAL, "solve: a wait between the CTAs of a front timed out");
  {
    float ms = 0.0f;
    cuda_check(cudaEventElapsedTime(&ms, ev0_, ev1_), "event time");
    dstats_.solve_ms += ms;
    dstats_.solves += 1;
    dstats_.solve_columns += nrhs;
  }
  last_solve_s_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

std::size_t GpuFactor::solve_scratch_doubles(std::int64_t nrhs) const {
  // contribution vectors of one sweep launch: 8 columns per chunk
  const std::int64_t nc = std::min<std::int64_t>(8 * kSweepChunks, nrhs);
  return static_cast<std::size_t>(n_ * nrhs + std::max<std::int64_t>(1, plan_->vec_total) * nc);
}

void GpuFactor::solve_with_scratch(double* b, std::int64_t nrhs, std::int64_t ldb, double* scratch,
                                   std::size_t cap) {
  HSG_REQUIRE(factored_, HSG_INTERNAL, "solve without a valid factorization");
  HSG_REQUIRE(nrhs >= 0 && ldb >= n_, HSG_INVALID_INPUT, "solve: nrhs < 0 or ldb < n");
  if (nrhs == 0) return;
  HSG_REQUIRE(b && scratch, HSG_INVALID_INPUT, "solve: null right-hand side or scratch");
  const std::size_t need = solve_scratch_doubles(nrhs);
  HSG_REQUIRE(need <= cap, HSG_INVALID_INPUT,
              "solve needs " << need << " doubles of scratch for n = " << n_ << " and nrhs = " << nrhs << ", "
                             << cap << " are available; pass fewer right-hand sides per call");
  DeviceGuard g(opt_.device);
  cudaStream_t s = stream_;
  const int nr = static_cast<int>(nrhs);
  double* xwork = scratch;
  double* vec = scratch + static_cast<std::size_t>(n_) * nr;
  cuda_check(cudaMemsetAsync(d_err_.p, 0, sizeof(int), s), "reset solve status");
  build_solve_operator();
  launch_gather_scale(n_, nr, b, ldb, d_scale_.p, plan_->iperm.p, xwork, s);
  run_sweeps(xwork, vec, nr, false);  // no graph: instantiating one may allocate
  launch_scatter_scale(n_, nr, b, ldb, d_scale_.p, plan_->iperm.p, xwork, s);
  cuda_check(cudaGetLastError(), "solve launch");
  int err = 0;
  cuda_check(cudaMemcpyAsync(&err, d_err_.p, sizeof(int), cudaMemcpyDeviceToHost, s), "solve status");
  cuda_check(cudaStreamSynchronize(s), "solve");
  HSG_REQUIRE(err == 0, HSG_INTERNAL, "solve: a wait between the CTAs of a front timed out");
}

void GpuFactor::clear_sweep_graphs() {
  for (SweepGraph& g : graphs_) cudaGraphExecDestroy(g.exec);
  graphs_.clear();
}

void GpuFactor::run_sweeps(double* xwork, double* vec, int nr, bool graph) {
  auto direct = [&] {
    if (single()) run_sweeps_t<float>(xwork, vec, nr);
    else run_sweeps_t<double>(xwork, vec, nr);
  };
  if (!graph || !graphs_ok_) return direct();
  for (const SweepGraph& g : graphs_)
    if (g.xwork == xwork && g.vec == vec && g.nr == nr) {
      note_launches(g.launches);
      cuda_check(cudaGraphLaunch(g.exec, stream_), "solve sweeps (graph)");
      return;
    }
  // capture the sequence once; where capturing is refused (e.g. a cooperative launch), launch
  // directly from now on
  const long long l0 = hsg_kernel_launches();
  cudaGraph_t cg = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::unique_lock<std::mutex> lk(capture_mu_);
  bool ok = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    try {
      direct();
    } catch (const Error&) {
      ok = false;
    }
    ok = cudaStreamEndCapture(stream_, &cg) == cudaSuccess && ok && cg;
    ok = ok && cudaGraphInstantiate(&exec, cg, 0) == cudaSuccess;
    if (cg) cudaGraphDestroy(cg);
  }
  lk.unlock();
  const long long captured = hsg_kernel_launches() - l0;
  note_launches(-captured);  // counted when the graph runs
  if (!ok) {
    cudaGetLastError();  // the failed capture's error is not sticky
    graphs_ok_ = false;
    return direct();
  }
  graphs_.push_back(SweepGraph{xwork, vec, nr, captured, exec});
  note_launches(captured);
  cuda_check(cudaGraphLaunch(exec, stream_), "solve sweeps (graph)");
}

template <class F>
void GpuFactor::run_sweeps_t(double* xwork, double* vec, int nr) {
  cudaStream_t s = stream_;
  const F* panels = panels_of<F>();
  const F* W = w_of<F>();
  const SolveTask* tasks = plan_->tasks.p;
  const int ns = sym_.ns;
  int* fcnt = d_sweep_cnt_.p;
  int* bcnt = fcnt + ns;
  int* arrive = bcnt + ns;
  int* hcnt = arrive + ns;
  // launches carry up to kSweepChunks chunks of 8 right-hand sides, each with its own contribution
  // vectors (vec_total x 8), work array and counters
  const int span = 8 * kSweepChunks;
  for (int c0 = 0; c0 < nr; c0 += span) {
    SweepChunks ck;
    ck.ncols = std::min(span, nr - c0);
    ck.cnt_stride = 3 * ns + plan_->hcnt_total;
    ck.x_stride = 8 * n_;
    ck.vec_stride = 8 * std::max<std::int64_t>(1, plan_->vec_total);
    ck.work_stride = std::max<std::int64_t>(1, plan_->work_max);
    const int c = (ck.ncols + 7) / 8 - 1;
    double* xw = xwork + static_cast<std::int64_t>(c0) * n_;
    cuda_check(cudaMemsetAsync(d_sweep_cnt_.p, 0, d_sweep_cnt_.n * sizeof(int), s), "reset sweep counters");
    for (const LevelPlan& L : plan_->levels) {
      if (L.tiny)  // one CTA per task in the plan (nr = 1): one warp per front here
        cuda_check(launch_fwd_tiny<F>(tasks + L.fwd_task_off[c], L.fwd_ctas[c], plan_->sn.p, plan_->cptr.p, plan_->cent.p,
                                      W, d_pidx_.p, xw, n_, vec, ck, s),
                   "forward solve");
      else
        cuda_check(launch_fwd_level<F>(tasks + L.fwd_task_off[c], L.fwd_ctas[c], L.fwd_coop[c], plan_->sn.p,
                                       plan_->cptr.p, plan_->cent.p, W, d_pidx_.p, xw, n_, vec, ck, d_work_.p, fcnt,
                                       d_err_.p, s),
                   "forward solve");
    }
    launch_solve_diag_flat<F>(n_, plan_->dpos.p, plan_->pfirst.p, panels, d_piv_.p, d_pidx_.p, xw, n_, ck.ncols, s);
    for (auto it = plan_->levels.rbegin(); it != plan_->levels.rend(); ++it) {
      if (it->tiny)
        cuda_check(launch_bwd_tiny<F>(tasks + it->bwd_task_off[c], it->bwd_ctas[c], plan_->sn.p, plan_->rows.p, W,
                                      d_pidx_.p, xw, n_, ck, s),
                   "backward solve");
      else
        cuda_check(launch_bwd_level<F>(tasks + it->bwd_task_off[c], it->bwd_ctas[c], it->bwd_coop[c], plan_->sn.p,
                                       plan_->rows.p, W, d_pidx_.p, xw, n_, ck, d_work_.p, bcnt, arrive, hcnt, d_err_.p, s),
                   "backward solve");
    }
  }
}

void GpuFactor::build_solve_operator() {
  if (w_ready_) return;
  if (single()) build_solve_operator_t<float>();
  else build_solve_operator_t<double>();
  w_ready_ = true;
}

template <class F>
void GpuFactor::build_solve_operator_t() {
  launch_sb_build<F>(plan_->sbl.p, plan_->nsbl, plan_->tiles.p, plan_->ntiles, plan_->sn.p, panels_of<F>(), d_piv_.p, w_of<F>(), stream_);
}

void GpuFactor::release() {
  factored_ = false;
  inertia_.valid = 0;
}

hsg_estimate_t GpuFactor::estimate() const {
  HSG_REQUIRE(analysed_, HSG_INTERNAL, "estimate before analyze");
  hsg_estimate_t e{};
  e.factor_entries = sym_.factor_entries;
  e.nnz_l = sym_.nnz_l;
  e.flops = sym_.flops;
  const double el = single() ? 4.0 : 8.0;  // bytes of a factor entry
  e.device_mb = (el * static_cast<double>(sym_.factor_entries + sym_.cb_arena) + 8.0 * static_cast<double>(4 * nnz_ + 4 * n_)) / 1e6;
  e.supernodes = sym_.ns;
  e.levels = sym_.nlevels;
  e.max_front = sym_.max_front;
  e.ordering_s = sym_.ordering_seconds;
  e.analyze_s = sym_.ordering_seconds + sym_.symbolic_seconds;
  return e;
}

void GpuFactor::pivot_order(std::int32_t* out) const {
  HSG_REQUIRE(analysed_, HSG_INTERNAL, "pivot_order before analyze");
  for (std::int64_t p = 0; p < n_; ++p) out[sym_.perm[p]] = static_cast<std::int32_t>(p + 1);
}

}  // namespace hsg
