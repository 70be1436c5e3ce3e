// Symbolic analysis (see symbolic.hpp). The steps are the textbook ones (Liu's elimination tree,
// postorder, Gilbert-Ng-Peyton column counts, fundamental supernodes, relaxed amalgamation as in
// supernodal Cholesky codes), written for this project.
#include "symbolic.hpp"

#include <algorithm>
#include <chrono>
#include <map>
#include <stdexcept>

namespace hsg {
namespace {

// Lower CSC of the permuted pattern: column j lists rows i >= j (diagonal included) and the index
// of the source entry in the caller's upper CSR.
struct LowerCsc {
  std::vector<std::int64_t> ptr;
  std::vector<std::int32_t> row;
  std::vector<std::int64_t> src;
};

LowerCsc lower_csc(std::int64_t n, const std::int64_t* rp, const std::int32_t* ci, const std::vector<std::int32_t>& iperm) {
  LowerCsc L;
  L.ptr.assign(n + 1, 0);
  const std::int64_t nnz = rp[n];
  for (std::int64_t r = 0; r < n; ++r)
    for (std::int64_t p = rp[r]; p < rp[r + 1]; ++p) {
      const std::int32_t a = iperm[r], b = iperm[ci[p]];
      L.ptr[std::min(a, b) + 1]++;
    }
  for (std::int64_t j = 0; j < n; ++j) L.ptr[j + 1] += L.ptr[j];
  L.row.resize(nnz);
  L.src.resize(nnz);
  std::vector<std::int64_t> cur(L.ptr.begin(), L.ptr.end() - 1);
  for (std::int64_t r = 0; r < n; ++r)
    for (std::int64_t p = rp[r]; p < rp[r + 1]; ++p) {
      const std::int32_t a = iperm[r], b = iperm[ci[p]];
      const std::int64_t q = cur[std::min(a, b)]++;
      L.row[q] = std::max(a, b);
      L.src[q] = p;
    }
  return L;
}

std::vector<std::int32_t> etree(std::int64_t n, const LowerCsc& L) {
  // Liu: needs, for each k, the columns j < k with K(k, j) != 0 (the transpose of the strict lower part)
  std::vector<std::int64_t> tp(n + 1, 0);
  for (std::int64_t j = 0; j < n; ++j)
    for (std::int64_t p = L.ptr[j]; p < L.ptr[j + 1]; ++p)
      if (L.row[p] > j) tp[L.row[p] + 1]++;
  for (std::int64_t k = 0; k < n; ++k) tp[k + 1] += tp[k];
  std::vector<std::int32_t> tj(tp[n]);
  std::vector<std::int64_t> cur(tp.begin(), tp.end() - 1);
  for (std::int64_t j = 0; j < n; ++j)
    for (std::int64_t p = L.ptr[j]; p < L.ptr[j + 1]; ++p)
      if (L.row[p] > j) tj[cur[L.row[p]]++] = static_cast<std::int32_t>(j);
  std::vector<std::int32_t> parent(n, -1), anc(n, -1);
  for (std::int64_t k = 0; k < n; ++k)
    for (std::int64_t p = tp[k]; p < tp[k + 1]; ++p) {
      std::int32_t r = tj[p];
      while (anc[r] != -1 && anc[r] != k) { const std::int32_t t = anc[r]; anc[r] = static_cast<std::int32_t>(k); r = t; }
      if (anc[r] == -1) { anc[r] = static_cast<std::int32_t>(k); parent[r] = static_cast<std::int32_t>(k); }
    }
  return parent;
}

std::vector<std::int32_t> postorder(std::int64_t n, const std::vector<std::int32_t>& parent) {
  std::vector<std::int32_t> head(n, -1), next(n, -1), stack, post;
  post.reserve(n);
  for (std::int64_t j = n - 1; j >= 0; --j)
    if (parent[j] >= 0) { next[j] = head[parent[j]]; head[parent[j]] = static_cast<std::int32_t>(j); }
  for (std::int64_t r = 0; r < n; ++r) {
    if (parent[r] != -1) continue;
    stack.push_back(static_cast<std::int32_t>(r));
    while (!stack.empty()) {
      const std::int32_t v = stack.back();
      const std::int32_t c = head[v];
      if (c == -1) { stack.pop_back(); post.push_back(v); }
      else { head[v] = next[c]; stack.push_back(c); }
    }
  }
  return post;
}

// Column counts of L (diagonal included) for a postordered etree (Gilbert, Ng, Peyton).
std::vector<std::int64_t> column_counts(std::int64_t n, const LowerCsc& L, const std::vector<std::int32_t>& parent) {
  std::vector<std::int32_t> firstd(n, -1), maxfirst(n, -1), prevleaf(n, -1), anc(n);
  std::vector<std::int64_t> delta(n, 0);
  for (std::int64_t k = 0; k < n; ++k) {
    std::int32_t j = static_cast<std::int32_t>(k);
    delta[j] = firstd[j] == -1 ? 1 : 0;
    for (; j != -1 && firstd[j] == -1; j = parent[j]) firstd[j] = static_cast<std::int32_t>(k);
  }
  for (std::int64_t i = 0; i < n; ++i) anc[i] = static_cast<std::int32_t>(i);
  for (std::int64_t j = 0; j < n; ++j) {
    if (parent[j] != -1) delta[parent[j]]--;
    for (std::int64_t p = L.ptr[j]; p < L.ptr[j + 1]; ++p) {
      const std::int32_t i = L.row[p];
      if (i <= j || firstd[j] <= maxfirst[i]) continue;
      maxfirst[i] = firstd[j];
      const std::int32_t jprev = prevleaf[i];
      prevleaf[i] = static_cast<std::int32_t>(j);
      delta[j]++;
      if (jprev != -1) {
        std::int32_t q = jprev;
        while (q != anc[q]) q = anc[q];
        for (std::int32_t s = jprev; s != q;) { const std::int32_t sp = anc[s]; anc[s] = q; s = sp; }
        delta[q]--;
      }
    }
    if (parent[j] != -1) anc[j] = parent[j];
  }
  for (std::int64_t j = 0; j < n; ++j)
    if (parent[j] != -1) delta[parent[j]] += delta[j];
  return delta;
}

// Build every derived array from perm / first / parent.
void finalize(Symbolic& S, const std::int64_t* rp, const std::int32_t* ci) {
  const std::int64_t n = S.n;
  const std::int32_t ns = S.ns;
  S.iperm.assign(n, 0);
  for (std::int64_t i = 0; i < n; ++i) S.iperm[S.perm[i]] = static_cast<std::int32_t>(i);
  LowerCsc L = lower_csc(n, rp, ci, S.iperm);
  // children
  S.child_ptr.assign(ns + 1, 0);
  for (std::int32_t s = 0; s < ns; ++s)
    if (S.parent[s] >= 0) S.child_ptr[S.parent[s] + 1]++;
  for (std::int32_t s = 0; s < ns; ++s) S.child_ptr[s + 1] += S.child_ptr[s];
  S.children.assign(S.child_ptr[ns], 0);
  {
    std::vector<std::int32_t> cur(S.child_ptr.begin(), S.child_ptr.end() - 1);
    for (std::int32_t s = 0; s < ns; ++s)
      if (S.parent[s] >= 0) S.children[cur[S.parent[s]]++] = s;
  }
  // row structures
  std::vector<std::int32_t> mark(n, -1), buf;
  S.rowptr.assign(ns + 1, 0);
  S.rows.clear();
  for (std::int32_t s = 0; s < ns; ++s) {
    buf.clear();
    for (std::int32_t j = S.first[s]; j < S.first[s + 1]; ++j) { mark[j] = s; buf.push_back(j); }
    for (std::int32_t j = S.first[s]; j < S.first[s + 1]; ++j)
      for (std::int64_t p = L.ptr[j]; p < L.ptr[j + 1]; ++p) {
        const std::int32_t i = L.row[p];
        if (mark[i] != s) { mark[i] = s; buf.push_back(i); }
      }
    for (std::int32_t q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q) {
      const std::int32_t c = S.children[q];
      const std::int32_t kc = S.first[c + 1] - S.first[c];
      for (std::int64_t p = S.rowptr[c] + kc; p < S.rowptr[c + 1]; ++p) {
        const std::int32_t i = S.rows[p];
        if (i < S.first[s]) throw std::logic_error("symbolic: contribution row below the parent's columns");
        if (mark[i] != s) { mark[i] = s; buf.push_back(i); }
      }
    }
    std::sort(buf.begin(), buf.end());
    S.rows.insert(S.rows.end(), buf.begin(), buf.end());
    S.rowptr[s + 1] = static_cast<std::int64_t>(S.rows.size());
  }
  // panels, statistics
  S.panel_off.assign(ns + 1, 0);
  S.flops = 0.0;
  S.nnz_l = 0;
  S.max_front = 0;
  for (std::int32_t s = 0; s < ns; ++s) {
    const std::int64_t k = S.k_of(s), m = S.m_of(s);
    S.panel_off[s + 1] = S.panel_off[s] + m * k;
    S.nnz_l += k * m - k * (k - 1) / 2;
    for (std::int64_t j = 0; j < k; ++j) {
      const double r = static_cast<double>(m - j - 1);
      S.flops += r + r * (r + 1.0);
    }
    S.max_front = std::max<std::int32_t>(S.max_front, static_cast<std::int32_t>(m));
  }
  S.factor_entries = S.panel_off[ns];
  // extend-add maps
  std::vector<std::int32_t> pos(n, -1);
  S.rmap_off.assign(ns + 1, 0);
  for (std::int32_t s = 0; s < ns; ++s) S.rmap_off[s + 1] = S.rmap_off[s] + (S.m_of(s) - S.k_of(s));
  S.rmap.assign(S.rmap_off[ns], 0);
  for (std::int32_t p = 0; p < ns; ++p) {
    for (std::int64_t q = S.rowptr[p]; q < S.rowptr[p + 1]; ++q) pos[S.rows[q]] = static_cast<std::int32_t>(q - S.rowptr[p]);
    for (std::int32_t q = S.child_ptr[p]; q < S.child_ptr[p + 1]; ++q) {
      const std::int32_t c = S.children[q];
      const std::int32_t kc = S.k_of(c);
      for (std::int64_t t = S.rowptr[c] + kc; t < S.rowptr[c + 1]; ++t) {
        const std::int32_t ps = pos[S.rows[t]];
        if (ps < 0) throw std::logic_error("symbolic: contribution row missing from the parent front");
        S.rmap[S.rmap_off[c] + (t - S.rowptr[c] - kc)] = ps;
      }
    }
    for (std::int64_t q = S.rowptr[p]; q < S.rowptr[p + 1]; ++q) pos[S.rows[q]] = -1;
  }
  for (std::int32_t s = 0; s < ns; ++s)
    if (S.parent[s] < 0 && S.m_of(s) != S.k_of(s)) throw std::logic_error("symbolic: root front with contribution rows");
  // original-entry destinations
  S.dest.assign(rp[n], -1);
  for (std::int32_t s = 0; s < ns; ++s) {
    const std::int64_t m = S.m_of(s);
    for (std::int64_t q = S.rowptr[s]; q < S.rowptr[s + 1]; ++q) pos[S.rows[q]] = static_cast<std::int32_t>(q - S.rowptr[s]);
    for (std::int32_t j = S.first[s]; j < S.first[s + 1]; ++j)
      for (std::int64_t p = L.ptr[j]; p < L.ptr[j + 1]; ++p)
        S.dest[L.src[p]] = S.panel_off[s] + static_cast<std::int64_t>(j - S.first[s]) * m + pos[L.row[p]];
    for (std::int64_t q = S.rowptr[s]; q < S.rowptr[s + 1]; ++q) pos[S.rows[q]] = -1;
  }
  // height levels
  S.height.assign(ns, 0);
  std::int32_t H = 0;
  for (std::int32_t s = 0; s < ns; ++s) {
    std::int32_t h = 0;
    for (std::int32_t q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q) h = std::max(h, S.height[S.children[q]] + 1);
    S.height[s] = h;
    H = std::max(H, h);
  }
  S.nlevels = ns ? H + 1 : 0;
  S.level_ptr.assign(S.nlevels + 1, 0);
  for (std::int32_t s = 0; s < ns; ++s) S.level_ptr[S.height[s] + 1]++;
  for (std::int32_t l = 0; l < S.nlevels; ++l) S.level_ptr[l + 1] += S.level_ptr[l];
  S.level_sn.assign(ns, 0);
  {
    std::vector<std::int32_t> cur(S.level_ptr.begin(), S.level_ptr.end() - 1);
    for (std::int32_t s = 0; s < ns; ++s) S.level_sn[cur[S.height[s]]++] = s;
  }
  // contribution-block plan: CB(s) lives from level height(s) to level height(parent(s))
  S.cb_off.assign(ns, -1);
  std::map<std::int64_t, std::int64_t> freel;  // offset -> size
  std::int64_t top = 0;
  auto alloc = [&](std::int64_t size) {
    for (auto it = freel.begin(); it != freel.end(); ++it) {
      if (it->second >= size) {
        const std::int64_t off = it->first, rest = it->second - size;
        freel.erase(it);
        if (rest > 0) freel[off + size] = rest;
        return off;
      }
    }
    // extend the top (merge with a free block ending at top)
    if (!freel.empty()) {
      auto last = std::prev(freel.end());
      if (last->first + last->second == top) {
        const std::int64_t off = last->first;
        freel.erase(last);
        top = off + size;
        return off;
      }
    }
    const std::int64_t off = top;
    top += size;
    return off;
  };
  auto release = [&](std::int64_t off, std::int64_t size) {
    auto it = freel.emplace(off, size).first;
    if (it != freel.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) { pv->second += it->second; freel.erase(it); it = pv; }
    }
    auto nx = std::next(it);
    if (nx != freel.end() && it->first + it->second == nx->first) { it->second += nx->second; freel.erase(nx); }
  };
  std::int64_t peak = 0;
  for (std::int32_t l = 0; l < S.nlevels; ++l) {
    for (std::int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
      const std::int32_t s = S.level_sn[q];
      const std::int64_t c = S.m_of(s) - S.k_of(s);
      if (c > 0) S.cb_off[s] = alloc(c * c);
    }
    peak = std::max(peak, top);
    for (std::int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
      const std::int32_t s = S.level_sn[q];
      for (std::int32_t t = S.child_ptr[s]; t < S.child_ptr[s + 1]; ++t) {
        const std::int32_t c = S.children[t];
        const std::int64_t cm = S.m_of(c) - S.k_of(c);
        if (cm > 0) release(S.cb_off[c], cm * cm);
      }
    }
  }
  S.cb_arena = peak;
}

}  // namespace

Symbolic analyze_pattern(std::int64_t n, const std::int64_t* rp, const std::int32_t* ci, const std::int32_t* order,
                         const SymbolicOptions& opt) {
  Symbolic S;
  S.n = n;
  S.nnz_upper = rp[n];
  if (order) {
    S.perm.assign(order, order + n);
    std::vector<char> seen(n, 0);
    for (std::int64_t i = 0; i < n; ++i) {
      if (S.perm[i] < 0 || S.perm[i] >= n || seen[S.perm[i]]) throw std::invalid_argument("pivot order is not a permutation");
      seen[S.perm[i]] = 1;
    }
  } else {
    Adjacency g = adjacency_from_upper(n, rp, ci);
    S.perm = nested_dissection(g, opt.ordering, &S.ordering_stats);
    S.ordering_seconds = S.ordering_stats.seconds;
  }
  const auto t1 = std::chrono::steady_clock::now();
  S.iperm.assign(n, 0);
  for (std::int64_t i = 0; i < n; ++i) S.iperm[S.perm[i]] = static_cast<std::int32_t>(i);
  LowerCsc L = lower_csc(n, rp, ci, S.iperm);
  std::vector<std::int32_t> par = etree(n, L);
  {
    const std::vector<std::int32_t> post = postorder(n, par);
    std::vector<std::int32_t> p2(n);
    for (std::int64_t i = 0; i < n; ++i) p2[i] = S.perm[post[i]];
    S.perm.swap(p2);
    for (std::int64_t i = 0; i < n; ++i) S.iperm[S.perm[i]] = static_cast<std::int32_t>(i);
    L = lower_csc(n, rp, ci, S.iperm);
    par = etree(n, L);
  }
  const std::vector<std::int64_t> cc = column_counts(n, L, par);
  std::vector<std::int32_t> nchild(n, 0);
  for (std::int64_t j = 0; j < n; ++j)
    if (par[j] >= 0) nchild[par[j]]++;
  // fundamental supernodes
  std::vector<std::int32_t> fs;  // first column of each
  for (std::int64_t j = 0; j < n; ++j) {
    const bool join = j > 0 && par[j - 1] == j && cc[j - 1] == cc[j] + 1 && nchild[j] == 1;
    if (!join) fs.push_back(static_cast<std::int32_t>(j));
  }
  const std::int32_t nf = static_cast<std::int32_t>(fs.size());
  fs.push_back(static_cast<std::int32_t>(n));
  std::vector<std::int32_t> col2f(n);
  for (std::int32_t s = 0; s < nf; ++s)
    for (std::int32_t j = fs[s]; j < fs[s + 1]; ++j) col2f[j] = s;
  std::vector<std::int32_t> fpar(nf);
  std::vector<std::int64_t> fk(nf), fm(nf);
  for (std::int32_t s = 0; s < nf; ++s) {
    const std::int32_t last = fs[s + 1] - 1;
    fpar[s] = par[last] >= 0 ? col2f[par[last]] : -1;
    fk[s] = fs[s + 1] - fs[s];
    fm[s] = cc[fs[s]];
  }
  // relaxed amalgamation: merge a supernode into its parent when their columns are contiguous
  struct Node { std::int32_t lo, hi; std::int64_t k, m, zeros; std::int32_t id; };
  std::vector<Node> stack;
  std::vector<std::int32_t> rep_of(nf, -1);
  for (std::int32_t s = 0; s < nf; ++s) {
    Node cur{fs[s], fs[s + 1], fk[s], fm[s], 0, s};
    while (opt.amalgamate && !stack.empty() && fpar[stack.back().id] == s && stack.back().hi == cur.lo) {
      const Node& c = stack.back();
      const std::int64_t k = c.k + cur.k, m = c.k + cur.m;
      const double store = static_cast<double>(k) * m - static_cast<double>(k) * (k - 1) / 2.0;
      const double nzc = static_cast<double>(c.k) * c.m - static_cast<double>(c.k) * (c.k - 1) / 2.0 - c.zeros;
      const double nzp = static_cast<double>(cur.k) * cur.m - static_cast<double>(cur.k) * (cur.k - 1) / 2.0 - cur.zeros;
      const double zeros = store - nzc - nzp;
      const double frac = zeros / store;
      bool merge = k <= opt.relax_small || (k <= opt.relax_mid && frac < 0.8) ||
                   (k <= opt.relax_big && frac < 0.1) || frac < 0.05;
      if (!merge) break;
      cur.lo = c.lo;
      cur.k = k;
      cur.m = m;
      cur.zeros = static_cast<std::int64_t>(zeros + 0.5);
      rep_of[c.id] = s;  // c merged into s
      stack.pop_back();
    }
    stack.push_back(cur);
  }
  // resolve merged groups: a fundamental supernode belongs to the node of its final representative
  auto resolve = [&](std::int32_t s) {
    while (rep_of[s] >= 0) s = rep_of[s];
    return s;
  };
  std::vector<std::int32_t> newid(nf, -1), ends;
  std::int32_t ns = 0;
  for (std::int32_t s = 0; s < nf; ++s) {
    if (rep_of[s] >= 0) continue;  // merged into a later (parent) node
    newid[s] = ns++;
    ends.push_back(fs[s + 1]);
  }
  S.ns = ns;
  S.first.assign(ns + 1, 0);
  S.parent.assign(ns, -1);
  for (std::int32_t s = 0; s < ns; ++s) S.first[s + 1] = ends[s];
  for (std::int32_t s = 0; s < nf; ++s) {
    if (rep_of[s] >= 0) continue;
    S.parent[newid[s]] = fpar[s] >= 0 ? newid[resolve(fpar[s])] : -1;
  }
  finalize(S, rp, ci);
  S.symbolic_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
  return S;
}

std::int64_t move_delayed(Symbolic& S, const std::int64_t* rp, const std::int32_t* ci, const std::vector<std::int32_t>& delayed) {
  const std::int32_t ns = S.ns;
  std::vector<std::int32_t> col2sn(S.n);
  for (std::int32_t s = 0; s < ns; ++s)
    for (std::int32_t j = S.first[s]; j < S.first[s + 1]; ++j) col2sn[j] = s;
  std::vector<char> moving(S.n, 0);
  std::int64_t moved = 0;
  for (std::int32_t j : delayed) {
    if (j < 0 || j >= S.n || moving[j]) continue;
    if (S.parent[col2sn[j]] < 0) continue;
    moving[j] = 1;
    ++moved;
  }
  if (!moved) return 0;
  // new column lists (original indices), parent keeps its own columns after the arrivals
  std::vector<std::vector<std::int32_t>> incoming(ns), own(ns);
  for (std::int32_t s = 0; s < ns; ++s)
    for (std::int32_t j = S.first[s]; j < S.first[s + 1]; ++j) {
      if (moving[j]) incoming[S.parent[s]].push_back(S.perm[j]);
      else own[s].push_back(S.perm[j]);
    }
  // keep the arrivals in elimination order: children in postorder, columns in order
  std::vector<std::int32_t> perm;
  perm.reserve(S.n);
  std::vector<std::int32_t> newid(ns, -1), firsts;
  std::int32_t k = 0;
  for (std::int32_t s = 0; s < ns; ++s) {
    const std::size_t cnt = incoming[s].size() + own[s].size();
    if (cnt == 0) continue;
    newid[s] = k++;
    firsts.push_back(static_cast<std::int32_t>(perm.size()));
    perm.insert(perm.end(), incoming[s].begin(), incoming[s].end());
    perm.insert(perm.end(), own[s].begin(), own[s].end());
  }
  firsts.push_back(static_cast<std::int32_t>(perm.size()));
  std::vector<std::int32_t> parent(k, -1);
  for (std::int32_t s = 0; s < ns; ++s) {
    if (newid[s] < 0) continue;
    std::int32_t p = S.parent[s];
    while (p >= 0 && newid[p] < 0) p = S.parent[p];  // an emptied supernode passes its children up
    parent[newid[s]] = p >= 0 ? newid[p] : -1;
  }
  S.perm.swap(perm);
  S.ns = k;
  S.first.swap(firsts);
  S.parent.swap(parent);
  S.delayed_moves += moved;
  finalize(S, rp, ci);
  return moved;
}

}  // namespace hsg
