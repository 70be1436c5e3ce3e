// Multilevel nested dissection (see ordering.hpp). Replaces hsolve's compute_ordering
// (src/factor/ordering.cpp:315; options include/hsolve/factor.hpp:197-242) with the same
// published scheme: heavy-edge matching, greedy graph growing + FM on the coarsest graph, FM
// refinement while uncoarsening, a minimum vertex cover of the cut edges (Konig) as vertex
// separator, node-FM separator refinement; separators ordered last, leaves by minimum degree.
#include "ordering.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <mutex>
#include <thread>
#include <cstring>
#include <queue>
#include <utility>

namespace hsg {
namespace {

struct Rng {
  std::uint64_t s;
  explicit Rng(std::uint64_t seed) : s(seed ^ 0x9E3779B97F4A7C15ull) {}
  std::uint64_t next() {
    std::uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  std::uint32_t below(std::uint32_t n) { return n ? static_cast<std::uint32_t>(next() % n) : 0; }
};

struct WGraph {
  int n = 0;
  std::vector<std::int64_t> xadj;
  std::vector<std::int32_t> adj;
  std::vector<std::int32_t> ew;
  std::vector<std::int32_t> vw;
  std::int64_t total = 0;
};

void shuffled(int n, Rng& rng, std::vector<int>& p) {
  p.resize(n);
  for (int i = 0; i < n; ++i) p[i] = i;
  for (int i = n - 1; i > 0; --i) std::swap(p[i], p[rng.below(i + 1)]);
}

// Heavy-edge matching contraction. cmap: fine -> coarse.
WGraph coarsen(const WGraph& g, std::vector<std::int32_t>& cmap, Rng& rng) {
  const int n = g.n;
  std::vector<int> match(n, -1), order;
  shuffled(n, rng, order);
  for (int v : order) {
    if (match[v] != -1) continue;
    int best = -1, bw = -1;
    for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p) {
      const int u = g.adj[p];
      if (match[u] != -1 || u == v) continue;
      if (g.ew[p] > bw || (g.ew[p] == bw && g.vw[u] < g.vw[best])) { bw = g.ew[p]; best = u; }
    }
    if (best < 0) match[v] = v;
    else { match[v] = best; match[best] = v; }
  }
  cmap.assign(n, -1);
  int cn = 0;
  std::vector<int> rep;
  rep.reserve(n);
  for (int v = 0; v < n; ++v) {
    if (cmap[v] != -1) continue;
    cmap[v] = cn;
    if (match[v] != v) cmap[match[v]] = cn;
    rep.push_back(v);
    ++cn;
  }
  WGraph c;
  c.n = cn;
  c.xadj.assign(cn + 1, 0);
  c.vw.assign(cn, 0);
  c.adj.reserve(g.adj.size());
  c.ew.reserve(g.adj.size());
  std::vector<int> slot(cn, -1);
  for (int cv = 0; cv < cn; ++cv) {
    const int a = rep[cv], b = match[a];
    const std::int64_t start = static_cast<std::int64_t>(c.adj.size());
    for (int t = 0; t < 2; ++t) {
      const int v = t == 0 ? a : b;
      if (t == 1 && b == a) break;
      c.vw[cv] += g.vw[v];
      for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p) {
        const int cu = cmap[g.adj[p]];
        if (cu == cv) continue;
        if (slot[cu] < 0) {
          slot[cu] = static_cast<int>(c.adj.size());
          c.adj.push_back(cu);
          c.ew.push_back(g.ew[p]);
        } else {
          c.ew[slot[cu]] += g.ew[p];
        }
      }
    }
    for (std::int64_t p = start; p < static_cast<std::int64_t>(c.adj.size()); ++p) slot[c.adj[p]] = -1;
    c.xadj[cv + 1] = static_cast<std::int64_t>(c.adj.size());
  }
  c.total = g.total;
  return c;
}

std::int64_t cut_of(const WGraph& g, const std::vector<std::int8_t>& part) {
  std::int64_t cut = 0;
  for (int v = 0; v < g.n; ++v)
    for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p)
      if (part[v] != part[g.adj[p]]) cut += g.ew[p];
  return cut / 2;
}

// Two-way FM refinement of an edge bisection under a weight bound per side.
void fm_refine(const WGraph& g, std::vector<std::int8_t>& part, std::int64_t maxw, int passes) {
  const int n = g.n;
  std::vector<std::int64_t> ed(n), id(n);
  std::vector<char> locked(n);
  std::int64_t pw[2] = {0, 0};
  for (int v = 0; v < n; ++v) pw[part[v]] += g.vw[v];
  for (int pass = 0; pass < passes; ++pass) {
    std::int64_t cut = 0;
    for (int v = 0; v < n; ++v) {
      ed[v] = id[v] = 0;
      for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p)
        (part[g.adj[p]] == part[v] ? id[v] : ed[v]) += g.ew[p];
      cut += ed[v];
    }
    cut /= 2;
    std::fill(locked.begin(), locked.end(), 0);
    std::priority_queue<std::pair<std::int64_t, int>> pq;
    for (int v = 0; v < n; ++v)
      if (ed[v] > 0) pq.push({ed[v] - id[v], v});
    std::vector<int> moves;
    std::int64_t best = cut, bestimb = std::llabs(pw[0] - pw[1]);
    std::size_t bestpos = 0;
    const std::size_t limit = static_cast<std::size_t>(std::max(25, std::min(n / 20, 400)));
    // an initially unbalanced side may only shrink until it fits
    while (!pq.empty() && moves.size() - bestpos < limit) {
      auto [gain, v] = pq.top();
      pq.pop();
      if (locked[v] || gain != ed[v] - id[v]) continue;
      const int from = part[v], to = 1 - from;
      if (pw[to] + g.vw[v] > maxw && pw[from] <= maxw) continue;
      part[v] = static_cast<std::int8_t>(to);
      pw[from] -= g.vw[v];
      pw[to] += g.vw[v];
      cut -= gain;
      locked[v] = 1;
      std::swap(ed[v], id[v]);
      moves.push_back(v);
      for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p) {
        const int u = g.adj[p];
        if (part[u] == to) { id[u] += g.ew[p]; ed[u] -= g.ew[p]; }
        else { ed[u] += g.ew[p]; id[u] -= g.ew[p]; }
        if (!locked[u]) pq.push({ed[u] - id[u], u});
      }
      const std::int64_t imb = std::llabs(pw[0] - pw[1]);
      const bool fits = pw[0] <= maxw && pw[1] <= maxw;
      if (fits && (cut < best || (cut == best && imb < bestimb))) {
        best = cut;
        bestimb = imb;
        bestpos = moves.size();
      }
    }
    for (std::size_t i = moves.size(); i > bestpos; --i) {
      const int v = moves[i - 1];
      const int from = part[v], to = 1 - from;
      part[v] = static_cast<std::int8_t>(to);
      pw[from] -= g.vw[v];
      pw[to] += g.vw[v];
    }
    if (bestpos == 0) break;
  }
}

// Greedy graph growing from random seeds on the coarsest graph; best refined cut wins.
std::vector<std::int8_t> initial_bisection(const WGraph& g, std::int64_t maxw, int tries, int passes, Rng& rng) {
  const int n = g.n;
  std::vector<std::int8_t> best;
  std::int64_t bestcut = -1;
  for (int t = 0; t < tries; ++t) {
    std::vector<std::int8_t> part(n, 1);
    std::vector<std::int64_t> conn(n, 0);  // edge weight into part 0
    std::int64_t w0 = 0;
    const std::int64_t half = g.total / 2;
    std::priority_queue<std::pair<std::int64_t, int>> pq;
    int seed = static_cast<int>(rng.below(n));
    std::vector<char> inq(n, 0);
    while (w0 < half) {
      int v = -1;
      while (!pq.empty()) {
        auto [gain, u] = pq.top();
        pq.pop();
        if (part[u] == 1) {
          std::int64_t tot = 0;
          for (std::int64_t p = g.xadj[u]; p < g.xadj[u + 1]; ++p) tot += g.ew[p];
          if (gain != 2 * conn[u] - tot) continue;
          v = u;
          break;
        }
      }
      if (v < 0) {  // disconnected remainder: restart growing elsewhere
        if (part[seed] == 1) v = seed;
        else {
          for (int u = 0; u < n; ++u)
            if (part[u] == 1) { v = u; break; }
        }
        if (v < 0) break;
      }
      part[v] = 0;
      w0 += g.vw[v];
      for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p) {
        const int u = g.adj[p];
        conn[u] += g.ew[p];
        if (part[u] == 1) {
          std::int64_t tot = 0;
          for (std::int64_t q = g.xadj[u]; q < g.xadj[u + 1]; ++q) tot += g.ew[q];
          pq.push({2 * conn[u] - tot, u});
        }
      }
    }
    fm_refine(g, part, maxw, passes);
    const std::int64_t cut = cut_of(g, part);
    std::int64_t pw0 = 0;
    for (int v = 0; v < n; ++v) if (part[v] == 0) pw0 += g.vw[v];
    const bool ok = pw0 <= maxw && g.total - pw0 <= maxw && pw0 > 0 && pw0 < g.total;
    if (ok && (bestcut < 0 || cut < bestcut)) { bestcut = cut; best = part; }
    if (!ok && bestcut < 0 && best.empty()) best = part;
  }
  return best;
}

// Hopcroft-Karp matching between boundary sets (left = side 0, right = side 1) over cut edges,
// then Konig's theorem: minimum vertex cover = (L \ Z) u (R n Z), Z = alternating-reachable from
// unmatched left vertices.
void min_cover_separator(const WGraph& g, std::vector<std::int8_t>& where) {
  const int n = g.n;
  std::vector<int> lidx, ridx;
  std::vector<int> lpos(n, -1), rpos(n, -1);
  for (int v = 0; v < n; ++v) {
    bool b = false;
    for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1] && !b; ++p) b = where[g.adj[p]] != where[v];
    if (!b) continue;
    if (where[v] == 0) { lpos[v] = static_cast<int>(lidx.size()); lidx.push_back(v); }
    else { rpos[v] = static_cast<int>(ridx.size()); ridx.push_back(v); }
  }
  const int L = static_cast<int>(lidx.size()), R = static_cast<int>(ridx.size());
  std::vector<int> ml(L, -1), mr(R, -1), dist(L);
  auto bfs = [&]() {
    std::vector<int> q;
    bool found = false;
    for (int l = 0; l < L; ++l) {
      if (ml[l] < 0) { dist[l] = 0; q.push_back(l); } else dist[l] = -1;
    }
    for (std::size_t h = 0; h < q.size(); ++h) {
      const int l = q[h];
      const int v = lidx[l];
      for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p) {
        const int r = rpos[g.adj[p]];
        if (r < 0) continue;
        const int l2 = mr[r];
        if (l2 < 0) found = true;
        else if (dist[l2] < 0) { dist[l2] = dist[l] + 1; q.push_back(l2); }
      }
    }
    return found;
  };
  std::vector<std::int64_t> it(L);
  // iterative DFS along layered graph
  auto dfs = [&](int root) {
    std::vector<int> stack{root};
    std::vector<int> path_r;
    while (!stack.empty()) {
      const int l = stack.back();
      const int v = lidx[l];
      bool advanced = false;
      for (; it[l] < g.xadj[v + 1]; ++it[l]) {
        const int r = rpos[g.adj[it[l]]];
        if (r < 0) continue;
        const int l2 = mr[r];
        if (l2 < 0) {
          // augment along the stack
          path_r.push_back(r);
          for (std::size_t k = stack.size(); k-- > 0;) {
            const int ll = stack[k];
            const int rr = path_r[k];
            const int prev = ml[ll];
            ml[ll] = rr;
            mr[rr] = ll;
            (void)prev;
          }
          return true;
        }
        if (dist[l2] == dist[l] + 1) {
          path_r.push_back(r);
          ++it[l];
          stack.push_back(l2);
          advanced = true;
          break;
        }
      }
      if (!advanced) {
        dist[l] = -1;
        stack.pop_back();
        if (!path_r.empty()) path_r.pop_back();
      }
    }
    return false;
  };
  while (bfs()) {
    for (int l = 0; l < L; ++l) it[l] = g.xadj[lidx[l]];
    for (int l = 0; l < L; ++l)
      if (ml[l] < 0) dfs(l);
  }
  // Konig: alternating BFS from unmatched left vertices
  std::vector<char> zl(L, 0), zr(R, 0);
  std::vector<int> q;
  for (int l = 0; l < L; ++l)
    if (ml[l] < 0) { zl[l] = 1; q.push_back(l); }
  for (std::size_t h = 0; h < q.size(); ++h) {
    const int l = q[h];
    const int v = lidx[l];
    for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p) {
      const int r = rpos[g.adj[p]];
      if (r < 0 || zr[r] || mr[r] == l) continue;
      zr[r] = 1;
      const int l2 = mr[r];
      if (l2 >= 0 && !zl[l2]) { zl[l2] = 1; q.push_back(l2); }
    }
  }
  for (int l = 0; l < L; ++l) if (!zl[l]) where[lidx[l]] = 2;
  for (int r = 0; r < R; ++r) if (zr[r]) where[ridx[r]] = 2;
}

// Node-FM refinement of a vertex separator (where: 0, 1 sides, 2 separator).
void node_refine(const WGraph& g, std::vector<std::int8_t>& where, std::int64_t maxside, int passes) {
  const int n = g.n;
  std::int64_t pw[3] = {0, 0, 0};
  for (int v = 0; v < n; ++v) pw[where[v]] += g.vw[v];
  std::vector<char> locked(n);
  auto gain = [&](int v, int to) {
    std::int64_t s = g.vw[v];
    for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p)
      if (where[g.adj[p]] == 1 - to) s -= g.vw[g.adj[p]];
    return s;
  };
  struct Move { int v; int to; std::vector<int> pulled; };
  for (int pass = 0; pass < passes; ++pass) {
    std::fill(locked.begin(), locked.end(), 0);
    std::priority_queue<std::tuple<std::int64_t, int, int>> pq;
    for (int v = 0; v < n; ++v)
      if (where[v] == 2) { pq.push({gain(v, 0), v, 0}); pq.push({gain(v, 1), v, 1}); }
    std::vector<Move> moves;
    std::int64_t best = pw[2], bestimb = std::llabs(pw[0] - pw[1]);
    std::size_t bestpos = 0;
    const std::size_t limit = static_cast<std::size_t>(std::max(25, std::min(n / 30, 300)));
    while (!pq.empty() && moves.size() - bestpos < limit) {
      auto [gn, v, to] = pq.top();
      pq.pop();
      if (locked[v] || where[v] != 2) continue;
      const std::int64_t cur = gain(v, to);
      if (cur != gn) { pq.push({cur, v, to}); continue; }
      if (pw[to] + g.vw[v] > maxside) continue;
      Move mv{v, to, {}};
      where[v] = static_cast<std::int8_t>(to);
      pw[to] += g.vw[v];
      pw[2] -= g.vw[v];
      locked[v] = 1;
      for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p) {
        const int u = g.adj[p];
        if (where[u] == 1 - to) {
          where[u] = 2;
          pw[1 - to] -= g.vw[u];
          pw[2] += g.vw[u];
          mv.pulled.push_back(u);
        }
      }
      for (int u : mv.pulled) {
        if (!locked[u]) { pq.push({gain(u, 0), u, 0}); pq.push({gain(u, 1), u, 1}); }
        for (std::int64_t p = g.xadj[u]; p < g.xadj[u + 1]; ++p) {
          const int w = g.adj[p];
          if (where[w] == 2 && !locked[w]) { pq.push({gain(w, 0), w, 0}); pq.push({gain(w, 1), w, 1}); }
        }
      }
      moves.push_back(std::move(mv));
      const std::int64_t imb = std::llabs(pw[0] - pw[1]);
      if (pw[2] < best || (pw[2] == best && imb < bestimb)) {
        best = pw[2];
        bestimb = imb;
        bestpos = moves.size();
      }
    }
    for (std::size_t i = moves.size(); i > bestpos; --i) {
      const Move& mv = moves[i - 1];
      for (int u : mv.pulled) { where[u] = static_cast<std::int8_t>(1 - mv.to); pw[1 - mv.to] += g.vw[u]; pw[2] -= g.vw[u]; }
      where[mv.v] = 2;
      pw[mv.to] -= g.vw[mv.v];
      pw[2] += g.vw[mv.v];
    }
    if (bestpos == 0) break;
  }
}

// Vertex separator of a connected graph: where[v] in {0, 1, 2 (separator)}.
std::vector<std::int8_t> separator(const WGraph& g0, const OrderingOptions& opt, Rng& rng) {
  std::vector<WGraph> levels;
  std::vector<std::vector<std::int32_t>> maps;
  levels.push_back(g0);
  while (levels.back().n > opt.coarsen_to) {
    std::vector<std::int32_t> cmap;
    WGraph c = coarsen(levels.back(), cmap, rng);
    if (c.n > 0.92 * levels.back().n) break;
    maps.push_back(std::move(cmap));
    levels.push_back(std::move(c));
  }
  const std::int64_t maxw = static_cast<std::int64_t>(opt.imbalance * g0.total / 2.0) + 1;
  std::vector<std::int8_t> part = initial_bisection(levels.back(), maxw, opt.init_tries, opt.refine_passes, rng);
  for (std::size_t lv = levels.size() - 1; lv > 0; --lv) {
    const auto& cmap = maps[lv - 1];
    const WGraph& fine = levels[lv - 1];
    std::vector<std::int8_t> fp(fine.n);
    for (int v = 0; v < fine.n; ++v) fp[v] = part[cmap[v]];
    part.swap(fp);
    fm_refine(fine, part, maxw, opt.refine_passes);
  }
  std::vector<std::int8_t> where = part;
  min_cover_separator(g0, where);
  node_refine(g0, where, maxw, opt.refine_passes);
  return where;
}

// Exact minimum degree on a small graph with explicit fill (bitset rows).
void min_degree_leaf(const std::vector<int>& verts, const std::vector<int>& loc, const Adjacency& g,
                     std::vector<std::int32_t>& out) {
  const int L = static_cast<int>(verts.size());
  const int W = (L + 63) / 64;
  std::vector<std::uint64_t> bits(static_cast<std::size_t>(L) * W, 0);
  auto row = [&](int i) { return bits.data() + static_cast<std::size_t>(i) * W; };
  for (int i = 0; i < L; ++i) {
    const int v = verts[i];
    for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p) {
      const int j = loc[g.adj[p]];
      if (j >= 0 && j != i) row(i)[j >> 6] |= 1ull << (j & 63);
    }
  }
  std::vector<char> gone(L, 0);
  std::vector<int> deg(L);
  for (int i = 0; i < L; ++i) {
    int d = 0;
    for (int w = 0; w < W; ++w) d += __builtin_popcountll(row(i)[w]);
    deg[i] = d;
  }
  for (int step = 0; step < L; ++step) {
    int best = -1;
    for (int i = 0; i < L; ++i)
      if (!gone[i] && (best < 0 || deg[i] < deg[best])) best = i;
    out.push_back(verts[best]);
    gone[best] = 1;
    std::uint64_t* rb = row(best);
    for (int i = 0; i < L; ++i) {
      if (!(rb[i >> 6] >> (i & 63) & 1ull)) continue;
      std::uint64_t* ri = row(i);
      ri[best >> 6] &= ~(1ull << (best & 63));
      for (int w = 0; w < W; ++w) ri[w] |= rb[w];
      ri[i >> 6] &= ~(1ull << (i & 63));
      int d = 0;
      for (int w = 0; w < W; ++w) d += __builtin_popcountll(ri[w]);
      deg[i] = d;
    }
    for (int w = 0; w < W; ++w) rb[w] = 0;
  }
}

}  // namespace

Adjacency adjacency_from_upper(std::int64_t n, const std::int64_t* rowptr, const std::int32_t* col) {
  Adjacency g;
  g.n = n;
  std::vector<std::int64_t> cnt(n + 1, 0);
  for (std::int64_t i = 0; i < n; ++i)
    for (std::int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p)
      if (col[p] != i) { cnt[i + 1]++; cnt[col[p] + 1]++; }
  for (std::int64_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
  g.xadj = cnt;
  g.adj.resize(cnt[n]);
  for (std::int64_t i = 0; i < n; ++i)
    for (std::int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p)
      if (col[p] != i) { g.adj[cnt[i]++] = col[p]; g.adj[cnt[col[p]]++] = static_cast<std::int32_t>(i); }
  // sort and unique each row (duplicates can come from duplicate CSR entries)
  std::vector<std::int64_t> nx(n + 1, 0);
  std::int64_t w = 0;
  for (std::int64_t i = 0; i < n; ++i) {
    auto b = g.adj.begin() + g.xadj[i], e = g.adj.begin() + g.xadj[i + 1];
    std::sort(b, e);
    auto u = std::unique(b, e);
    for (auto q = b; q != u; ++q) g.adj[w++] = *q;
    nx[i + 1] = w;
  }
  g.adj.resize(w);
  g.xadj = nx;
  return g;
}

namespace {

struct NdTask {
  std::vector<int> verts;
  std::int64_t lo = 0;
};

// Per-task random stream: a function of the seed, the task's first position and its size, so the
// order does not depend on how the tasks are scheduled over threads.
std::uint64_t task_seed(std::uint64_t seed, std::int64_t lo, std::size_t m) {
  Rng r(seed ^ (static_cast<std::uint64_t>(lo) * 0xD1B54A32D192ED03ull) ^ (static_cast<std::uint64_t>(m) << 40));
  return r.next();
}

struct NdShared {
  const Adjacency& g;
  const OrderingOptions& opt;
  std::vector<std::int32_t>& order;
  std::mutex mu;
  std::condition_variable cv;
  std::vector<NdTask> queue;
  int active = 0;
  std::atomic<std::int64_t> nsep{0}, nleaf{0}, topsep{-1};
  NdShared(const Adjacency& gr, const OrderingOptions& o, std::vector<std::int32_t>& ord) : g(gr), opt(o), order(ord) {}
};

// Subproblems with more vertices than this go to the shared queue; smaller ones stay with the
// thread that split them.
constexpr std::size_t kNdParallelMin = 3000;

// Orders one subproblem and, depth first, the small subproblems it splits into.
void nd_process(NdShared& S, NdTask root, std::vector<int>& loc, std::vector<std::int32_t>& leaf_out) {
  const Adjacency& g = S.g;
  const OrderingOptions& opt = S.opt;
  std::vector<NdTask> stack;
  stack.push_back(std::move(root));
  auto hand_off = [&](NdTask&& t) {
    if (t.verts.size() > kNdParallelMin) {
      std::lock_guard<std::mutex> lk(S.mu);
      S.queue.push_back(std::move(t));
      S.cv.notify_one();
    } else {
      stack.push_back(std::move(t));
    }
  };
  while (!stack.empty()) {
    NdTask t = std::move(stack.back());
    stack.pop_back();
    const int m = static_cast<int>(t.verts.size());
    if (m == 0) continue;
    for (int i = 0; i < m; ++i) loc[t.verts[i]] = i;
    if (m <= opt.leaf_size) {
      leaf_out.clear();
      min_degree_leaf(t.verts, loc, g, leaf_out);
      for (int i = 0; i < m; ++i) S.order[t.lo + i] = leaf_out[i];
      for (int v : t.verts) loc[v] = -1;
      S.nleaf++;
      continue;
    }
    // local graph
    WGraph w;
    w.n = m;
    w.xadj.assign(m + 1, 0);
    for (int i = 0; i < m; ++i) {
      const int v = t.verts[i];
      for (std::int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p)
        if (loc[g.adj[p]] >= 0) { w.adj.push_back(loc[g.adj[p]]); }
      w.xadj[i + 1] = static_cast<std::int64_t>(w.adj.size());
    }
    w.ew.assign(w.adj.size(), 1);
    w.vw.assign(m, 1);
    w.total = m;
    // connected components
    std::vector<int> comp(m, -1);
    int nc = 0;
    std::vector<int> q;
    for (int s0 = 0; s0 < m; ++s0) {
      if (comp[s0] >= 0) continue;
      q.assign(1, s0);
      comp[s0] = nc;
      for (std::size_t h = 0; h < q.size(); ++h)
        for (std::int64_t p = w.xadj[q[h]]; p < w.xadj[q[h] + 1]; ++p)
          if (comp[w.adj[p]] < 0) { comp[w.adj[p]] = nc; q.push_back(w.adj[p]); }
      ++nc;
    }
    if (nc > 1) {
      std::vector<NdTask> parts(nc);
      for (int i = 0; i < m; ++i) parts[comp[i]].verts.push_back(t.verts[i]);
      std::int64_t lo = t.lo;
      for (auto& pt : parts) { pt.lo = lo; lo += static_cast<std::int64_t>(pt.verts.size()); }
      for (int v : t.verts) loc[v] = -1;
      for (auto it = parts.rbegin(); it != parts.rend(); ++it) hand_off(std::move(*it));
      continue;
    }
    Rng rng(task_seed(opt.seed, t.lo, t.verts.size()));
    std::vector<std::int8_t> where = separator(w, opt, rng);
    NdTask a, b;
    std::vector<int> sep;
    for (int i = 0; i < m; ++i) {
      if (where[i] == 0) a.verts.push_back(t.verts[i]);
      else if (where[i] == 1) b.verts.push_back(t.verts[i]);
      else sep.push_back(t.verts[i]);
    }
    for (int v : t.verts) loc[v] = -1;
    if (a.verts.empty() || b.verts.empty()) {
      // degenerate split: order this subgraph by minimum degree (still valid)
      for (int i = 0; i < m; ++i) loc[t.verts[i]] = i;
      leaf_out.clear();
      min_degree_leaf(t.verts, loc, g, leaf_out);
      for (int i = 0; i < m; ++i) S.order[t.lo + i] = leaf_out[i];
      for (int v : t.verts) loc[v] = -1;
      S.nleaf++;
      continue;
    }
    S.nsep++;
    if (t.lo == 0 && static_cast<std::int64_t>(t.verts.size()) == g.n) S.topsep = static_cast<std::int64_t>(sep.size());
    a.lo = t.lo;
    b.lo = t.lo + static_cast<std::int64_t>(a.verts.size());
    const std::int64_t slo = b.lo + static_cast<std::int64_t>(b.verts.size());
    for (std::size_t i = 0; i < sep.size(); ++i) S.order[slo + static_cast<std::int64_t>(i)] = sep[i];
    hand_off(std::move(b));
    hand_off(std::move(a));
  }
}

}  // namespace

std::vector<std::int32_t> nested_dissection(const Adjacency& g, const OrderingOptions& opt, OrderingStats* stats) {
  const auto t0 = std::chrono::steady_clock::now();
  const std::int64_t n = g.n;
  std::vector<std::int32_t> order(n, -1);
  NdShared S(g, opt, order);
  {
    NdTask t;
    t.verts.resize(n);
    for (std::int64_t i = 0; i < n; ++i) t.verts[i] = static_cast<int>(i);
    S.queue.push_back(std::move(t));
  }
  int nthreads = opt.threads;
  if (nthreads <= 0) {
    const char* env = std::getenv("HSOLVE_B200_ORDERING_THREADS");
    nthreads = env ? std::atoi(env) : 0;
  }
  if (nthreads <= 0) nthreads = static_cast<int>(std::thread::hardware_concurrency());
  nthreads = std::max(1, std::min(nthreads, 32));
  if (n < 2 * static_cast<std::int64_t>(kNdParallelMin)) nthreads = 1;
  auto worker = [&]() {
    std::vector<int> loc(n, -1);
    std::vector<std::int32_t> leaf_out;
    for (;;) {
      NdTask t;
      {
        std::unique_lock<std::mutex> lk(S.mu);
        S.cv.wait(lk, [&] { return !S.queue.empty() || S.active == 0; });
        if (S.queue.empty()) return;  // nothing queued and nobody left to queue more
        t = std::move(S.queue.back());
        S.queue.pop_back();
        ++S.active;
      }
      nd_process(S, std::move(t), loc, leaf_out);
      {
        std::lock_guard<std::mutex> lk(S.mu);
        --S.active;
        if (S.active == 0 && S.queue.empty()) S.cv.notify_all();
      }
    }
  };
  std::vector<std::thread> pool;
  for (int i = 1; i < nthreads; ++i) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  if (stats) {
    stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    stats->separators = S.nsep;
    stats->leaves = S.nleaf;
    stats->top_separator = S.topsep < 0 ? 0 : S.topsep.load();
  }
  return order;
}

}  // namespace hsg
