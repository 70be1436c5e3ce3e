// Fill-reducing pivot order by multilevel nested dissection (host C++).
//
// Replaces the reference's hs::compute_ordering (include/hsolve/factor.hpp:598-633,
// src/factor/ordering.cpp:315), which is kept on the CPU there too: multilevel vertex separators
// (heavy-edge matching, greedy growing, FM refinement), applied recursively, leaves ordered by
// minimum degree. Deterministic: a function of the pattern and the seed only, whatever the number
// of threads that order the independent subproblems.
#pragma once

#include <cstdint>
#include <vector>

namespace hsg {

struct OrderingOptions {
  int leaf_size = 120;        // subgraphs of at most this many vertices: minimum degree
  double imbalance = 1.2;     // each side of a separator weighs at most imbalance * |V| / 2
  int coarsen_to = 100;       // coarsest graph size of the multilevel bisection
  int init_tries = 7;         // greedy-growing attempts on the coarsest graph
  int refine_passes = 8;      // FM passes per level
  std::uint64_t seed = 2026;
  int threads = 0;             // host threads (0: $HSOLVE_B200_ORDERING_THREADS, else all); the order
                               // does not depend on it
};

struct OrderingStats {
  double seconds = 0.0;
  std::int64_t separators = 0;
  std::int64_t leaves = 0;
  std::int64_t top_separator = 0;
};

// Symmetric adjacency (no self loops) in CSR form.
struct Adjacency {
  std::int64_t n = 0;
  std::vector<std::int64_t> xadj;
  std::vector<std::int32_t> adj;
};

// Adjacency of the symmetric matrix whose upper triangle (row <= col) is given as CSR.
Adjacency adjacency_from_upper(std::int64_t n, const std::int64_t* rowptr, const std::int32_t* col);

// Pivot order: order[new] = old (new -> old).
std::vector<std::int32_t> nested_dissection(const Adjacency& g, const OrderingOptions& opt,
                                            OrderingStats* stats = nullptr);

}  // namespace hsg
