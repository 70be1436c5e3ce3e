// Symbolic analysis of the multifrontal LDL^T (host C++).
//
// Replaces the symbolic phase that hsolve delegates to MUMPS JOB=1 (SparseFactorization::analyze,
// include/hsolve/factor.hpp:352-358; src/factor/mumps_factorization.cpp:189-283): from a pivot
// order, the elimination tree, its postorder, column counts, fundamental supernodes with relaxed
// amalgamation, the row structure of every front, the maps that scatter original entries and
// children's contribution blocks into fronts, the height levels that batch fronts on the GPU, and
// a memory plan for contribution blocks. Delayed pivots re-plan the partition (move_delayed).
#pragma once

#include <cstdint>
#include <vector>

#include "ordering.hpp"

namespace hsg {

struct SymbolicOptions {
  OrderingOptions ordering;
  bool amalgamate = true;
  int relax_small = 4;          // always merge up to this many columns
  int relax_mid = 16;           // ... up to this many with < 80% explicit zeros
  int relax_big = 48;           // ... up to this many with < 10% explicit zeros, then < 5%
};

struct Symbolic {
  std::int64_t n = 0;
  std::int64_t nnz_upper = 0;            // entries of the analysed upper pattern
  std::vector<std::int32_t> perm;        // pivot position -> original index
  std::vector<std::int32_t> iperm;       // original index -> pivot position
  std::int32_t ns = 0;                   // supernodes (fronts), postordered
  std::vector<std::int32_t> first;       // ns + 1: columns [first[s], first[s+1])
  std::vector<std::int32_t> parent;      // ns: parent supernode, -1 for roots
  std::vector<std::int64_t> rowptr;      // ns + 1
  std::vector<std::int32_t> rows;        // sorted pivot positions of each front's rows; the
                                         // first k = first[s+1]-first[s] are its own columns
  std::vector<std::int32_t> child_ptr;   // ns + 1
  std::vector<std::int32_t> children;    // children of each supernode, ascending
  // storage
  std::vector<std::int64_t> panel_off;   // ns + 1: offset of the m x k panel (ld m)
  std::vector<std::int64_t> cb_off;      // ns: offset of the (m-k)^2 contribution block (ld m-k)
  std::int64_t cb_arena = 0;             // doubles needed by the contribution-block plan
  std::vector<std::int64_t> rmap_off;    // ns + 1: positions of each CB row in the parent's rows
  std::vector<std::int32_t> rmap;
  std::vector<std::int64_t> dest;        // per entry of the upper pattern: offset into the panels
  // schedule
  std::int32_t nlevels = 0;
  std::vector<std::int32_t> height;      // ns
  std::vector<std::int32_t> level_ptr;   // nlevels + 1
  std::vector<std::int32_t> level_sn;    // supernodes by level
  // statistics
  double flops = 0.0;                    // elimination flops, MUMPS RINFOG(1) convention
  std::int64_t nnz_l = 0;                // entries of L incl. D (lower trapezoids)
  std::int64_t factor_entries = 0;       // panel storage, sum of m*k
  std::int32_t max_front = 0;
  std::int64_t delayed_moves = 0;        // columns moved to a parent by move_delayed
  double ordering_seconds = 0.0;
  double symbolic_seconds = 0.0;
  OrderingStats ordering_stats;

  std::int32_t k_of(std::int32_t s) const { return first[s + 1] - first[s]; }
  std::int32_t m_of(std::int32_t s) const { return static_cast<std::int32_t>(rowptr[s + 1] - rowptr[s]); }
};

// Full analysis of the symmetric pattern given by its upper triangle (row <= col, CSR).
// order: pivot order (position -> original index) or nullptr for nested dissection.
Symbolic analyze_pattern(std::int64_t n, const std::int64_t* rowptr, const std::int32_t* col,
                         const std::int32_t* order, const SymbolicOptions& opt);

// Move the given columns (pivot positions) out of their supernodes into the parents' fully-summed
// blocks (what a delayed pivot does in a multifrontal factorization), renumber and rebuild every
// derived array. Columns of roots cannot move and are ignored. Returns the number moved.
std::int64_t move_delayed(Symbolic& sym, const std::int64_t* rowptr, const std::int32_t* col,
                          const std::vector<std::int32_t>& delayed);

}  // namespace hsg
