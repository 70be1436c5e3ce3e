// Top-level shift-invert driver: the device-resident equivalent of hs::solve for HEP / GHEP / GHIEP
// (hsolve include/hsolve/solver.hpp:545-547; src/driver/solver.cpp:307-520, definite.cpp,
// indefinite.cpp).
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "hsg_solve.h"

namespace hsg {

struct CsrHost {
  std::int64_t n = 0;
  std::vector<std::int64_t> rp;
  std::vector<std::int32_t> ci;
  std::vector<double> v;
};

struct SolveOutput {
  std::vector<double> eigenvalues;
  std::vector<double> vectors;  // n x m, column-major
  // GHIEP: genuinely complex pairs, values and n x mc vectors as interleaved (re, im) doubles
  std::vector<double> complex_eigenvalues;
  std::vector<double> complex_vectors;
  std::int64_t n = 0;
  std::string report_json;
};

// A pencil resident on the GPU with its analysis (ordering, symbolic factorization) and norm bounds
// computed once; solve() serves any number of targets on it (symbolic reuse across shifts).
class Session {
 public:
  Session(const CsrHost& a, const CsrHost* b, int device, std::uint64_t seed);
  ~Session();
  Session(const Session&) = delete;
  Session& operator=(const Session&) = delete;
  SolveOutput solve(const hsg_solve_config_t& cfg, bool include_setup = false);
  // randomized exclusion certificate on the factorization at opt.sigma (x: host, n x m, ld ldx)
  hsg_exclusion_result_t exclusion_check(const double* x, std::int64_t m, std::int64_t ldx,
                                         const hsg_exclusion_options_t& opt);
  std::int64_t order() const;
  hsg_estimate_t estimate() const;

 private:
  // one attempt at the requested precision; `fallback` (non-empty) records why an earlier FP32
  // attempt was abandoned
  SolveOutput solve_once(const hsg_solve_config_t& cfg, bool include_setup, const std::string& fallback);
  struct Impl;
  std::unique_ptr<Impl> d_;
};

SolveOutput solve_pencil(const CsrHost& a, const CsrHost* b, const hsg_solve_config_t& cfg);

}  // namespace hsg
