// C ABI of the whole eigensolve (include/hsg_solve.h).
#include <cmath>
#include <memory>
#include <string>

#include "common.hpp"
#include "driver.hpp"
#include "eigen.hpp"
#include "hsg_solve.h"

struct hsg_solution {
  hsg::SolveOutput out;
};

struct hsg_session {
  std::unique_ptr<hsg::Session> impl;
};

using namespace hsg;

namespace {
CsrHost copy_csr(int64_t n, const int64_t* rp, const int32_t* ci, const double* v, const char* name) {
  HSG_REQUIRE(rp && ci && v, HSG_INVALID_INPUT, name << ": null CSR array");
  CsrHost m;
  m.n = n;
  m.rp.assign(rp, rp + n + 1);
  HSG_REQUIRE(m.rp[0] == 0, HSG_INVALID_INPUT, name << ": rowptr[0] != 0");
  for (int64_t i = 0; i < n; ++i) HSG_REQUIRE(m.rp[i + 1] >= m.rp[i], HSG_INVALID_INPUT, name << ": rowptr not monotone");
  const int64_t nnz = m.rp[n];
  m.ci.assign(ci, ci + nnz);
  m.v.assign(v, v + nnz);
  for (int64_t p = 0; p < nnz; ++p) {
    HSG_REQUIRE(m.ci[p] >= 0 && m.ci[p] < n, HSG_INVALID_INPUT, name << ": column index out of range");
    HSG_REQUIRE(std::isfinite(m.v[p]), HSG_INVALID_INPUT, name << ": non-finite entry");
  }
  return m;
}
}  // namespace

extern "C" {

void hsg_default_solve_config(hsg_solve_config_t* c) {
  if (!c) return;
  c->mode = 0;
  c->sigma = 0.0;
  c->k = 6;
  c->lower = 0.0;
  c->upper = 0.0;
  c->problem = 0;
  c->tol = 1e-10;
  c->inner_tol_factor = 0.1;
  c->ncv = 0;
  c->block_size = 0;
  c->slice_size = 0;
  c->max_restarts = 1000;
  c->seed = 2026;
  c->certificate = 0;
  c->max_shift_retries = 5;
  c->factor_precision = 0;
  c->device = 0;
  c->verbose = 0;
  c->batch_shifts = 1;
  c->complex_tol = 1e-8;
  c->zero_filter_tol = -1.0;
}

int hsg_eigsolve(int64_t n, const int64_t* a_rowptr, const int32_t* a_col, const double* a_val,
                 const int64_t* b_rowptr, const int32_t* b_col, const double* b_val, const hsg_solve_config_t* cfg,
                 hsg_solution** out) {
  return guarded([&] {
    HSG_REQUIRE(out, HSG_INVALID_INPUT, "hsg_eigsolve: null output");
    *out = nullptr;
    HSG_REQUIRE(n > 0, HSG_INVALID_INPUT, "hsg_eigsolve: n must be positive");
    hsg_solve_config_t c;
    hsg_default_solve_config(&c);
    if (cfg) c = *cfg;
    CsrHost a = copy_csr(n, a_rowptr, a_col, a_val, "A");
    std::unique_ptr<CsrHost> b;
    if (b_rowptr) b = std::make_unique<CsrHost>(copy_csr(n, b_rowptr, b_col, b_val, "B"));
    auto sol = std::make_unique<hsg_solution>();
    sol->out = solve_pencil(a, b.get(), c);
    *out = sol.release();
  });
}

int hsg_session_create(int64_t n, const int64_t* a_rowptr, const int32_t* a_col, const double* a_val,
                       const int64_t* b_rowptr, const int32_t* b_col, const double* b_val, int32_t device, uint64_t seed,
                       hsg_session** out) {
  return guarded([&] {
    HSG_REQUIRE(out, HSG_INVALID_INPUT, "hsg_session_create: null output");
    *out = nullptr;
    HSG_REQUIRE(n > 0, HSG_INVALID_INPUT, "hsg_session_create: n must be positive");
    CsrHost a = copy_csr(n, a_rowptr, a_col, a_val, "A");
    std::unique_ptr<CsrHost> b;
    if (b_rowptr) b = std::make_unique<CsrHost>(copy_csr(n, b_rowptr, b_col, b_val, "B"));
    auto s = std::make_unique<hsg_session>();
    s->impl = std::make_unique<Session>(a, b.get(), device, seed);
    *out = s.release();
  });
}

int hsg_session_estimate(const hsg_session* s, hsg_estimate_t* out) {
  return guarded([&] {
    HSG_REQUIRE(s && s->impl && out, HSG_INVALID_INPUT, "hsg_session_estimate: null argument");
    *out = s->impl->estimate();
  });
}

int hsg_session_solve(hsg_session* s, const hsg_solve_config_t* cfg, hsg_solution** out) {
  return guarded([&] {
    HSG_REQUIRE(s && s->impl && out, HSG_INVALID_INPUT, "hsg_session_solve: null argument");
    *out = nullptr;
    hsg_solve_config_t c;
    hsg_default_solve_config(&c);
    if (cfg) c = *cfg;
    auto sol = std::make_unique<hsg_solution>();
    sol->out = s->impl->solve(c, false);
    *out = sol.release();
  });
}

void hsg_session_free(hsg_session* s) { delete s; }

void hsg_default_exclusion_options(hsg_exclusion_options_t* opt) {
  if (!opt) return;
  *opt = hsg_exclusion_options_t{};
  opt->delta = 1e-12;
  opt->block_size = 4;
  opt->max_krylov_vectors = 512;
  opt->seed = 2026;
  opt->kappa = 1.0;
  opt->rounding_margin = 1e-6;
}

int hsg_session_exclusion_check(hsg_session* s, const double* x, int64_t m, int64_t ldx,
                                const hsg_exclusion_options_t* opt, hsg_exclusion_result_t* out) {
  return guarded([&] {
    HSG_REQUIRE(s && s->impl && x && opt && out, HSG_INVALID_INPUT, "hsg_session_exclusion_check: null argument");
    *out = s->impl->exclusion_check(x, m, ldx, *opt);
  });
}

double hsg_exclusion_failure_bound(double epsilon, int64_t block_steps, int64_t dimension, int64_t block_size,
                                   double kappa, int32_t complex_scalars) {
  double v = std::nan("");
  const int st = guarded([&] {
    v = hsg::exclusion_failure_bound(epsilon, block_steps, dimension, block_size, kappa, complex_scalars != 0);
  });
  return st == 0 ? v : std::nan("");
}

int64_t hsg_exclusion_block_steps(double epsilon, double delta, int64_t dimension, int64_t block_size, double kappa,
                                  int32_t complex_scalars) {
  int64_t v = -1;
  const int st = guarded([&] {
    v = hsg::exclusion_block_steps(epsilon, delta, dimension, block_size, kappa, complex_scalars != 0);
  });
  return st == 0 ? v : -1;
}

int hsg_solution_sizes(const hsg_solution* s, int64_t* n, int64_t* m) {
  return guarded([&] {
    HSG_REQUIRE(s, HSG_INVALID_INPUT, "null solution");
    if (n) *n = s->out.n;
    if (m) *m = static_cast<int64_t>(s->out.eigenvalues.size());
  });
}

int hsg_solution_copy(const hsg_solution* s, double* eigenvalues, double* eigenvectors) {
  return guarded([&] {
    HSG_REQUIRE(s, HSG_INVALID_INPUT, "null solution");
    if (eigenvalues) std::copy(s->out.eigenvalues.begin(), s->out.eigenvalues.end(), eigenvalues);
    if (eigenvectors) std::copy(s->out.vectors.begin(), s->out.vectors.end(), eigenvectors);
  });
}

int hsg_solution_complex_count(const hsg_solution* s, int64_t* mc) {
  return guarded([&] {
    HSG_REQUIRE(s && mc, HSG_INVALID_INPUT, "null argument");
    *mc = static_cast<int64_t>(s->out.complex_eigenvalues.size() / 2);
  });
}

int hsg_solution_complex_copy(const hsg_solution* s, double* eigenvalues, double* eigenvectors) {
  return guarded([&] {
    HSG_REQUIRE(s, HSG_INVALID_INPUT, "null solution");
    if (eigenvalues) std::copy(s->out.complex_eigenvalues.begin(), s->out.complex_eigenvalues.end(), eigenvalues);
    if (eigenvectors) std::copy(s->out.complex_vectors.begin(), s->out.complex_vectors.end(), eigenvectors);
  });
}

const char* hsg_solution_report(const hsg_solution* s) { return s ? s->out.report_json.c_str() : ""; }

void hsg_solution_free(hsg_solution* s) { delete s; }

}  // extern "C"
