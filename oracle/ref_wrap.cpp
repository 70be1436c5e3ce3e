// ORACLE (test infrastructure only): plain C entry points over parts of the reference itself that
// compile from their own sources (nested-dissection ordering, the pencil pattern, the sparse
// kernels), linked with them into oracle/_ref/libhsolve_ref.so by `make -C oracle ref`. Only tests/
// use it, as a checker: the reference's pivot order and its shifted residual are compared with this
// project's. Reference interfaces wrapped: hs::compute_ordering (include/hsolve/factor.hpp:631),
// hs::ShiftedPencil (include/hsolve/sparse.hpp:176-223), hs::shifted_residual and hs::spmm
// (include/hsolve/sparse.hpp:140-174).
#include <cstdint>
#include <cstring>
#include <exception>
#include <vector>

#include "hsolve/factor.hpp"
#include "hsolve/sparse.hpp"

namespace {

hs::CsrMatrix<double> csr(std::int64_t n, const std::int64_t* rp, const std::int32_t* ci, const double* v) {
  hs::CsrMatrix<double> m;
  m.nrows = n;
  m.ncols = n;
  m.rowptr.assign(rp, rp + n + 1);
  m.colind.assign(ci, ci + rp[n]);
  m.values.assign(v, v + rp[n]);
  return m;
}

}  // namespace

extern "C" {

// PERM_IN of the reference's nested dissection for the pencil (A, B) (B may be null: identity);
// full symmetric CSR input. Returns 0 on success, 1 on an exception.
int ref_compute_ordering(std::int64_t n, const std::int64_t* arp, const std::int32_t* aci, const double* av,
                         const std::int64_t* brp, const std::int32_t* bci, const double* bv,
                         std::uint64_t seed, int threads, std::int32_t* perm_in, std::int64_t* top_separator) {
  try {
    const hs::CsrMatrix<double> a = csr(n, arp, aci, av);
    hs::CsrMatrix<double> b;
    if (brp) b = csr(n, brp, bci, bv);
    const hs::ShiftedPencil<double> pencil(a, brp ? &b : nullptr);
    hs::OrderingOptions opt;
    opt.seed = seed;
    opt.threads = threads;
    hs::OrderingStats st;
    const std::vector<int> p = hs::compute_ordering(pencil, opt, &st);
    for (std::int64_t i = 0; i < n; ++i) perm_in[i] = p[static_cast<std::size_t>(i)];
    if (top_separator) *top_separator = st.top_separator;
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

// R = B X - (A Y - sigma B Y) for p columns (B null: identity), column-major with ld n, and the
// componentwise backward error of every column (omega, p entries), on the reference path.
int ref_shifted_residual(std::int64_t n, const std::int64_t* arp, const std::int32_t* aci, const double* av,
                         const std::int64_t* brp, const std::int32_t* bci, const double* bv, double sigma,
                         const double* x, const double* y, double* r, std::int64_t p, double* omega) {
  try {
    const hs::CsrMatrix<double> a = csr(n, arp, aci, av);
    hs::CsrMatrix<double> b;
    if (brp) b = csr(n, brp, bci, bv);
    hs::KernelOptions ko;
    ko.path = hs::KernelPath::Reference;
    hs::shifted_residual(a, brp ? &b : nullptr, sigma, x, n, y, n, r, n, p, ko, omega);
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

// Y = A X for p columns (ld n), on the reference path.
int ref_spmm(std::int64_t n, const std::int64_t* arp, const std::int32_t* aci, const double* av, const double* x,
             double* y, std::int64_t p) {
  try {
    const hs::CsrMatrix<double> a = csr(n, arp, aci, av);
    hs::KernelOptions ko;
    ko.path = hs::KernelPath::Reference;
    hs::spmm(a, x, n, y, n, p, 1.0, 0.0, ko);
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

}  // extern "C"
