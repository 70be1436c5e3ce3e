// Numeric multifrontal LDL^T kernels for sm_100a (FP64).
//
// What replaces MUMPS JOB=2 (hsolve src/factor/mumps_factorization.cpp:300-356; the arithmetic of
// MUMPS dfac_front_LDLT_type1.F / dfac_front_aux.F / dfac_asm.F): symmetric equilibration of
// K = alpha A + beta B, scatter of K into the fronts' panels, extend-add of children's contribution
// blocks, and the partial factorization of every front with 1x1 / 2x2 threshold pivots restricted
// to its fully-summed columns. Inertia (neg / zero / pos) is counted from D as pivots are accepted.
//
// Fronts are processed level by level (height in the assembly tree). Small fronts (m <= 64) are
// factorized entirely in shared memory by one CTA with right-looking threshold Bunch-Kaufman.
// Larger fronts use a-posteriori threshold pivoting by panels of NB columns: the diagonal block is
// factorized with Bunch-Kaufman restricted to the block, the rows below are solved against it while
// the largest |l| of every column is recorded, the longest acceptable prefix of pivots is kept
// (|l| <= 1/u), rejected columns are restored from a backup and moved behind the candidates, and
// the trailing matrix receives the rank-q update. Columns no candidate order can pivot are reported
// (failed) so that the host can move them into the parent front and factorize again.
#include <cooperative_groups.h>
#include <cstdint>

#include "common.hpp"
#include "device.cuh"
#include "factor_kernels.cuh"

namespace hsg {

namespace {

constexpr double kAlphaBK = 0.6403882032022076;  // (1 + sqrt(17)) / 8

// ------------------------------------------------------------------ scaling and assembly

__global__ void k_fill(double* x, std::int64_t n, double v) {
  for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::int64_t>(gridDim.x) * blockDim.x)
    x[i] = v;
}

__global__ void k_zero_u64(unsigned long long* x, std::int64_t n) {
  for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::int64_t>(gridDim.x) * blockDim.x)
    x[i] = 0ull;
}

// r[i] = max_j |d_i K_ij d_j| over both triangles (atomic max on non-negative doubles)
__global__ void k_scale_rowmax(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                               const double* b, double alpha, double beta, const double* d, unsigned long long* r) {
  for (std::int64_t p = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; p < nnz;
       p += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int32_t i = row[p], j = col[p];
    const double v = fabs((alpha * a[p] + beta * b[p]) * d[i] * d[j]);
    atomic_max_nonneg(&r[i], v);
    if (i != j) atomic_max_nonneg(&r[j], v);
  }
}

__global__ void k_scale_update(std::int64_t n, double* d, unsigned long long* r) {
  for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const double v = __longlong_as_double(static_cast<long long>(r[i]));
    if (v > 0.0) d[i] = d[i] / sqrt(v);
    r[i] = 0ull;
  }
}

// panels[dest[p]] = d_i d_j (alpha a_p + beta b_p); records max |.| for the null-pivot threshold
__global__ void k_scatter(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                          const double* b, double alpha, double beta, const double* d, const std::int64_t* dest,
                          double* panels, FactorCounters* cnt) {
  double mx = 0.0;
  for (std::int64_t p = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; p < nnz;
       p += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int32_t i = row[p], j = col[p];
    const double v = (alpha * a[p] + beta * b[p]) * d[i] * d[j];
    panels[dest[p]] = v;
    mx = fmax(mx, fabs(v));
  }
  mx = warp_max(mx);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&cnt->amax_bits, mx);
}

// zero the contribution blocks of the listed fronts (grid: fronts x chunks)
__global__ void k_zero_cb(const std::int32_t* list, const SnDev* sn, double* cb) {
  const SnDev s = sn[list[blockIdx.x]];
  const std::int64_t c = s.m - s.k;
  const std::int64_t total = c * c;
  double* base = cb + s.cb_off;
  for (std::int64_t i = blockIdx.y * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::int64_t>(gridDim.y) * blockDim.x)
    base[i] = 0.0;
}

// Extend-add: item = (child, first column of a column block). Adds the child's lower CB
// columns [b0, b0 + EA_COLS) into its parent front (panel part or contribution block).
__global__ void k_extend_add(const int2* items, const SnDev* sn, const std::int32_t* rmap, double* panels, double* cb) {
  const int2 it = items[blockIdx.x];
  const SnDev c = sn[it.x];
  const SnDev p = sn[c.parent];
  const std::int32_t mc = c.m - c.k;
  const std::int32_t* rm = rmap + c.rmap_off;
  const double* src = cb + c.cb_off;
  const std::int32_t pc = p.m - p.k;
  const std::int32_t bend = min(it.y + kExtendAddCols, mc);
  for (std::int32_t bb = it.y; bb < bend; ++bb) {
    const std::int32_t pb = rm[bb];
    double* dst;
    std::int64_t ld_off;
    if (pb < p.k) { dst = panels + p.panel_off + static_cast<std::int64_t>(pb) * p.m; ld_off = 0; }
    else { dst = cb + p.cb_off + static_cast<std::int64_t>(pb - p.k) * pc; ld_off = p.k; }
    const double* col = src + static_cast<std::int64_t>(bb) * mc;
    for (std::int32_t a = bb + threadIdx.x; a < mc; a += blockDim.x) dst[rm[a] - ld_off] += col[a];
  }
}

// ------------------------------------------------------------ dense pivoting in shared memory

// Decision of one pivot step (computed by warp 0).
enum : int { kFail = 0, kOneJ = 1, kOneR = 2, kTwoR = 3, kNull = 4 };

struct StepShared {
  int j, lim, prog, force, dec, r, stop;
  int neg, pos, zero, two, forced;
};

// Warp 0: decide the pivot at column j of the lower-stored matrix F (order m, ld ld) with
// candidates [j, nfs). Row maxima cover all rows [j, m).
__device__ void decide_pivot(const double* F, int ld, int m, int nfs, int j, double u, double thr, bool force,
                             StepShared& st) {
  const int lane = threadIdx.x & 31;
  const double* cj = F + static_cast<std::int64_t>(j) * ld;
  double gc = 0.0, best = 0.0;
  int r = -1;
  for (int i = j + 1 + lane; i < m; i += 32) {
    const double v = fabs(cj[i]);
    gc = fmax(gc, v);
    if (i < nfs && v > best) { best = v; r = i; }
  }
  gc = warp_max(gc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int orr = __shfl_xor_sync(0xffffffffu, r, o);
    if (ob > best || (ob == best && orr >= 0 && (r < 0 || orr < r))) { best = ob; r = orr; }
  }
  const double dcc = fabs(cj[j]);
  int dec = kFail;
  if (thr >= 0.0 && fmax(dcc, gc) <= thr) dec = kNull;
  else if (dcc > 0.0 && dcc >= u * gc) dec = kOneJ;
  else if (force && (r < 0 || best == 0.0 || dcc >= kAlphaBK * gc)) dec = dcc > 0.0 ? kOneJ : kNull;
  if (dec == kFail && r >= 0 && best > 0.0) {
    // maxima of columns j and r excluding rows {j, r}
    const double* cr = F + static_cast<std::int64_t>(r) * ld;
    double gc2 = 0.0, gr2 = 0.0;
    for (int i = j + 1 + lane; i < m; i += 32) {
      if (i != r) gc2 = fmax(gc2, fabs(cj[i]));
      if (i < r && i != j) gr2 = fmax(gr2, fabs(F[r + static_cast<std::int64_t>(i) * ld]));
      if (i > r) gr2 = fmax(gr2, fabs(cr[i]));
    }
    gc2 = warp_max(gc2);
    gr2 = warp_max(gr2);
    const double a = cj[j], b = cj[r], c = cr[r];
    const double det = a * c - b * b;
    if (force) {
      dec = det != 0.0 ? kTwoR : (dcc > 0.0 ? kOneJ : kNull);
    } else {
      if (det != 0.0) {
        const double ia = fabs(c / det), ib = fabs(b / det), ic = fabs(a / det);
        if (ia * gc2 + ib * gr2 <= 1.0 / u && ib * gc2 + ic * gr2 <= 1.0 / u) dec = kTwoR;
      }
      if (dec == kFail) {
        const double drr = fabs(c);
        if (drr > 0.0 && drr >= u * fmax(fabs(b), gr2)) dec = kOneR;
      }
    }
  }
  if (lane == 0) { st.dec = dec; st.r = r; }
}

// symmetric swap of positions p, q (< m) of the lower-stored matrix; labels follow
__device__ void sym_swap(double* F, int ld, int m, int p, int q, int* lab) {
  if (p == q) return;
  if (p > q) { const int t = p; p = q; q = t; }
  const int n1 = p, n2 = q - p - 1, n3 = m - q - 1;
  for (int t = threadIdx.x; t < n1 + n2 + n3 + 1; t += blockDim.x) {
    double *x, *y;
    if (t < n1) { x = F + p + static_cast<std::int64_t>(t) * ld; y = F + q + static_cast<std::int64_t>(t) * ld; }
    else if (t < n1 + n2) { const int c = p + 1 + (t - n1); x = F + c + static_cast<std::int64_t>(p) * ld; y = F + q + static_cast<std::int64_t>(c) * ld; }
    else if (t < n1 + n2 + n3) { const int i = q + 1 + (t - n1 - n2); x = F + i + static_cast<std::int64_t>(p) * ld; y = F + i + static_cast<std::int64_t>(q) * ld; }
    else { x = F + p + static_cast<std::int64_t>(p) * ld; y = F + q + static_cast<std::int64_t>(q) * ld; }
    const double v = *x; *x = *y; *y = v;
  }
  if (threadIdx.x == 0 && lab) { const int t = lab[p]; lab[p] = lab[q]; lab[q] = t; }
}

// eliminate a 1x1 (or null) pivot at j: column scaled to l, trailing rows/cols [j+1, m) updated
__device__ void elim1(double* F, int ld, int m, int j, bool null_piv, double* tmp) {
  const double d = F[j + static_cast<std::int64_t>(j) * ld];
  double* cj = F + static_cast<std::int64_t>(j) * ld;
  for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) {
    const double x = cj[i];
    tmp[i] = null_piv ? 0.0 : x;
    cj[i] = null_piv ? 0.0 : x / d;
  }
  __syncthreads();
  if (!null_piv) {
    const int w = m - j - 1;
    const double inv = 1.0 / d;
    for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
      const int i = j + 1 + t % w, c = j + 1 + t / w;
      if (i >= c) F[i + static_cast<std::int64_t>(c) * ld] -= tmp[i] * tmp[c] * inv;
    }
  }
  __syncthreads();
}

// eliminate the 2x2 pivot (j, j+1)
__device__ void elim2(double* F, int ld, int m, int j, double* tmp0, double* tmp1) {
  const double a = F[j + static_cast<std::int64_t>(j) * ld], b = F[j + 1 + static_cast<std::int64_t>(j) * ld];
  const double c = F[j + 1 + static_cast<std::int64_t>(j + 1) * ld];
  const double det = a * c - b * b;
  const double ia = c / det, ib = -b / det, ic = a / det;
  double* c0 = F + static_cast<std::int64_t>(j) * ld;
  double* c1 = F + static_cast<std::int64_t>(j + 1) * ld;
  for (int i = j + 2 + threadIdx.x; i < m; i += blockDim.x) {
    const double x0 = c0[i], x1 = c1[i];
    tmp0[i] = x0;
    tmp1[i] = x1;
    c0[i] = ia * x0 + ib * x1;
    c1[i] = ib * x0 + ic * x1;
  }
  __syncthreads();
  const int w = m - j - 2;
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
    const int i = j + 2 + t % w, cc = j + 2 + t / w;
    if (i >= cc) F[i + static_cast<std::int64_t>(cc) * ld] -= c0[i] * tmp0[cc] + c1[i] * tmp1[cc];
  }
  __syncthreads();
}

// Threshold Bunch-Kaufman on a lower-stored dense matrix in shared memory: candidates [0, nfs),
// rows [0, m). root: pivots may be forced (never fail). Returns the number of eliminated columns
// (positions [e, nfs) failed); pv[t] in {0 null, 1 1x1, 2/3 2x2}; lab follows the swaps.
__device__ int dense_bk(double* F, int ld, int m, int nfs, bool root, double u, double thr, int* lab, signed char* pv,
                        double* tmp0, double* tmp1, StepShared& st) {
  if (threadIdx.x == 0) {
    st.j = 0; st.lim = nfs; st.prog = 0; st.force = 0; st.stop = 0;
    st.neg = st.pos = st.zero = st.two = st.forced = 0;
  }
  __syncthreads();
  while (true) {
    if (threadIdx.x == 0) {
      st.stop = 0;
      if (st.j >= nfs) st.stop = 1;
      else if (st.j >= st.lim) {
        if (st.prog) { st.lim = nfs; st.prog = 0; st.stop = 2; }
        else if (root && !st.force) { st.force = 1; st.lim = nfs; st.stop = 2; }
        else st.stop = 1;
      }
    }
    __syncthreads();
    if (st.stop == 1) break;
    if (st.stop == 2) continue;
    const int j = st.j;
    if (threadIdx.x < 32) decide_pivot(F, ld, m, nfs, j, u, thr, st.force != 0, st);
    __syncthreads();
    const int dec = st.dec, r = st.r;
    if (dec == kFail) {
      sym_swap(F, ld, m, j, st.lim - 1, lab);
      __syncthreads();
      if (threadIdx.x == 0) st.lim -= 1;
      __syncthreads();
      continue;
    }
    if (dec == kOneR) { sym_swap(F, ld, m, j, r, lab); __syncthreads(); }
    if (dec == kTwoR) { sym_swap(F, ld, m, j + 1, r, lab); __syncthreads(); }
    if (dec == kTwoR) {
      if (threadIdx.x == 0) {
        const double a = F[j + static_cast<std::int64_t>(j) * ld], b = F[j + 1 + static_cast<std::int64_t>(j) * ld];
        const double c = F[j + 1 + static_cast<std::int64_t>(j + 1) * ld];
        const double det = a * c - b * b;
        if (det < 0) { st.neg++; st.pos++; } else if (a + c < 0) st.neg += 2; else st.pos += 2;
        st.two++;
        if (st.force) st.forced++;
        pv[j] = 2; pv[j + 1] = 3;
      }
      elim2(F, ld, m, j, tmp0, tmp1);
      if (threadIdx.x == 0) {
        st.j = j + 2; st.prog = 1; st.force = 0;
        if (st.lim < st.j) st.lim = st.j;
        if (st.lim == j + 1) st.lim = j + 2;
      }
    } else {
      const bool nul = dec == kNull;
      if (threadIdx.x == 0) {
        const double d = F[j + static_cast<std::int64_t>(j) * ld];
        if (nul) { st.zero++; pv[j] = 0; }
        else { if (d < 0) st.neg++; else st.pos++; pv[j] = 1; }
        if (st.force) st.forced++;
      }
      elim1(F, ld, m, j, nul, tmp0);
      if (threadIdx.x == 0) {
        st.j = j + 1; st.prog = 1; st.force = 0;
        if (st.lim < st.j) st.lim = st.j;
      }
    }
    __syncthreads();
  }
  __syncthreads();
  return st.j;
}

}  // namespace

// ---------------------------------------------------------------------- small fronts (smem)

template <int MAXM>
__global__ void __launch_bounds__(256) k_front_small(const std::int32_t* list, const SnDev* sn, double* panels,
                                                      double* cb, signed char* piv_out, std::int32_t* pidx_out,
                                                      FactorParams prm, FactorCounters* cnt, std::int32_t* failed) {
  extern __shared__ double F[];
  __shared__ double tmp0[MAXM], tmp1[MAXM];
  __shared__ int lab[MAXM];
  __shared__ signed char pv[MAXM];
  __shared__ StepShared st;
  const SnDev d = sn[list[blockIdx.x]];
  const int m = d.m, k = d.k, ld = m, c = m - k;
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int i = t % m, j = t / m;
    if (i < j) continue;
    F[t] = j < k ? panels[d.panel_off + static_cast<std::int64_t>(j) * m + i]
                 : cb[d.cb_off + static_cast<std::int64_t>(j - k) * c + (i - k)];
  }
  for (int t = threadIdx.x; t < m; t += blockDim.x) lab[t] = t;
  __syncthreads();
  const double thr = null_threshold(prm);
  const int e = dense_bk(F, ld, m, k, d.parent < 0, prm.u, thr, lab, pv, tmp0, tmp1, st);
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int i = t % m, j = t / m;
    if (i < j) continue;
    if (j < k) panels[d.panel_off + static_cast<std::int64_t>(j) * m + i] = F[t];
    else cb[d.cb_off + static_cast<std::int64_t>(j - k) * c + (i - k)] = F[t];
  }
  for (int t = threadIdx.x; t < k; t += blockDim.x) {
    pidx_out[d.first + t] = lab[t];
    piv_out[d.first + t] = t < e ? pv[t] : static_cast<signed char>(-1);
  }
  if (threadIdx.x == 0) {
    if (st.neg) atomicAdd(&cnt->neg, static_cast<unsigned long long>(st.neg));
    if (st.pos) atomicAdd(&cnt->pos, static_cast<unsigned long long>(st.pos));
    if (st.zero) atomicAdd(&cnt->zero, static_cast<unsigned long long>(st.zero));
    if (st.two) atomicAdd(&cnt->two_by_two, static_cast<unsigned long long>(st.two));
    if (st.forced) atomicAdd(&cnt->forced, static_cast<unsigned long long>(st.forced));
    if (e < k) {
      const unsigned long long at = atomicAdd(&cnt->failed, static_cast<unsigned long long>(k - e));
      for (int t = e; t < k; ++t)
        if (at + (t - e) < static_cast<unsigned long long>(prm.failed_cap)) failed[at + (t - e)] = d.first + lab[t];
    }
  }
}

// ------------------------------------------------------------- larger fronts: a-posteriori pivoting
//
// One front is processed by nr CTAs (nr = 1 for the one-CTA-per-front kernel; nr >= 1 per front in the
// cooperative kernel, where every step is separated by a grid-wide barrier). The pivoting state of a
// front lives in its global scratch (AppCtrl + block + labels + column maxima + backup), written by
// the front's rank-0 CTA and read by all its CTAs after the barrier.

namespace {

struct FrontView {
  double* panel;  // m x k, ld m
  double* cbb;    // (m-k)^2, ld m-k
  int m, k;
  __device__ double* col(int c) const {
    return c < k ? panel + static_cast<std::int64_t>(c) * m : cbb + static_cast<std::int64_t>(c - k) * (m - k) - k;
  }
  __device__ double& at(int i, int c) const { return col(c)[i]; }
};

struct AppCtrl {
  int p, lim, prog, force, stop, w, eb, q;
  int neg, pos, zero, two, forced, finished, pad0, pad1;
};

struct AppFront {
  FrontView f;
  int first;
  bool root;
  AppCtrl* ctrl;
  double* B;       // factored diagonal block, kNB x kNB col-major
  double* Borig;   // the block before factorization
  int* lab;        // block permutation
  signed char* pv; // block pivot types
  unsigned long long* cmax;
  unsigned long long* rmax;
  double* backup;  // kNB columns of m rows
  std::int32_t* plab;
  signed char* ppv;
};

__device__ AppFront make_front(const SnDev& d, double* panels, double* cb, double* scratch, signed char* piv_out,
                               std::int32_t* pidx_out) {
  AppFront F;
  F.f = FrontView{panels + d.panel_off, d.cb_off >= 0 ? cb + d.cb_off : nullptr, d.m, d.k};
  F.first = d.first;
  F.root = d.parent < 0;
  double* s = scratch + d.scratch_off;
  F.ctrl = reinterpret_cast<AppCtrl*>(s);
  s += kAppCtrlDoubles;
  F.B = s;
  s += kNB * kNB;
  F.Borig = s;
  s += kNB * kNB;
  F.lab = reinterpret_cast<int*>(s);
  s += kNB / 2;
  F.pv = reinterpret_cast<signed char*>(s);
  s += kNB / 8;
  F.cmax = reinterpret_cast<unsigned long long*>(s);
  s += kNB;
  F.rmax = reinterpret_cast<unsigned long long*>(s);
  s += kNB;
  F.backup = s;
  F.plab = pidx_out + d.first;
  F.ppv = piv_out + d.first;
  return F;
}

// symmetric swap of fully-summed positions a, b (< k) of the front in global memory
__device__ void front_swap(const FrontView& f, int a, int b, std::int32_t* lab) {
  if (a == b) return;
  if (a > b) { const int t = a; a = b; b = t; }
  const int n1 = a, n2 = b - a - 1, n3 = f.m - b - 1;
  for (int t = threadIdx.x; t < n1 + n2 + n3 + 1; t += blockDim.x) {
    double *x, *y;
    if (t < n1) { x = &f.at(a, t); y = &f.at(b, t); }
    else if (t < n1 + n2) { const int c = a + 1 + (t - n1); x = &f.at(c, a); y = &f.at(b, c); }
    else if (t < n1 + n2 + n3) { const int i = b + 1 + (t - n1 - n2); x = &f.at(i, a); y = &f.at(i, b); }
    else { x = &f.at(a, a); y = &f.at(b, b); }
    const double v = *x; *x = *y; *y = v;
  }
  if (threadIdx.x == 0) { const std::int32_t t = lab[a]; lab[a] = lab[b]; lab[b] = t; }
}

// Init (all ranks split the label work; rank 0 the control block).
__device__ void app_init(AppFront& F, int rank, int nr) {
  const int k = F.f.k;
  for (int t = rank * blockDim.x + threadIdx.x; t < k; t += nr * blockDim.x) { F.plab[t] = t; F.ppv[t] = -1; }
  if (rank == 0 && threadIdx.x == 0) {
    AppCtrl c{};
    c.lim = k;
    *F.ctrl = c;
  }
}

// Rank 0: decide what the next panel is (stop = 1: front finished), and factorize its diagonal block
// with block-restricted threshold Bunch-Kaufman; permute the L rows of the block; publish to scratch.
__device__ void app_control_and_block(AppFront& F, const FactorParams& prm, double thr, double* Bs, double* tmp0,
                                      double* tmp1, int* slab, signed char* spv, StepShared& bst, int* shared_stop,
                                      FactorCounters* cnt, std::int32_t* failed, int* level_done) {
  AppCtrl* c = F.ctrl;
  const int k = F.f.k;
  if (threadIdx.x == 0) {
    int stop = 1;
    if (!c->finished) {
      while (true) {
        if (c->p >= k) { stop = 1; break; }
        if (c->p >= c->lim) {
          if (c->prog) { c->lim = k; c->prog = 0; continue; }
          if (F.root && !c->force) { c->force = 1; c->lim = k; continue; }
          stop = 1;
          break;
        }
        stop = 0;
        c->w = min(kNB, c->lim - c->p);
        break;
      }
    }
    c->stop = stop;
    *shared_stop = stop;
    if (stop && !c->finished) {
      c->finished = 1;
      const int e = c->p;
      if (c->neg) atomicAdd(&cnt->neg, static_cast<unsigned long long>(c->neg));
      if (c->pos) atomicAdd(&cnt->pos, static_cast<unsigned long long>(c->pos));
      if (c->zero) atomicAdd(&cnt->zero, static_cast<unsigned long long>(c->zero));
      if (c->two) atomicAdd(&cnt->two_by_two, static_cast<unsigned long long>(c->two));
      if (c->forced) atomicAdd(&cnt->forced, static_cast<unsigned long long>(c->forced));
      if (e < k) {
        const unsigned long long at = atomicAdd(&cnt->failed, static_cast<unsigned long long>(k - e));
        for (int t = e; t < k; ++t)
          if (at + (t - e) < static_cast<unsigned long long>(prm.failed_cap)) failed[at + (t - e)] = F.first + F.plab[t];
      }
      if (level_done) atomicAdd(level_done, 1);
    }
  }
  __syncthreads();
  if (*shared_stop) return;
  const int p = c->p, w = c->w;
  const bool force = c->force != 0;
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
    const int i = t % w, j = t / w;
    if (i >= j) {
      const double v = F.f.at(p + i, p + j);
      Bs[i + j * kNB] = v;
      F.Borig[i + j * kNB] = v;
    }
  }
  for (int t = threadIdx.x; t < w; t += blockDim.x) slab[t] = t;
  __syncthreads();
  const int eb = dense_bk(Bs, kNB, w, w, force, prm.u, thr, slab, spv, tmp0, tmp1, bst);
  // permute the L rows p..p+w-1 of the eliminated columns c < p
  for (int c0 = 0; c0 < p; c0 += blockDim.x / kNB) {
    const int cc = c0 + threadIdx.x / kNB, a = threadIdx.x % kNB;
    double v = 0.0;
    if (cc < p && a < w) v = F.f.at(p + slab[a], cc);
    __syncthreads();
    if (cc < p && a < w) F.f.at(p + a, cc) = v;
    __syncthreads();
  }
  {
    int old = 0;
    if (threadIdx.x < w) old = F.plab[p + slab[threadIdx.x]];
    __syncthreads();
    if (threadIdx.x < w) F.plab[p + threadIdx.x] = old;
  }
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
    const int i = t % w, j = t / w;
    if (i >= j) F.f.at(p + i, p + j) = Bs[i + j * kNB];
  }
  for (int t = threadIdx.x; t < kNB * kNB; t += blockDim.x) F.B[t] = Bs[t];
  for (int t = threadIdx.x; t < kNB; t += blockDim.x) {
    F.lab[t] = slab[t];
    F.pv[t] = spv[t];
    F.cmax[t] = 0ull;
    F.rmax[t] = 0ull;
  }
  if (threadIdx.x == 0) c->eb = eb;
}

// All ranks: rows [p+w, m) solved against the block (L21 = F21 P L11^-T D^-1), backup, column maxima.
__device__ void app_rows(AppFront& F, int rank, int nr, double* Bs, int* slab, signed char* spv,
                         unsigned long long* scm, unsigned long long* srm) {
  const AppCtrl* c = F.ctrl;
  const int p = c->p, w = c->w, eb = c->eb, m = F.f.m;
  for (int t = threadIdx.x; t < kNB * kNB; t += blockDim.x) Bs[t] = F.B[t];
  for (int t = threadIdx.x; t < kNB; t += blockDim.x) {
    slab[t] = F.lab[t];
    spv[t] = F.pv[t];
    scm[t] = 0ull;
    srm[t] = 0ull;
  }
  __syncthreads();
  for (int i = p + w + rank * blockDim.x + threadIdx.x; i < m; i += nr * blockDim.x) {
    double x[kNB], y[kNB];
#pragma unroll
    for (int t = 0; t < kNB; ++t) x[t] = t < w ? F.f.at(i, p + t) : 0.0;
#pragma unroll
    for (int t = 0; t < kNB; ++t)
      if (t < w) F.backup[static_cast<std::int64_t>(t) * m + i] = x[t];
    for (int t = 0; t < w; ++t) {
      double v = x[slab[t]];
      const int lim_s = t < eb ? t : eb;
      for (int s = 0; s < lim_s; ++s) {
        if (spv[s] == 2 && s + 1 == t) continue;
        v -= y[s] * Bs[t + s * kNB];
      }
      y[t] = v;
    }
    for (int t = 0; t < w; ++t) {
      double out;
      if (t < eb) {
        const signed char ty = spv[t];
        if (ty == 0) out = 0.0;
        else if (ty == 1) out = y[t] / Bs[t + t * kNB];
        else if (ty == 2) {
          const double a = Bs[t + t * kNB], b = Bs[t + 1 + t * kNB], cc = Bs[t + 1 + (t + 1) * kNB];
          out = (cc * y[t] - b * y[t + 1]) / (a * cc - b * b);
        } else {
          const double a = Bs[t - 1 + (t - 1) * kNB], b = Bs[t + (t - 1) * kNB], cc = Bs[t + t * kNB];
          out = (-b * y[t - 1] + a * y[t]) / (a * cc - b * b);
        }
        atomic_max_nonneg(&scm[t], fabs(out));
        atomic_max_nonneg(&srm[t], fabs(y[t]));
      } else {
        out = y[t];
      }
      F.f.at(i, p + t) = out;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < w; t += blockDim.x) {
    if (scm[t]) atomicMax(&F.cmax[t], scm[t]);
    if (srm[t]) atomicMax(&F.rmax[t], srm[t]);
  }
}

// All ranks: the accepted prefix q (identical in every CTA); rank 0 books the inertia.
__device__ int app_accept(AppFront& F, int rank, bool force, double thr, double inv_u, int* sq) {
  const AppCtrl* c = F.ctrl;
  const int eb = c->eb;
  if (threadIdx.x == 0) {
    int q = 0;
    while (q < eb) {
      const signed char ty = F.pv[q];
      const double cm = __longlong_as_double(static_cast<long long>(F.cmax[q]));
      if (ty == 0) {
        if (!force && __longlong_as_double(static_cast<long long>(F.rmax[q])) > thr) break;
        q += 1;
      } else if (ty == 1) {
        if (!force && cm > inv_u) break;
        q += 1;
      } else {
        const double cm2 = __longlong_as_double(static_cast<long long>(F.cmax[q + 1]));
        if (!force && fmax(cm, cm2) > inv_u) break;
        q += 2;
      }
    }
    *sq = q;
  }
  __syncthreads();
  const int q = *sq;
  if (rank == 0) {
    for (int t = threadIdx.x; t < q; t += blockDim.x) F.ppv[c->p + t] = F.pv[t];
    if (threadIdx.x == 0) {
      AppCtrl* cw = F.ctrl;
      cw->q = q;
      for (int t = 0; t < q; ++t) {
        const signed char ty = F.pv[t];
        if (ty == 0) cw->zero++;
        else if (ty == 1) { if (F.B[t + t * kNB] < 0) cw->neg++; else cw->pos++; }
        else if (ty == 2) {
          const double a = F.B[t + t * kNB], b = F.B[t + 1 + t * kNB], cc = F.B[t + 1 + (t + 1) * kNB];
          const double det = a * cc - b * b;
          if (det < 0) { cw->neg++; cw->pos++; } else if (a + cc < 0) cw->neg += 2; else cw->pos += 2;
          cw->two++;
        }
      }
      if (force) cw->forced += q;
    }
  }
  return q;
}

// All ranks: restore the rejected block columns [q, w) from the backup / original block.
__device__ void app_restore(AppFront& F, int rank, int nr, int q) {
  const AppCtrl* c = F.ctrl;
  const int p = c->p, w = c->w, m = F.f.m;
  for (int i = p + w + rank * blockDim.x + threadIdx.x; i < m; i += nr * blockDim.x)
    for (int t = q; t < w; ++t) F.f.at(i, p + t) = F.backup[static_cast<std::int64_t>(F.lab[t]) * m + i];
  if (rank == 0) {
    for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
      const int a = t % w, b = t / w;
      if (b >= q && a >= b) {
        const int la = F.lab[a], lb = F.lab[b];
        F.f.at(p + a, p + b) = la >= lb ? F.Borig[la + lb * kNB] : F.Borig[lb + la * kNB];
      }
    }
  }
}

// All ranks: C(i, c) -= sum_{s<q} L(i, p+s) W(c, s), from <= c <= i < m, W = L D; 64 x 64 tiles
// of the lower triangle dealt round-robin to the ranks; 4 x 4 outputs per thread.
__device__ void app_update(AppFront& F, int rank, int nr, int q, double* Ls, double* Ws, const double* Bs,
                           const signed char* spv) {
  const AppCtrl* c = F.ctrl;
  const int p = c->p, from = p + q, m = F.f.m;
  const int rows = m - from;
  if (rows <= 0 || q <= 0) return;
  const int nt = (rows + kTile - 1) / kTile;
  const int ntiles = nt * (nt + 1) / 2;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  for (int tile = rank; tile < ntiles; tile += nr) {
    int ti = static_cast<int>((sqrt(8.0 * tile + 1.0) - 1.0) * 0.5);
    while ((ti + 1) * (ti + 2) / 2 <= tile) ++ti;
    while (ti * (ti + 1) / 2 > tile) --ti;
    const int tj = tile - ti * (ti + 1) / 2;
    const int i0 = from + ti * kTile, j0 = from + tj * kTile;
    __syncthreads();
    for (int t = threadIdx.x; t < q * kTile; t += blockDim.x) {
      const int s = t / kTile, r = t % kTile;
      const int i = i0 + r, cc = j0 + r;
      Ls[s * kTile + r] = i < m ? F.f.at(i, p + s) : 0.0;
      double wv = 0.0;
      if (cc < m) {
        const signed char tyv = spv[s];
        if (tyv == 1) wv = F.f.at(cc, p + s) * Bs[s * kNB + s];
        else if (tyv == 2) wv = F.f.at(cc, p + s) * Bs[s * kNB + s] + F.f.at(cc, p + s + 1) * Bs[s * kNB + s + 1];
        else if (tyv == 3) wv = F.f.at(cc, p + s - 1) * Bs[(s - 1) * kNB + s] + F.f.at(cc, p + s) * Bs[s * kNB + s];
      }
      Ws[s * kTile + r] = wv;
    }
    __syncthreads();
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int s = 0; s < q; ++s) {
      double l[4], wv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) l[a] = Ls[s * kTile + tx + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) wv[b] = Ws[s * kTile + ty + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(l[a], wv[b], acc[a][b]);
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int cc = j0 + ty + 16 * b;
      if (cc >= m) continue;
      double* colp = F.f.col(cc);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int i = i0 + tx + 16 * a;
        if (i < m && cc <= i) colp[i] -= acc[a][b];
      }
    }
  }
}

// Rank 0: advance past the accepted pivots; move rejected columns behind the candidates.
__device__ void app_advance(AppFront& F, int q) {
  AppCtrl* c = F.ctrl;
  const int p = c->p, w = c->w;
  const int np = p + q, r = w - q;
  const int lim = c->lim;
  if (r > 0 && np + r < lim) {
    for (int t = 0; t < r; ++t) {
      front_swap(F.f, np + t, lim - r + t, F.plab);
      __syncthreads();
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    c->p = np;
    if (q > 0) { c->prog = 1; c->force = 0; }
    if (r > 0) c->lim = np + r < lim ? lim - r : np;
  }
  __syncthreads();
}

struct AppSmem {
  double Bs[kNB * kNB];
  double tmp0[kNB], tmp1[kNB];
  int slab[kNB];
  signed char spv[kNB];
  unsigned long long scm[kNB], srm[kNB];
  StepShared bst;
  int stop, q;
};

}  // namespace

// One CTA per front (nr = 1), fronts listed in `list`.
__global__ void __launch_bounds__(kAppThreads) k_front_app(const std::int32_t* list, const SnDev* sn, double* panels,
                                                           double* cb, double* scratch, signed char* piv_out,
                                                           std::int32_t* pidx_out, FactorParams prm,
                                                           FactorCounters* cnt, std::int32_t* failed) {
  extern __shared__ double app_dyn[];
  double* Ls = app_dyn;
  double* Ws = app_dyn + kNB * kTile;
  __shared__ AppSmem sm;
  const SnDev d = sn[list[blockIdx.x]];
  AppFront F = make_front(d, panels, cb, scratch, piv_out, pidx_out);
  const double thr = null_threshold(prm);
  const double inv_u = 1.0 / prm.u;
  app_init(F, 0, 1);
  __syncthreads();
  while (true) {
    app_control_and_block(F, prm, thr, sm.Bs, sm.tmp0, sm.tmp1, sm.slab, sm.spv, sm.bst, &sm.stop, cnt, failed, nullptr);
    __syncthreads();
    if (sm.stop) break;
    app_rows(F, 0, 1, sm.Bs, sm.slab, sm.spv, sm.scm, sm.srm);
    __syncthreads();
    const bool force = F.ctrl->force != 0;
    const int q = app_accept(F, 0, force, thr, inv_u, &sm.q);
    __syncthreads();
    if (q < F.ctrl->w) app_restore(F, 0, 1, q);
    __syncthreads();
    app_update(F, 0, 1, q, Ls, Ws, sm.Bs, sm.spv);
    __syncthreads();
    app_advance(F, q);
  }
}

// Cooperative: the fronts of a level share the grid; front f owns CTAs [cta_start[f], cta_start[f+1]).
// Grid-wide barriers separate the steps; the loop ends when every front has finished (level_done).
__global__ void __launch_bounds__(kAppThreads) k_front_coop(const std::int32_t* list, const std::int32_t* cta_start,
                                                            int nfronts, const SnDev* sn, double* panels, double* cb,
                                                            double* scratch, signed char* piv_out,
                                                            std::int32_t* pidx_out, FactorParams prm,
                                                            FactorCounters* cnt, std::int32_t* failed,
                                                            int* level_done) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ double app_dyn[];
  double* Ls = app_dyn;
  double* Ws = app_dyn + kNB * kTile;
  __shared__ AppSmem sm;
  int fi = 0;
  while (fi + 1 < nfronts && cta_start[fi + 1] <= static_cast<int>(blockIdx.x)) ++fi;
  const int rank = static_cast<int>(blockIdx.x) - cta_start[fi];
  const int nr = cta_start[fi + 1] - cta_start[fi];
  const SnDev d = sn[list[fi]];
  AppFront F = make_front(d, panels, cb, scratch, piv_out, pidx_out);
  const double thr = null_threshold(prm);
  const double inv_u = 1.0 / prm.u;
  app_init(F, rank, nr);
  grid.sync();
  while (true) {
    if (rank == 0) {
      app_control_and_block(F, prm, thr, sm.Bs, sm.tmp0, sm.tmp1, sm.slab, sm.spv, sm.bst, &sm.stop, cnt, failed,
                            level_done);
    }
    grid.sync();
    if (*reinterpret_cast<volatile int*>(level_done) >= nfronts) break;
    const bool active = F.ctrl->stop == 0;
    if (active) app_rows(F, rank, nr, sm.Bs, sm.slab, sm.spv, sm.scm, sm.srm);
    grid.sync();
    int q = 0;
    if (active) {
      q = app_accept(F, rank, F.ctrl->force != 0, thr, inv_u, &sm.q);
      if (q < F.ctrl->w) app_restore(F, rank, nr, q);
    }
    grid.sync();
    if (active) app_update(F, rank, nr, q, Ls, Ws, sm.Bs, sm.spv);
    grid.sync();
    if (active && rank == 0) app_advance(F, q);
  }
}

// ------------------------------------------------------------------------------ launchers

void launch_fill(double* x, std::int64_t n, double v, cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = static_cast<int>(std::min<std::int64_t>((n + 255) / 256, 148 * 16));
  note_launches(1);
  k_fill<<<blocks, 256, 0, s>>>(x, n, v);
}

void launch_zero_u64(unsigned long long* x, std::int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = static_cast<int>(std::min<std::int64_t>((n + 255) / 256, 148 * 16));
  note_launches(1);
  k_zero_u64<<<blocks, 256, 0, s>>>(x, n);
}

void launch_scale_rowmax(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                         const double* b, double alpha, double beta, const double* d, unsigned long long* r,
                         cudaStream_t s) {
  const int blocks = static_cast<int>(std::min<std::int64_t>((nnz + 255) / 256, 148 * 16));
  note_launches(1);
  k_scale_rowmax<<<blocks, 256, 0, s>>>(nnz, row, col, a, b, alpha, beta, d, r);
}

void launch_scale_update(std::int64_t n, double* d, unsigned long long* r, cudaStream_t s) {
  const int blocks = static_cast<int>(std::min<std::int64_t>((n + 255) / 256, 148 * 16));
  note_launches(1);
  k_scale_update<<<blocks, 256, 0, s>>>(n, d, r);
}

void launch_scatter(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                    const double* b, double alpha, double beta, const double* d, const std::int64_t* dest,
                    double* panels, FactorCounters* cnt, cudaStream_t s) {
  const int blocks = static_cast<int>(std::min<std::int64_t>((nnz + 255) / 256, 148 * 16));
  note_launches(1);
  k_scatter<<<blocks, 256, 0, s>>>(nnz, row, col, a, b, alpha, beta, d, dest, panels, cnt);
}

void launch_zero_cb(const std::int32_t* list, int nlist, int chunks, const SnDev* sn, double* cb, cudaStream_t s) {
  if (nlist <= 0) return;
  dim3 grid(nlist, chunks);
  note_launches(1);
  k_zero_cb<<<grid, 256, 0, s>>>(list, sn, cb);
}

void launch_extend_add(const int2* items, int nitems, const SnDev* sn, const std::int32_t* rmap, double* panels,
                       double* cb, cudaStream_t s) {
  if (nitems <= 0) return;
  note_launches(1);
  k_extend_add<<<nitems, 128, 0, s>>>(items, sn, rmap, panels, cb);
}

void launch_front_small(int maxm, const std::int32_t* list, int nlist, const SnDev* sn, double* panels, double* cb,
                        signed char* piv, std::int32_t* pidx, const FactorParams& prm, FactorCounters* cnt,
                        std::int32_t* failed, cudaStream_t s) {
  if (nlist <= 0) return;
  const std::size_t smem = static_cast<std::size_t>(maxm) * maxm * sizeof(double);
  if (maxm <= 32) { note_launches(1); k_front_small<32><<<nlist, 128, smem, s>>>(list, sn, panels, cb, piv, pidx, prm, cnt, failed); }
  else { note_launches(1); k_front_small<kSmallMax><<<nlist, 256, smem, s>>>(list, sn, panels, cb, piv, pidx, prm, cnt, failed); }
}

void launch_front_app(const std::int32_t* list, int nlist, const SnDev* sn, double* panels, double* cb,
                      double* scratch, signed char* piv, std::int32_t* pidx, const FactorParams& prm,
                      FactorCounters* cnt, std::int32_t* failed, cudaStream_t s) {
  if (nlist <= 0) return;
  constexpr std::size_t smem = 2 * kNB * kTile * sizeof(double);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_front_app, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    configured = true;
  }
  note_launches(1);
  k_front_app<<<nlist, kAppThreads, smem, s>>>(list, sn, panels, cb, scratch, piv, pidx, prm, cnt, failed);
}

int coop_max_ctas(int device) {
  constexpr std::size_t smem = 2 * kNB * kTile * sizeof(double);
  cudaFuncSetAttribute(k_front_coop, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  int per_sm = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_front_coop, kAppThreads, smem);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return per_sm * sms;
}

cudaError_t launch_front_coop(const std::int32_t* list, const std::int32_t* cta_start, int nfronts, int nctas,
                              const SnDev* sn, double* panels, double* cb, double* scratch, signed char* piv,
                              std::int32_t* pidx, const FactorParams& prm, FactorCounters* cnt, std::int32_t* failed,
                              int* level_done, cudaStream_t s) {
  if (nfronts <= 0) return cudaSuccess;
  constexpr std::size_t smem = 2 * kNB * kTile * sizeof(double);
  FactorParams p = prm;
  void* args[] = {const_cast<std::int32_t**>(&list), const_cast<std::int32_t**>(&cta_start), &nfronts,
                  const_cast<SnDev**>(&sn), &panels, &cb, &scratch, &piv, &pidx, &p, &cnt, &failed, &level_done};
  note_launches(1);
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_front_coop), dim3(nctas), dim3(kAppThreads), args, smem, s);
}

}  // namespace hsg
