// Supernodal forward / diagonal / backward solves with up to 8 right-hand sides per sweep (replaces
// MUMPS JOB=3, hsolve src/factor/mumps_factorization.cpp:459-527; MUMPS dsol_fwd.F / dsol_bwd.F).
//
// Solve operator. The pivots of every front are cut into super-blocks of kSB = 128 (a 2 x 2 pivot may
// straddle a boundary: its coupling entry is D, not L, and reads as zero). For a super-block
// B = [b, b + bs) of a front with unit lower panel L (m x k, column-major, ld m):
//     W[B, B] = L_BB^{-1}                 (lower triangular, zero above the diagonal)
//     W[i, B] = L[i, B] L_BB^{-1},  i >= b + bs  (later pivot rows and the contribution rows),
// stored like the panel in a separate buffer and built once per factorization before its first
// solve. Forward L z = t, super-block by super-block: z_B = W[B, B] t_B and t_i -= W[i, B] t_B below
// B (both read only t_B, so they run at once). Backward L^T x = y, from the last super-block down:
//     s_j = (W[A, A]^T y_A)_j - W[CB, j]^T x_CB        for every pivot j (A = j's super-block),
//     x_B = s_B after every later super-block C has been applied by s_j -= W[C, j]^T x_C.
//
// Schedule. Fronts are solved level by level of the elimination tree (children first forward,
// parents first backward), one launch per level and sweep. A front gets nr CTAs by its panel size
// (a task per CTA: front, rank, nr). Forward, 32-row groups belong to CTA (group mod nr) for the
// whole sweep; backward, 32-column chunks to CTA (chunk mod nr). The CTAs of a front publish the
// groups / chunks they finish through a per-front counter (fence + atomic add; the readers poll
// with acquire loads and a bound), so a front's steps need no grid barrier. A level whose fronts
// each have one CTA is an ordinary launch, any other level a cooperative launch (co-resident CTAs).
// No data is accumulated with atomics: every value has one writer and every sum is formed in a
// fixed order, so the results are bitwise reproducible.
#include <cstdint>
#include <mutex>

#include "common.hpp"
#include "device.cuh"
#include "solve_kernels.cuh"

namespace hsg {

namespace {

__global__ void k_gather_scale(std::int64_t n, int nrhs, const double* b, std::int64_t ldb, const double* d,
                               const std::int32_t* iperm, double* x) {
  const std::int64_t total = n * nrhs;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t i = t % n, r = t / n;
    x[iperm[i] + r * n] = b[i + r * ldb] * d[i];
  }
}

__global__ void k_scatter_scale(std::int64_t n, int nrhs, double* b, std::int64_t ldb, const double* d,
                                const std::int32_t* iperm, const double* x) {
  const std::int64_t total = n * nrhs;
  for (std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    const std::int64_t i = t % n, r = t / n;
    b[i + r * ldb] = x[iperm[i] + r * n] * d[i];
  }
}

}  // namespace

// Diagonal solve D y = z over all pivots at once (one thread per pivot position p): dpos[p] is the
// panel index of D(p, p), pfirst[p] the first global column of p's front.
template <class F>
__global__ void k_solve_diag_flat(std::int64_t npiv, const std::int64_t* dpos, const std::int32_t* pfirst,
                                  const F* panels, const signed char* piv, const std::int32_t* pidx, double* x,
                                  std::int64_t n, int nrhs) {
  const std::int64_t p = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= npiv) return;
  const signed char ty = piv[p];
  if (ty == 3) return;
  const std::int64_t g0 = pfirst[p] + pidx[p];
  if (ty <= 0) {
    for (int r = 0; r < nrhs; ++r) x[g0 + r * n] = 0.0;
  } else if (ty == 1) {
    const double dj = panels[dpos[p]];
    for (int r = 0; r < nrhs; ++r) x[g0 + r * n] /= dj;
  } else {
    const std::int64_t g1 = pfirst[p] + pidx[p + 1];
    const double a = panels[dpos[p]], b = panels[dpos[p] + 1], c = panels[dpos[p + 1]];
    const double det = a * c - b * b;
    for (int r = 0; r < nrhs; ++r) {
      const double y0 = x[g0 + r * n], y1 = x[g1 + r * n];
      x[g0 + r * n] = (c * y0 - b * y1) / det;
      x[g1 + r * n] = (-b * y0 + a * y1) / det;
    }
  }
}

// W[B, B] = L_BB^{-1} for one super-block per CTA: row-by-row substitution X[i, c] =
// -sum_{c <= j < i} L[i, j] X[j, c] on packed triangles in shared memory (two threads per column).
template <class F>
__global__ void __launch_bounds__(256) k_sb_inverse(const int2* sbl, const SnDev* sn, const F* panels,
                                                     const signed char* piv, F* W) {
  extern __shared__ double sm[];
  double* Lp = sm;                                // strictly lower rows, row i at i(i-1)/2
  double* Xp = sm + kSB * (kSB - 1) / 2;          // lower rows incl. diagonal, row i at i(i+1)/2
  double* part = Xp + kSB * (kSB + 1) / 2;        // second-half partial sums
  const int2 e = sbl[blockIdx.x];
  const SnDev d = sn[e.x];
  const int m = d.m;
  const int b = e.y * kSB, bs = min(kSB, d.k - b);
  const F* P = panels + d.panel_off;
  const signed char* pv = piv + d.first;
  for (int idx = threadIdx.x; idx < bs * bs; idx += blockDim.x) {
    const int j = idx / bs, i = idx % bs;
    if (i > j) Lp[i * (i - 1) / 2 + j] = (j + 1 == i && pv[b + j] == 2) ? 0.0 : P[(b + i) + static_cast<std::int64_t>(b + j) * m];
  }
  __syncthreads();
  const int c = threadIdx.x & (kSB - 1), h = threadIdx.x / kSB;
  for (int i = 0; i < bs; ++i) {
    double acc = 0.0;
    const double* Li = Lp + i * (i - 1) / 2;
    for (int j = h; j < i; j += 2)
      if (j >= c) acc = fma(Li[j], Xp[j * (j + 1) / 2 + c], acc);
    if (h == 1) part[c] = acc;
    __syncthreads();
    if (h == 0 && c <= i) Xp[i * (i + 1) / 2 + c] = c == i ? 1.0 : -(acc + part[c]);
    __syncthreads();
  }
  F* Wd = W + d.w_off + b + static_cast<std::int64_t>(b) * m;
  for (int idx = threadIdx.x; idx < bs * bs; idx += blockDim.x) {
    const int cc = idx / bs, i = idx % bs;
    Wd[i + static_cast<std::int64_t>(cc) * m] = static_cast<F>(i >= cc ? Xp[i * (i + 1) / 2 + cc] : 0.0);
  }
}

// W[r0 : r0 + 64, B] = L[r0 : r0 + 64, B] W[B, B] for one 64-row tile below a super-block per CTA.
template <class F>
__global__ void __launch_bounds__(256) k_sb_apply(const int4* tiles, const SnDev* sn, const F* panels,
                                                   const signed char* piv, F* W) {
  __shared__ double Ls[32][64];
  __shared__ double Xs[32][kSB];
  const int4 e = tiles[blockIdx.x];
  const SnDev d = sn[e.x];
  const int m = d.m;
  const int b = e.y * kSB, bs = min(kSB, d.k - b), r0 = e.z;
  const F* P = panels + d.panel_off;
  const signed char* pv = piv + d.first;
  F* Wf = W + d.w_off;
  const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;  // rows tr + 16 q, columns tc * 8 + p
  double acc[4][8];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int p = 0; p < 8; ++p) acc[q][p] = 0.0;
  for (int j0 = 0; j0 < bs; j0 += 32) {
    for (int idx = threadIdx.x; idx < 32 * 64; idx += blockDim.x) {
      const int jj = idx / 64, row = idx % 64, i = r0 + row, j = j0 + jj;
      // a 2 x 2 pivot split by the super-block boundary: its coupling entry is D, not L
      const bool coupling = i == b + j + 1 && pv[b + j] == 2;
      Ls[jj][row] = (i < m && j < bs && !coupling) ? P[i + static_cast<std::int64_t>(b + j) * m] : 0.0;
    }
    for (int idx = threadIdx.x; idx < 32 * kSB; idx += blockDim.x) {
      const int cc = idx / 32, jj = idx % 32, j = j0 + jj;
      Xs[jj][cc] = (j < bs && cc < bs) ? Wf[(b + j) + static_cast<std::int64_t>(b + cc) * m] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int jj = 0; jj < 32; ++jj) {
      double a[4], x[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) a[q] = Ls[jj][tr + 16 * q];
#pragma unroll
      for (int p = 0; p < 8; ++p) x[p] = Xs[jj][tc * 8 + p];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int p = 0; p < 8; ++p) acc[q][p] = fma(a[q], x[p], acc[q][p]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = r0 + tr + 16 * q;
    if (i >= m) continue;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int cc = tc * 8 + p;
      if (cc < bs) Wf[i + static_cast<std::int64_t>(b + cc) * m] = static_cast<F>(acc[q][p]);
    }
  }
}

namespace {

constexpr long long kSweepSpinLimit = 1LL << 22;
constexpr int kTilePitch = 33;  // padded column pitch of a 32 x 32 W tile in shared memory
constexpr int kRowPitch = 9;    // padded row pitch of a tile's right-hand sides
constexpr int kWarpSmem = 32 * kTilePitch + 32 * kRowPitch;
// backward sweep: one W tile and its right-hand-side rows per warp, then the step buffer
constexpr std::size_t kBwdSmemBytes = sizeof(double) * (8 * kWarpSmem + kSB * 8);

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// thread 0 polls until *cnt >= target, then the whole CTA proceeds. The wait gives up, setting
// *err, after kSweepSpinLimit polls or as soon as another wait has given up (the solve is then
// reported invalid by the host).
__device__ __forceinline__ void wait_count(const int* cnt, int target, int* err) {
  if (threadIdx.x == 0) {
    long long it = 0;
    while (ld_acquire(cnt) < target) {
      ++it;
      if (it > kSweepSpinLimit || ((it & 255) == 0 && *reinterpret_cast<volatile int*>(err) != 0)) {
        atomicExch(err, 1);
        break;
      }
      __nanosleep(32);
    }
  }
  __syncthreads();
}

// thread 0, after a block barrier that orders the CTA's writes before it: add `count` to a counter
// with release semantics (an acq_rel fence at device scope, then a relaxed reduction), so that a CTA
// whose acquire load sees the new count also sees those writes
__device__ __forceinline__ void add_release(int* cnt, int count) {
  asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.s32 [%0], %1;" :: "l"(cnt), "r"(count) : "memory");
}

// all threads, after their writes: make them visible to the front's other CTAs and add `count` to
// the front's counter. A front solved by one CTA only synchronizes its threads.
__device__ __forceinline__ void publish(int* cnt, int count, int nr) {
  __syncthreads();
  if (nr > 1 && threadIdx.x == 0 && count > 0) add_release(cnt, count);
}

// groups / chunks g belong to CTA g mod nr: how many of `rank`'s lie below `hi`
__device__ __forceinline__ int owned_below(int hi, int rank, int nr) { return hi > rank ? (hi - rank + nr - 1) / nr : 0; }

// 32-row groups (32-column chunks) of super-block q of a front with k pivots
__device__ __forceinline__ int sb_groups(int q, int k) {
  const int bs = min(kSB, k - q * kSB);
  return (bs + 31) / 32;
}

}  // namespace

// Forward sweep of one level. t (the front's rows, t[i * 8 + r]) lives in the work array.
// Assembly: each owned row gathers its pivot entry of x and its children's contributions (listed per
// front position in child order: cptr / cent). Step q: the owned groups at or below super-block q
// form their rows of W[:, B] t_B - one warp per group when the CTA has at least four groups, else the
// eight warps share each group's columns and add their partial sums in warp order. Rows of B give
// z_B (written to x), rows below update t, and at the last step the contribution rows go to the
// front's contribution vector.
template <class F>
__global__ void __launch_bounds__(256, 2) k_fwd_level(const SolveTask* tasks, const SnDev* sn, const std::int32_t* cptr,
                                                       const ContribEntry* cent, const F* W,
                                                       const std::int32_t* pidx, double* x, std::int64_t n,
                                                       double* vec, SweepChunks ck, double* work, int* cnts, int* err) {
  __shared__ double tb[kSB * 8];
  __shared__ double red[8][32][9];
  const int nrhs = min(8, ck.ncols - 8 * static_cast<int>(blockIdx.y));
  x += blockIdx.y * ck.x_stride;
  vec += blockIdx.y * ck.vec_stride;
  work += blockIdx.y * ck.work_stride;
  cnts += blockIdx.y * ck.cnt_stride;
  const SolveTask tk = tasks[blockIdx.x];
  const SnDev d = sn[tk.s];
  const int m = d.m, k = d.k, c = m - k, rank = tk.rank, nr = tk.nr;
  double* t = work + tk.wofs;
  int* cnt = cnts + tk.s;
  const F* Wf = W + d.w_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* cp = cptr + d.cptr_off;
  double* v = vec + d.vec_off * nrhs;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nsb = (k + kSB - 1) / kSB, ngt = (m + 31) / 32;
  const int nown = owned_below(ngt, rank, nr);
  for (int idx = threadIdx.x; idx < nown * 32; idx += blockDim.x) {
    const int i = (rank + (idx >> 5) * nr) * 32 + (idx & 31);
    if (i >= m) continue;
    const int pos = i < k ? pl[i] : i;
    double val[8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
      val[r] = (i < k && r < nrhs) ? x[d.first + pos + static_cast<std::int64_t>(r) * n] : 0.0;
    const int e1 = cp[pos + 1];
    for (int e = cp[pos]; e < e1; ++e) {
      const ContribEntry ce = cent[e];
      const double* src = vec + ce.vec_off * nrhs + ce.a;
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < nrhs) val[r] += src[static_cast<std::int64_t>(r) * ce.mc];
    }
    if (nsb == 0) {  // no pivots: the rows pass to the parent unchanged
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < nrhs) v[(i - k) + static_cast<std::int64_t>(r) * c] = val[r];
    } else {
#pragma unroll
      for (int r = 0; r < 8; ++r) t[static_cast<std::int64_t>(i) * 8 + r] = val[r];
    }
  }
  if (nsb == 0) return;
  publish(cnt, owned_below(sb_groups(0, k), rank, nr), nr);
  int target = 0;
  for (int q = 0; q < nsb; ++q) {
    const int b = q * kSB, be = min(b + kSB, k), bs = be - b;
    target += sb_groups(q, k);
    const int g0 = owned_below(b / 32, rank, nr);
    const int ng = nown - g0;  // owned groups at or below super-block q (uniform over the CTA)
    if (ng <= 0) break;
    const bool last = q + 1 == nsb;
    const int nb0 = (q + 1) * (kSB / 32), nb1 = last ? nb0 : nb0 + sb_groups(q + 1, k);
    if (nr > 1) wait_count(cnt, target, err);
    for (int idx = threadIdx.x; idx < kSB * 8; idx += blockDim.x) {
      const int j = idx >> 3;
      tb[idx] = j < bs ? __ldcg(&t[static_cast<std::int64_t>(b + j) * 8 + (idx & 7)]) : 0.0;
    }
    __syncthreads();
    if (ng >= 4) {
      for (int gi = warp; gi < ng; gi += 8) {
        const int i = (rank + (g0 + gi) * nr) * 32 + lane;
        if (i >= m) continue;
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const F* Wi = Wf + i + static_cast<std::int64_t>(b) * m;
        // 16-column batches; the next batch's loads are issued before this one is summed
        double wv[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) wv[u] = u < bs ? static_cast<double>(Wi[static_cast<std::int64_t>(u) * m]) : 0.0;
        for (int j0 = 0; j0 < bs; j0 += 16) {
          double wn[16];
#pragma unroll
          for (int u = 0; u < 16; ++u)
            wn[u] = j0 + 16 + u < bs ? static_cast<double>(Wi[static_cast<std::int64_t>(j0 + 16 + u) * m]) : 0.0;
#pragma unroll
          for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int r = 0; r < 8; ++r) acc[r] = fma(wv[u], tb[(j0 + u) * 8 + r], acc[r]);
#pragma unroll
          for (int u = 0; u < 16; ++u) wv[u] = wn[u];
        }
        double* ti = t + static_cast<std::int64_t>(i) * 8;
        if (i < be) {
#pragma unroll
          for (int r = 0; r < 8; ++r)
            if (r < nrhs) x[d.first + pl[i] + static_cast<std::int64_t>(r) * n] = acc[r];
        } else if (last && i >= k) {
#pragma unroll
          for (int r = 0; r < 8; ++r)
            if (r < nrhs) v[(i - k) + static_cast<std::int64_t>(r) * c] = __ldcg(&ti[r]) - acc[r];
        } else {
#pragma unroll
          for (int r = 0; r < 8; ++r) ti[r] = __ldcg(&ti[r]) - acc[r];
        }
      }
    } else {
      const int j0 = warp * 16;
      for (int gi = 0; gi < ng; ++gi) {
        const int G = rank + (g0 + gi) * nr;
        const int i = G * 32 + lane;
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (i < m) {
          double wv[16];
#pragma unroll
          for (int u = 0; u < 16; ++u)
            wv[u] = j0 + u < bs ? static_cast<double>(Wf[i + static_cast<std::int64_t>(b + j0 + u) * m]) : 0.0;
#pragma unroll
          for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int r = 0; r < 8; ++r) acc[r] = fma(wv[u], tb[(j0 + u) * 8 + r], acc[r]);
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) red[warp][lane][r] = acc[r];
        __syncthreads();
        {
          const int row = threadIdx.x >> 3, rr = threadIdx.x & 7;
          const int ii = G * 32 + row;
          if (ii < m) {
            double val = 0.0;
#pragma unroll
            for (int w = 0; w < 8; ++w) val += red[w][row][rr];
            double* tr = t + static_cast<std::int64_t>(ii) * 8 + rr;
            if (ii < be) {
              if (rr < nrhs) x[d.first + pl[ii] + static_cast<std::int64_t>(rr) * n] = val;
            } else if (last && ii >= k) {
              if (rr < nrhs) v[(ii - k) + static_cast<std::int64_t>(rr) * c] = __ldcg(tr) - val;
            } else {
              *tr = __ldcg(tr) - val;
            }
          }
        }
        __syncthreads();
      }
    }
    publish(cnt, owned_below(nb1, rank, nr) - owned_below(nb0, rank, nr), nr);
  }
}

// Backward sweep of one level. sv (s_j, sv[j * 8 + r]) and ta (the front's pivot rows of x on entry,
// ta[i * 8 + r]) live in the work array. (1) Each CTA copies the pivot rows of its chunks to ta; once
// every CTA of the front has done so, the front's pivot rows of x are only written (final values).
// (2) For each owned chunk, s_j over rows A and CB: 32 x 32 tiles of W, one tile per warp at a time,
// staged in shared memory so that lane c forms column c's sums (no shuffles), warps added in order.
// (3) From the last super-block down: the owners of the columns below super-block B apply x_B; the
// owners of the next super-block's columns write their final x and publish.
template <class F>
__global__ void __launch_bounds__(256, 2) k_bwd_level(const SolveTask* tasks, const SnDev* sn, const std::int32_t* rows,
                                                       const F* W, const std::int32_t* pidx, double* x,
                                                       std::int64_t n, SweepChunks ck, double* work, int* cnts,
                                                       int* arrive, int* hcnts, int* err) {
  extern __shared__ double dsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* wt = dsm + warp * kWarpSmem;     // wt[c * kTilePitch + i]: W[i0 + i, j0 + c]
  double* tt = wt + 32 * kTilePitch;       // tt[i * kRowPitch + r]: the tile's rows, signed
  double* xb = dsm + 8 * kWarpSmem;        // xb[r * kSB + i]: x of the super-block being applied
  double* red = dsm;                       // [8][32][9] partial sums, over the tiles once they are used
  const int nrhs = min(8, ck.ncols - 8 * static_cast<int>(blockIdx.y));
  x += blockIdx.y * ck.x_stride;
  work += blockIdx.y * ck.work_stride;
  cnts += blockIdx.y * ck.cnt_stride;
  arrive += blockIdx.y * ck.cnt_stride;
  const SolveTask tk = tasks[blockIdx.x];
  const SnDev d = sn[tk.s];
  const int m = d.m, k = d.k, rank = tk.rank, nr = tk.nr, P = tk.parts;
  if (k == 0) return;
  double* sv = work + tk.wofs;
  double* ta = sv + static_cast<std::int64_t>(k) * 8;
  double* partial = ta + static_cast<std::int64_t>(k) * 8;  // [chunk][part - 1][32 columns][8]
  int* cnt = cnts + tk.s;
  int* hc = hcnts + blockIdx.y * ck.cnt_stride + tk.hcnt;  // per chunk: helper parts published
  const F* Wf = W + d.w_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* rw = rows + d.rows_off;
  const int nsb = (k + kSB - 1) / kSB, nch = (k + 31) / 32;
  const int t2 = (m - k + 31) / 32;  // contribution-row tiles of a chunk
  // the warp's share of ntl tiles of chunk j0: tiles tau < t1o are rows [bA, beA) of the chunk's
  // super-block (entry values from ta, sign +), the others contribution-row tiles cb0 + (tau - t1o)
  // (x of the ancestors, sign -); every tile is staged in shared memory so that lane c sums column c
  auto sum_tiles = [&](int j0, int t1o, int bA, int beA, int cb0, int ntl, double* acc) {
    for (int tau = warp; tau < ntl; tau += 8) {
      const bool own = tau < t1o;
      const int i = (own ? bA + 32 * tau : k + 32 * (cb0 + tau - t1o)) + lane;
      const bool ok = i < (own ? beA : m);
      const F* Wi = Wf + i + static_cast<std::int64_t>(j0) * m;
      double wv[32];
#pragma unroll
      for (int cc = 0; cc < 32; ++cc)
        wv[cc] = (ok && j0 + cc < k) ? static_cast<double>(Wi[static_cast<std::int64_t>(cc) * m]) : 0.0;
      double rv[8];
      if (ok && own) {
        const double* ti = ta + static_cast<std::int64_t>(i) * 8;
#pragma unroll
        for (int r = 0; r < 8; ++r) rv[r] = __ldcg(&ti[r]);
      } else if (ok) {
        const std::int64_t g = rw[i];
#pragma unroll
        for (int r = 0; r < 8; ++r) rv[r] = r < nrhs ? -x[g + static_cast<std::int64_t>(r) * n] : 0.0;
      } else {
#pragma unroll
        for (int r = 0; r < 8; ++r) rv[r] = 0.0;
      }
#pragma unroll
      for (int cc = 0; cc < 32; ++cc) wt[cc * kTilePitch + lane] = wv[cc];
#pragma unroll
      for (int r = 0; r < 8; ++r) tt[lane * kRowPitch + r] = rv[r];
      __syncwarp();
#pragma unroll 8
      for (int ii = 0; ii < 32; ++ii) {
        const double w = wt[lane * kTilePitch + ii];
#pragma unroll
        for (int r = 0; r < 8; ++r) acc[r] = fma(w, tt[ii * kRowPitch + r], acc[r]);
      }
      __syncwarp();
    }
  };
  if (rank >= nr) {
    // helper: part q of chunk ch's contribution-row tiles; its sum goes to the chunk's partials
    // (it reads only W and the ancestors' final x, so it waits for nothing)
    const int h = rank - nr, ch = h % nch, q = 1 + h / nch;
    const int lo = (q * t2) / P, hi = ((q + 1) * t2) / P;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    sum_tiles(ch * 32, 0, 0, 0, lo, hi - lo, acc);
    __syncthreads();  // red overlays the tiles
#pragma unroll
    for (int r = 0; r < 8; ++r) red[(warp * 32 + lane) * 9 + r] = acc[r];
    __syncthreads();
    {
      const int cc = threadIdx.x >> 3, r = threadIdx.x & 7;
      double sum = 0.0;
#pragma unroll
      for (int w = 0; w < 8; ++w) sum += red[(w * 32 + cc) * 9 + r];
      partial[(static_cast<std::int64_t>(ch) * (P - 1) + (q - 1)) * 256 + cc * 8 + r] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) add_release(hc + ch, 1);
    return;
  }
  const int nown = owned_below(nch, rank, nr);
  for (int idx = threadIdx.x; idx < nown * 32; idx += blockDim.x) {
    const int i = (rank + (idx >> 5) * nr) * 32 + (idx & 31);
    if (i >= k) continue;
#pragma unroll
    for (int r = 0; r < 8; ++r)
      ta[static_cast<std::int64_t>(i) * 8 + r] = r < nrhs ? x[d.first + pl[i] + static_cast<std::int64_t>(r) * n] : 0.0;
  }
  if (nr > 1) {
    publish(arrive + tk.s, 1, nr);
    wait_count(arrive + tk.s, nr, err);
  } else {
    __syncthreads();
  }
  const int lastb = (nsb - 1) * kSB;
  for (int u = 0; u < nown; ++u) {
    const int ch = rank + u * nr, j0 = ch * 32;
    const int bA = (j0 / kSB) * kSB, beA = min(bA + kSB, k);
    const int t1 = (beA - bA + 31) / 32;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    sum_tiles(j0, t1, bA, beA, 0, t1 + t2 / P, acc);  // the super-block's rows and part 0
    __syncthreads();  // every warp is done with its tiles: red overlays them
#pragma unroll
    for (int r = 0; r < 8; ++r) red[(warp * 32 + lane) * 9 + r] = acc[r];
    __syncthreads();
    if (P > 1) wait_count(hc + ch, P - 1, err);  // the helpers' parts of this chunk
    const bool fin = bA == lastb;  // the last super-block: s is x
    {
      const int cc = threadIdx.x >> 3, r = threadIdx.x & 7, j = j0 + cc;
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < 8; ++w) s += red[(w * 32 + cc) * 9 + r];
      for (int q = 1; q < P; ++q) s += __ldcg(&partial[(static_cast<std::int64_t>(ch) * (P - 1) + (q - 1)) * 256 + cc * 8 + r]);
      if (j < k) {
        sv[static_cast<std::int64_t>(j) * 8 + r] = s;
        if (fin && r < nrhs) x[d.first + pl[j] + static_cast<std::int64_t>(r) * n] = s;
      }
    }
    publish(cnt, fin ? 1 : 0, nr);
  }
  int target = 0;
  const int sub = threadIdx.x & 7, col = threadIdx.x >> 3;  // 8 lanes per column, 32 columns per chunk
  for (int q = nsb - 1; q >= 1; --q) {
    const int b = q * kSB, bs = min(kSB, k - b);
    target += sb_groups(q, k);
    const int nlow = owned_below(b / 32, rank, nr);
    if (nlow == 0) break;  // uniform over the CTA
    // the first chunk's W entries and old values do not depend on the wait
    int u = nlow - 1;
    int j = (rank + u * nr) * 32 + col;
    double wv[16];
    {
      const F* Wj = Wf + b + static_cast<std::int64_t>(j) * m;
#pragma unroll
      for (int e = 0; e < 16; ++e) wv[e] = sub + 8 * e < bs ? static_cast<double>(Wj[sub + 8 * e]) : 0.0;
    }
    if (nr > 1) wait_count(cnt, target, err);
    for (int idx = threadIdx.x; idx < kSB * 8; idx += blockDim.x) {
      const int r = idx / kSB, i = idx % kSB;
      xb[idx] = i < bs ? __ldcg(&sv[static_cast<std::int64_t>(b + i) * 8 + r]) : 0.0;
    }
    __syncthreads();
    for (;;) {
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int e = 0; e < 16; ++e)
#pragma unroll
        for (int r = 0; r < 8; ++r) acc[r] = fma(wv[e], xb[r * kSB + sub + 8 * e], acc[r]);
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 4);
        acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 2);
        acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 1);
      }
      double a = acc[0];
#pragma unroll
      for (int r = 1; r < 8; ++r)
        if (sub == r) a = acc[r];
      double* sj = sv + static_cast<std::int64_t>(j) * 8 + sub;
      const double nv = __ldcg(sj) - a;
      *sj = nv;
      const bool next = j - col >= b - kSB;  // the chunk lies in super-block q - 1: final now
      if (next) {
        if (sub < nrhs) x[d.first + pl[j] + static_cast<std::int64_t>(sub) * n] = nv;
        publish(cnt, 1, nr);
      }
      if (--u < 0) break;
      j = (rank + u * nr) * 32 + col;
      const F* Wj = Wf + b + static_cast<std::int64_t>(j) * m;
#pragma unroll
      for (int e = 0; e < 16; ++e) wv[e] = sub + 8 * e < bs ? static_cast<double>(Wj[sub + 8 * e]) : 0.0;
    }
    __syncthreads();  // xb is rewritten by the next step
  }
}


// Levels of tiny fronts (m <= kTinyRows, k <= 32: one super-block, no chain): one warp per front,
// eight fronts per CTA, no block barrier. Forward: lane owns rows lane, lane + 32, lane + 64; the pivot
// rows' assembled values go to shared memory for z = W[B, B] t_B and the contribution rows' updates.
// Backward: the front's rows of x (pivot rows' entry values, minus the contribution rows) are staged in
// shared memory and lane j < k forms x_j = W[:, j]^T of them, reading its own column of W.
template <class F>
__global__ void __launch_bounds__(256) k_fwd_tiny(const SolveTask* tasks, int ntasks, const SnDev* sn,
                                                   const std::int32_t* cptr, const ContribEntry* cent, const F* W,
                                                   const std::int32_t* pidx, double* x, std::int64_t n, double* vec,
                                                   SweepChunks ck) {
  __shared__ double tbs[8][32][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ti = blockIdx.x * 8 + warp;
  if (ti >= ntasks) return;  // the whole warp: no block barrier follows
  const int nrhs = min(8, ck.ncols - 8 * static_cast<int>(blockIdx.y));
  x += blockIdx.y * ck.x_stride;
  vec += blockIdx.y * ck.vec_stride;
  const SnDev d = sn[tasks[ti].s];
  const int m = d.m, k = d.k, c = m - k;
  const F* Wf = W + d.w_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* cp = cptr + d.cptr_off;
  double* v = vec + d.vec_off * nrhs;
  double t[kTinyRows / 32][8];
#pragma unroll
  for (int u = 0; u < kTinyRows / 32; ++u) {
    const int i = lane + 32 * u;
#pragma unroll
    for (int r = 0; r < 8; ++r) t[u][r] = 0.0;
    if (i >= m) continue;
    const int pos = i < k ? pl[i] : i;
    if (i < k) {
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < nrhs) t[u][r] = x[d.first + pos + static_cast<std::int64_t>(r) * n];
    }
    const int e1 = cp[pos + 1];
    for (int e = cp[pos]; e < e1; ++e) {
      const ContribEntry ce = cent[e];
      const double* src = vec + ce.vec_off * nrhs + ce.a;
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < nrhs) t[u][r] += src[static_cast<std::int64_t>(r) * ce.mc];
    }
  }
  if (lane < k) {
#pragma unroll
    for (int r = 0; r < 8; ++r) tbs[warp][lane][r] = t[0][r];
  }
  __syncwarp();
#pragma unroll
  for (int u = 0; u < kTinyRows / 32; ++u) {
    const int i = lane + 32 * u;
    if (i >= m) continue;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 0; j < k; ++j) {
      const double w = static_cast<double>(Wf[i + static_cast<std::int64_t>(j) * m]);
#pragma unroll
      for (int r = 0; r < 8; ++r) acc[r] = fma(w, tbs[warp][j][r], acc[r]);
    }
    if (i < k) {
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < nrhs) x[d.first + pl[i] + static_cast<std::int64_t>(r) * n] = acc[r];
    } else {
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < nrhs) v[(i - k) + static_cast<std::int64_t>(r) * c] = t[u][r] - acc[r];
    }
  }
}

template <class F>
__global__ void __launch_bounds__(256) k_bwd_tiny(const SolveTask* tasks, int ntasks, const SnDev* sn,
                                                   const std::int32_t* rows, const F* W, const std::int32_t* pidx,
                                                   double* x, std::int64_t n, SweepChunks ck) {
  __shared__ double xs[8][kTinyRows][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ti = blockIdx.x * 8 + warp;
  if (ti >= ntasks) return;  // the whole warp: no block barrier follows
  const int nrhs = min(8, ck.ncols - 8 * static_cast<int>(blockIdx.y));
  x += blockIdx.y * ck.x_stride;
  const SnDev d = sn[tasks[ti].s];
  const int m = d.m, k = d.k;
  if (k == 0) return;
  const F* Wf = W + d.w_off;
  const std::int32_t* pl = pidx + d.first;
  const std::int32_t* rw = rows + d.rows_off;
#pragma unroll
  for (int u = 0; u < kTinyRows / 32; ++u) {
    const int i = lane + 32 * u;
    if (i >= m) continue;
    const std::int64_t g = i < k ? d.first + pl[i] : rw[i];
    const double sg = i < k ? 1.0 : -1.0;
#pragma unroll
    for (int r = 0; r < 8; ++r) xs[warp][i][r] = r < nrhs ? sg * x[g + static_cast<std::int64_t>(r) * n] : 0.0;
  }
  __syncwarp();
  if (lane < k) {
    const F* Wj = Wf + static_cast<std::int64_t>(lane) * m;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = lane; i < m; ++i) {  // W[i, j] = 0 above the diagonal
      const double w = static_cast<double>(Wj[i]);
#pragma unroll
      for (int r = 0; r < 8; ++r) acc[r] = fma(w, xs[warp][i][r], acc[r]);
    }
#pragma unroll
    for (int r = 0; r < 8; ++r)
      if (r < nrhs) x[d.first + pl[lane] + static_cast<std::int64_t>(r) * n] = acc[r];
  }
}

void launch_gather_scale(std::int64_t n, int nrhs, const double* b, std::int64_t ldb, const double* d,
                         const std::int32_t* iperm, double* x, cudaStream_t s) {
  const std::int64_t total = n * nrhs;
  const int blocks = static_cast<int>(std::min<std::int64_t>((total + 255) / 256, 148 * 16));
  note_launches(1);
  k_gather_scale<<<blocks, 256, 0, s>>>(n, nrhs, b, ldb, d, iperm, x);
}

void launch_scatter_scale(std::int64_t n, int nrhs, double* b, std::int64_t ldb, const double* d,
                          const std::int32_t* iperm, const double* x, cudaStream_t s) {
  const std::int64_t total = n * nrhs;
  const int blocks = static_cast<int>(std::min<std::int64_t>((total + 255) / 256, 148 * 16));
  note_launches(1);
  k_scatter_scale<<<blocks, 256, 0, s>>>(n, nrhs, b, ldb, d, iperm, x);
}

template <class F>
void launch_solve_diag_flat(std::int64_t npiv, const std::int64_t* dpos, const std::int32_t* pfirst, const F* panels,
                            const signed char* piv, const std::int32_t* pidx, double* x, std::int64_t n, int nrhs,
                            cudaStream_t s) {
  if (npiv <= 0) return;
  note_launches(1);
  k_solve_diag_flat<F><<<static_cast<unsigned>((npiv + 255) / 256), 256, 0, s>>>(npiv, dpos, pfirst, panels, piv, pidx,
                                                                                x, n, nrhs);
}

namespace {
template <class F>
void configure_bwd() {
  static std::once_flag configured;
  std::call_once(configured, [] {
    cudaFuncSetAttribute(k_bwd_level<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kBwdSmemBytes));
  });
}

template <class F>
int solve_coop_max_of(int device) {
  configure_bwd<F>();
  int a = 0, b = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_fwd_level<F>, 256, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_bwd_level<F>, 256, kBwdSmemBytes);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return (a < b ? a : b) * sms;
}
}  // namespace

// co-resident CTAs of the sweep kernels, valid for both factor types
int solve_coop_max_ctas(int device) {
  const int a = solve_coop_max_of<double>(device), b = solve_coop_max_of<float>(device);
  return a < b ? a : b;
}

template <class F>
void launch_sb_build(const int2* sbl, int nsb, const int4* tiles, int ntiles, const SnDev* sn, const F* panels,
                     const signed char* piv, F* W, cudaStream_t s) {
  if (nsb <= 0) return;
  constexpr std::size_t smem = sizeof(double) * (kSB * (kSB - 1) / 2 + kSB * (kSB + 1) / 2 + kSB);
  static std::once_flag configured;
  std::call_once(configured, [&] {
    cudaFuncSetAttribute(k_sb_inverse<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  });
  note_launches(1);
  k_sb_inverse<F><<<nsb, 256, smem, s>>>(sbl, sn, panels, piv, W);
  if (ntiles > 0) {
    note_launches(1);
    k_sb_apply<F><<<ntiles, 256, 0, s>>>(tiles, sn, panels, piv, W);
  }
}

template <class F>
cudaError_t launch_fwd_level(const SolveTask* tasks, int nctas, bool coop, const SnDev* sn, const std::int32_t* cptr,
                             const ContribEntry* cent, const F* W, const std::int32_t* pidx, double* x, std::int64_t n,
                             double* vec, const SweepChunks& ck, double* work, int* cnts, int* err, cudaStream_t s) {
  if (nctas <= 0 || ck.ncols <= 0) return cudaSuccess;
  const dim3 grid(nctas, (ck.ncols + 7) / 8);
  SweepChunks c = ck;
  note_launches(1);
  if (!coop) {
    k_fwd_level<F><<<grid, 256, 0, s>>>(tasks, sn, cptr, cent, W, pidx, x, n, vec, c, work, cnts, err);
    return cudaGetLastError();
  }
  void* args[] = {&tasks, &sn, &cptr, &cent, &W, &pidx, &x, &n, &vec, &c, &work, &cnts, &err};
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_fwd_level<F>), grid, dim3(256), args, 0, s);
}

template <class F>
cudaError_t launch_bwd_level(const SolveTask* tasks, int nctas, bool coop, const SnDev* sn, const std::int32_t* rows,
                             const F* W, const std::int32_t* pidx, double* x, std::int64_t n, const SweepChunks& ck,
                             double* work, int* cnts, int* arrive, int* hcnts, int* err, cudaStream_t s) {
  if (nctas <= 0 || ck.ncols <= 0) return cudaSuccess;
  configure_bwd<F>();
  const dim3 grid(nctas, (ck.ncols + 7) / 8);
  SweepChunks c = ck;
  note_launches(1);
  if (!coop) {
    k_bwd_level<F><<<grid, 256, kBwdSmemBytes, s>>>(tasks, sn, rows, W, pidx, x, n, c, work, cnts, arrive, hcnts, err);
    return cudaGetLastError();
  }
  void* args[] = {&tasks, &sn, &rows, &W, &pidx, &x, &n, &c, &work, &cnts, &arrive, &hcnts, &err};
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_bwd_level<F>), grid, dim3(256), args, kBwdSmemBytes,
                                     s);
}

template <class F>
cudaError_t launch_fwd_tiny(const SolveTask* tasks, int ntasks, const SnDev* sn, const std::int32_t* cptr,
                            const ContribEntry* cent, const F* W, const std::int32_t* pidx, double* x, std::int64_t n,
                            double* vec, const SweepChunks& ck, cudaStream_t s) {
  if (ntasks <= 0 || ck.ncols <= 0) return cudaSuccess;
  note_launches(1);
  k_fwd_tiny<F><<<dim3((ntasks + 7) / 8, (ck.ncols + 7) / 8), 256, 0, s>>>(tasks, ntasks, sn, cptr, cent, W, pidx, x,
                                                                          n, vec, ck);
  return cudaGetLastError();
}

template <class F>
cudaError_t launch_bwd_tiny(const SolveTask* tasks, int ntasks, const SnDev* sn, const std::int32_t* rows, const F* W,
                            const std::int32_t* pidx, double* x, std::int64_t n, const SweepChunks& ck, cudaStream_t s) {
  if (ntasks <= 0 || ck.ncols <= 0) return cudaSuccess;
  note_launches(1);
  k_bwd_tiny<F><<<dim3((ntasks + 7) / 8, (ck.ncols + 7) / 8), 256, 0, s>>>(tasks, ntasks, sn, rows, W, pidx, x, n, ck);
  return cudaGetLastError();
}

#define HSG_SOLVE_INSTANTIATE(F)                                                                                       \
  template void launch_solve_diag_flat<F>(std::int64_t, const std::int64_t*, const std::int32_t*, const F*,          \
                                          const signed char*, const std::int32_t*, double*, std::int64_t, int,        \
                                          cudaStream_t);                                                               \
  template void launch_sb_build<F>(const int2*, int, const int4*, int, const SnDev*, const F*, const signed char*,    \
                                   F*, cudaStream_t);                                                                  \
  template cudaError_t launch_fwd_level<F>(const SolveTask*, int, bool, const SnDev*, const std::int32_t*,           \
                                           const ContribEntry*, const F*, const std::int32_t*, double*, std::int64_t,  \
                                           double*, const SweepChunks&, double*, int*, int*, cudaStream_t);            \
  template cudaError_t launch_bwd_level<F>(const SolveTask*, int, bool, const SnDev*, const std::int32_t*, const F*, \
                                           const std::int32_t*, double*, std::int64_t, const SweepChunks&, double*,    \
                                           int*, int*, int*, int*, cudaStream_t);                                      \
  template cudaError_t launch_fwd_tiny<F>(const SolveTask*, int, const SnDev*, const std::int32_t*,                  \
                                          const ContribEntry*, const F*, const std::int32_t*, double*, std::int64_t,   \
                                          double*, const SweepChunks&, cudaStream_t);                                  \
  template cudaError_t launch_bwd_tiny<F>(const SolveTask*, int, const SnDev*, const std::int32_t*, const F*,        \
                                          const std::int32_t*, double*, std::int64_t, const SweepChunks&, cudaStream_t);
HSG_SOLVE_INSTANTIATE(double)
HSG_SOLVE_INSTANTIATE(float)
#undef HSG_SOLVE_INSTANTIATE

}  // namespace hsg
