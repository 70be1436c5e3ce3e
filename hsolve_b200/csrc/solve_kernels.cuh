// Launchers of the solve kernels (solve_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device.cuh"

namespace hsg {

void launch_gather_scale(std::int64_t n, int nrhs, const double* b, std::int64_t ldb, const double* d,
                         const std::int32_t* iperm, double* x, cudaStream_t s);
void launch_scatter_scale(std::int64_t n, int nrhs, double* b, std::int64_t ldb, const double* d,
                          const std::int32_t* iperm, const double* x, cudaStream_t s);

// The kernels below that read the factor are instantiated for F = double (FP64 factors) and
// F = float (FP32 factors of the mixed-precision operator); right-hand sides, contribution vectors
// and all accumulation stay in FP64 either way.

// D y = z for all pivots, one thread each (dpos: panel index of each D(p, p); pfirst: front's first column)
template <class F>
void launch_solve_diag_flat(std::int64_t npiv, const std::int64_t* dpos, const std::int32_t* pfirst, const F* panels,
                            const signed char* piv, const std::int32_t* pidx, double* x, std::int64_t n, int nrhs,
                            cudaStream_t s);

// Super-blocks of kSB pivots per front; their solve operator W (L_BB^{-1} on the diagonal block,
// L L_BB^{-1} below it) is built once per factorization by launch_sb_build.
constexpr int kSB = 128;
// sbl: (front, super-block) pairs; tiles: (front, super-block, first row) of the 64-row tiles below
template <class F>
void launch_sb_build(const int2* sbl, int nsb, const int4* tiles, int ntiles, const SnDev* sn, const F* panels,
                     const signed char* piv, F* W, cudaStream_t s);
// co-resident CTAs of the sweep kernels (the bound of a cooperative level launch)
int solve_coop_max_ctas(int device);
// One level of the forward / backward sweep: one CTA per task (front, rank, nr, work offset) and
// 8-column chunk of the ck.ncols right-hand sides (grid nctas x chunks); coop: the level has fronts
// of several CTAs (cooperative launch, nctas x chunks <= solve_coop_max_ctas). cnts / arrive: one
// counter per front and chunk, zero at the first launch of a sweep; err: set to 1 when a wait
// between the CTAs of a front ran out (the solve is then invalid); hcnts: backward, one counter per
// 32-column chunk of every front (at SolveTask::hcnt), zero at the first launch. Work per front and
// chunk: 8 m doubles forward, 16 k + 256 nch (parts - 1) backward.
constexpr int kSweepChunks = 2;  // 8-column chunks carried by one sweep launch
// levels whose fronts all have m <= kTinyRows and k <= 32 are solved one warp per front (tasks with
// nr = 1, eight per CTA; ordinary launch)
constexpr int kTinyRows = 96;
template <class F>
cudaError_t launch_fwd_tiny(const SolveTask* tasks, int ntasks, const SnDev* sn, const std::int32_t* cptr,
                            const ContribEntry* cent, const F* W, const std::int32_t* pidx, double* x, std::int64_t n,
                            double* vec, const SweepChunks& ck, cudaStream_t s);
template <class F>
cudaError_t launch_bwd_tiny(const SolveTask* tasks, int ntasks, const SnDev* sn, const std::int32_t* rows, const F* W,
                            const std::int32_t* pidx, double* x, std::int64_t n, const SweepChunks& ck, cudaStream_t s);
template <class F>
cudaError_t launch_fwd_level(const SolveTask* tasks, int nctas, bool coop, const SnDev* sn, const std::int32_t* cptr,
                             const ContribEntry* cent, const F* W, const std::int32_t* pidx, double* x, std::int64_t n,
                             double* vec, const SweepChunks& ck, double* work, int* cnts, int* err, cudaStream_t s);
template <class F>
cudaError_t launch_bwd_level(const SolveTask* tasks, int nctas, bool coop, const SnDev* sn, const std::int32_t* rows,
                             const F* W, const std::int32_t* pidx, double* x, std::int64_t n, const SweepChunks& ck,
                             double* work, int* cnts, int* arrive, int* hcnts, int* err, cudaStream_t s);

}  // namespace hsg
