// Launchers of the solve kernels (solve_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device.cuh"

namespace hsg {

constexpr std::size_t kSolveSmemMax = 200 * 1024;  // dynamic shared memory of a solve CTA

// right-hand sides carried together by one solve CTA of fronts up to maxm rows
int solve_rhs_chunk(int maxm, int nrhs);

void launch_gather_scale(std::int64_t n, int nrhs, const double* b, std::int64_t ldb, const double* d,
                         const std::int32_t* iperm, double* x, cudaStream_t s);
void launch_scatter_scale(std::int64_t n, int nrhs, double* b, std::int64_t ldb, const double* d,
                          const std::int32_t* iperm, const double* x, cudaStream_t s);
constexpr int kMaxBlocksPerFront = 2048;  // <= 32-column solve blocks per front (fronts up to ~63k pivots)

// The kernels below that read the factor are instantiated for F = double (FP64 factors) and
// F = float (FP32 factors of the mixed-precision operator); right-hand sides, contribution vectors
// and all accumulation stay in FP64 either way.

// block partition + inverse diagonal blocks of the fronts solved one CTA per front (before the
// first solve of each factorization)
template <class F>
void launch_inv_blocks(int ns, const SnDev* sn, const F* panels, const signed char* piv, std::int32_t* blk,
                       std::int32_t* nblk, F* inv, cudaStream_t s);
template <class F>
void launch_solve_fwd(const std::int32_t* list, int nlist, int maxm, const SnDev* sn, const std::int32_t* child_ptr,
                      const std::int32_t* children, const std::int32_t* rmap, const F* panels,
                      const signed char* piv, const std::int32_t* pidx, const std::int32_t* blk,
                      const std::int32_t* nblk, const F* inv, double* x, std::int64_t n, double* vec, int nrhs,
                      cudaStream_t s);
// D y = z for all pivots, one thread each (dpos: panel index of each D(p, p); pfirst: front's first column)
template <class F>
void launch_solve_diag_flat(std::int64_t npiv, const std::int64_t* dpos, const std::int32_t* pfirst, const F* panels,
                            const signed char* piv, const std::int32_t* pidx, double* x, std::int64_t n, int nrhs,
                            cudaStream_t s);
template <class F>
void launch_solve_diag(int ns, const SnDev* sn, const F* panels, const signed char* piv, const std::int32_t* pidx,
                       double* x, std::int64_t n, int nrhs, cudaStream_t s);
template <class F>
void launch_solve_bwd(const std::int32_t* list, int nlist, int maxm, const SnDev* sn, const std::int32_t* rows,
                      const F* panels, const std::int32_t* pidx, const std::int32_t* blk, const std::int32_t* nblk,
                      const F* inv, double* x, std::int64_t n, int nrhs, cudaStream_t s);

// cooperative sweeps over the few large fronts of a level (nrhs <= 8 per launch), by super-blocks of
// kSB pivots whose solve operator W (L_BB^{-1} on the diagonal block, L L_BB^{-1} below it) is built
// once per factorization by launch_sb_build
constexpr int kSB = 128;
// sbl: (front, super-block) pairs; tiles: (front, super-block, first row) of the 64-row tiles below
template <class F>
void launch_sb_build(const int2* sbl, int nsb, const int4* tiles, int ntiles, const SnDev* sn, const F* panels,
                     const signed char* piv, F* W, cudaStream_t s);
int solve_coop_max_ctas(int device);
// cnts: one publication counter per front of the launch, zero at launch; err: set to 1 when a
// wait between the CTAs of a front ran out (the solve is then not valid)
template <class F>
cudaError_t launch_solve_fwd_coop(const std::int32_t* list, const std::int32_t* cta_start, int nfronts, int nctas,
                                  const SnDev* sn, const std::int32_t* cptr, const ContribEntry* cent, const F* W,
                                  const std::int32_t* pidx, double* x, std::int64_t n, double* vec, int nrhs,
                                  double* work, const std::int64_t* work_off, int* cnts, int* err, cudaStream_t s);
template <class F>
cudaError_t launch_solve_bwd_coop(const std::int32_t* list, const std::int32_t* cta_start, int nfronts, int nctas,
                                  const SnDev* sn, const std::int32_t* rows, const F* W, const std::int32_t* pidx,
                                  double* x, std::int64_t n, int nrhs, double* work, const std::int64_t* work_off,
                                  int* cnts, int* err, cudaStream_t s);

}  // namespace hsg
