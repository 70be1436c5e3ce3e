// Launchers of the factorization kernels (factor_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device.cuh"

namespace hsg {

constexpr int kSmallMax = 64;          // fronts up to this order are factorized in shared memory
constexpr int kNB = 32;                // panel width of the a-posteriori pivoting kernel
constexpr int kTile = 64;              // trailing-update tile (rows = cols)
constexpr int kKB = 128;               // pending pivots whose trailing update is applied at once (blocked step)
constexpr int kUpdLd = kTile + 4;      // column stride of the staged update operands (conflict-free fragment reads)
constexpr int kAppDynDoubles = 2 * kKB * kUpdLd;  // dynamic shared memory of the panel kernels
constexpr int kRowStage = kNB * kNB + 4 * kNB;   // panel row step: the block's L and the D^-1 coefficients
constexpr int kRowChunk = (kAppDynDoubles - kRowStage) / kNB;  // rows staged at once by the panel row step
constexpr int kAppThreads = 256;
constexpr int kCoopMinFront = 192;     // levels whose largest panel front is at least this use the cooperative kernel
constexpr int kColsPerThread = kTile * kTile / kAppThreads;  // 16
constexpr int kExtendAddCols = 8;      // contribution-block columns per extend-add CTA
// per-front scratch of the panel kernels (doubles): control block, two sets (alternate panels) of
// block, original block, labels, pivot types and column maxima, backup of the panel's rows
constexpr int kAppCtrlDoubles = 8;
constexpr int kAppSlotDoubles = 2 * kNB * kNB + kNB / 2 + kNB / 8 + 2 * kNB;
inline std::int64_t app_scratch_doubles(int m) {
  return kAppCtrlDoubles + 2 * kAppSlotDoubles + static_cast<std::int64_t>(m) * kNB;
}

void launch_fill(double* x, std::int64_t n, double v, cudaStream_t s);
void launch_zero_u64(unsigned long long* x, std::int64_t n, cudaStream_t s);
void launch_scale_rowmax(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                         const double* b, double alpha, double beta, const double* d, unsigned long long* r,
                         cudaStream_t s);
void launch_scale_update(std::int64_t n, double* d, unsigned long long* r, cudaStream_t s);
// The front kernels are instantiated for R = double (the FP64 factorization that certifies inertia)
// and R = float (the FP32 operator factorization of the mixed-precision path): panels and
// contribution blocks hold R, the pivot scratch stays in units of doubles.
template <class R>
void launch_scatter(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a,
                    const double* b, double alpha, double beta, const double* d, const std::int64_t* dest,
                    R* panels, FactorCounters* cnt, cudaStream_t s);
// inertia-only counts: the largest scaled entry alone, and the scatter of one level's entries
void launch_amax(std::int64_t nnz, const std::int32_t* row, const std::int32_t* col, const double* a, const double* b,
                 double alpha, double beta, const double* d, FactorCounters* cnt, cudaStream_t s);
template <class R>
void launch_scatter_list(const std::int64_t* idx, std::int64_t count, const std::int32_t* row, const std::int32_t* col,
                         const double* a, const double* b, double alpha, double beta, const double* d,
                         const std::int64_t* dest, R* panels, cudaStream_t s);
template <class R>
void launch_zero_cb(const std::int32_t* list, int nlist, int chunks, const SnDev* sn, R* cb, cudaStream_t s);
template <class R>
void launch_extend_add(const int2* items, int nitems, const SnDev* sn, const std::int32_t* rmap, R* panels, R* cb,
                       cudaStream_t s);
template <class R>
void launch_front_small(int maxm, const std::int32_t* list, int nlist, const SnDev* sn, R* panels, R* cb,
                        signed char* piv, std::int32_t* pidx, const FactorParams& prm, FactorCounters* cnt,
                        std::int32_t* failed, cudaStream_t s);
template <class R>
void launch_front_app(const std::int32_t* list, int nlist, const SnDev* sn, R* panels, R* cb, double* scratch,
                      signed char* piv, std::int32_t* pidx, const FactorParams& prm, FactorCounters* cnt,
                      std::int32_t* failed, cudaStream_t s);

// cooperative launch over the large fronts of a level (see factor_kernels.cu); the co-resident grid
// is the smaller of the two instantiations'
int coop_max_ctas(int device);
template <class R>
cudaError_t launch_front_coop(const std::int32_t* list, const std::int32_t* cta_start, int nfronts, int nctas,
                              const SnDev* sn, R* panels, R* cb, double* scratch, signed char* piv, std::int32_t* pidx,
                              const FactorParams& prm, FactorCounters* cnt, std::int32_t* failed, int* level_done,
                              cudaStream_t s);

}  // namespace hsg
