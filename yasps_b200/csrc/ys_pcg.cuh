// Shared PCG device state and reductions (ys_pcg.cu, ys_mas.cu).
#pragma once

#include "ys_common.cuh"
#include "ys_spmv.cuh"

namespace ys {

// Device scalar slots of one PCG solve (double[kSlots]).
enum PcgSlot : int {
  kDelta0 = 0,     // reference preconditioned residual r0^T M^-1 r0 (or rhs^T M^-1 rhs)
  kDeltaNew = 1,   // current r^T z
  kCurv = 2,       // p^T H p
  kDeltaOld = 3,
  kAlpha = 4,
  kBeta = 5,
  kStatus = 6,     // PcgStatus
  kIter = 7,
  kRR = 8,         // current r^T r
  kRR0 = 9,
  kGG = 10,        // rhs^T rhs
  kTolAbs = 11,    // threshold in the units of the stop rule
  kBarrierFail = 12,  // nonzero: a grid barrier wait ran out (the solve is void)
  kTolParam = 13,  // solve parameters, written by the host before each launch
  kMaxItParam = 14,
  kPollLimitParam = 15,  // polls a block makes at a grid barrier before it gives up
  kRestart = 16,   // nonzero: this iteration took a zero step (non-positive curvature), beta = 0 next
  kSlots = 20
};

enum PcgStatus : int { kContinue = 0, kConverged = 1, kNonSpd = 2, kInvalidInit = 3, kMaxIter = 4 };

constexpr int kPcgBlock = 256;

// Polls a block makes at a grid barrier of the PCG loop before it gives up
// and marks the solve void (kBarrierFail).  The grids that wait are
// co-resident, so the wait always ends well before this; the bound only keeps
// a failure from hanging the device.
constexpr uint32_t kDefaultPollLimit = 1u << 24;

// Deterministic grid-wide reduction of NV values: every block stores its
// block sums, the last block to arrive (ticket) reduces the partials in a
// fixed order.  Returns true in the last block, whose threads all receive
// the totals.  partials: [NV * gridDim.x]; ticket: zero on entry, reset here.
// This thread's share (entries threadIdx.x + j blockDim.x) of the sum of n
// block partials, in four independent chains so four loads are in flight;
// the order is fixed by n and the block size.
__device__ __forceinline__ double thread_partial_sum(const double* __restrict__ p, unsigned n) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  unsigned b = threadIdx.x;
  for (; b + 3 * blockDim.x < n; b += 4 * blockDim.x) {
    a0 += __ldcg(p + b);
    a1 += __ldcg(p + b + blockDim.x);
    a2 += __ldcg(p + b + 2 * blockDim.x);
    a3 += __ldcg(p + b + 3 * blockDim.x);
  }
  for (; b < n; b += blockDim.x) a0 += __ldcg(p + b);
  return (a0 + a1) + (a2 + a3);
}

template <int NV, int BLOCK = kPcgBlock>
__device__ __forceinline__ bool grid_reduce_last(double (&v)[NV], double* __restrict__ partials,
                                                 unsigned* __restrict__ ticket) {
  __shared__ double red[BLOCK / 32];
  __shared__ bool last;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    const double s = block_sum<BLOCK>(v[k], red);
    if (threadIdx.x == 0) partials[(uint64_t)k * gridDim.x + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    v[k] = block_sum<BLOCK>(thread_partial_sum(partials + (uint64_t)k * gridDim.x, gridDim.x), red);
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

}  // namespace ys
