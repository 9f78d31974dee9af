// Preconditioned CG with the loop on the device.
//
// The reference's block-Jacobi PCG runs a host loop with ~10 launches and a
// device->host copy per iteration (PKG/kernel/Solver/solverKernel.pyx:606-686);
// its MAS PCG drives a CUDA graph with a conditional while node
// (PKG/solver/mas/cuda/pcg.cu:373-383).  Here one CUDA graph holds the whole
// solve: initial residual, a conditional while node whose body is
//   spmv_dot  : q = H p, curvature p^T q -> alpha         (last-block finish)
//   update    : x += alpha p, r -= alpha q, z = M^-1 r,
//               r^T z, r^T r -> beta, stop test, loop flag  (last-block finish)
//   direction : p = z + beta p
// and a single device->host read of the status per solve.  All reductions are
// deterministic (fixed-order block trees, fixed-order partial sums).
#include <algorithm>
#include <cmath>
#include <vector>

#include "ys_mas.cuh"
#include "ys_pcg.cuh"
#include "ys_spmv_stream.cuh"

namespace ys {

struct PcgParams {
  SpmvSet sets[2];
  int nsets;
  int fp32;
  uint32_t nv;
  const double* rhs;
  double* x;
  double* r;
  double* p;
  float4* p32;  // FP32 copy of p (x, y, z, 0) for the FP32 SpMV, else null
  double* q;
  double* z;
  const double* jinv;
  double* st;
  double* partials;
  unsigned* tickets;
  int stop_rule;
  int zero_guess;
  int restart_on_curvature;  // MAS: a non-positive curvature restarts from M^-1 r (zero step, beta = 0)
  TiledSet tiled;            // tile plan of the FP32 set (pcg_spmv_dot_tiled)
  StreamSet streamed;        // streamed-tile plan of the FP32 set (pcg_spmv_dot_streamed)
  const uint32_t* jgroup;    // block-Jacobi groups (first var | size << 30) or null: 3x3 blocks
  double tolerance;
  uint32_t max_it;
  cudaGraphConditionalHandle cond;
};

__device__ __forceinline__ void jacobi3(const double* __restrict__ inv, uint32_t i, double r0, double r1, double r2,
                                        double& z0, double& z1, double& z2) {
  const double* m = inv + 9ull * i;
  z0 = m[0] * r0 + m[1] * r1 + m[2] * r2;
  z1 = m[3] * r0 + m[4] * r1 + m[5] * r2;
  z2 = m[6] * r0 + m[7] * r1 + m[8] * r2;
}

__device__ __forceinline__ bool stop_reached(const PcgParams& P, double delta_new, double rr) {
  return P.stop_rule == YS_STOP_RESIDUAL ? rr <= P.st[kTolAbs] : delta_new <= P.st[kTolAbs];
}

// Start of the solve from the initial reductions v = (r.z, r.r, g.g,
// g.M^-1 g) (thread 0 of the last block): the stop threshold and the status.
__device__ __forceinline__ void pcg_init_finish(const PcgParams& P, const double (&v)[4]) {
  double* st = P.st;
  const double delta_new = v[0];
  const double delta0 = P.zero_guess ? v[0] : v[3];
  st[kDeltaNew] = delta_new;
  st[kDelta0] = delta0;
  st[kRR] = v[1];
  st[kRR0] = v[1];
  st[kGG] = v[2];
  st[kIter] = 0.0;
  st[kAlpha] = 0.0;
  st[kBeta] = 0.0;
  st[kBarrierFail] = 0.0;
  st[kRestart] = 0.0;
  int status = kContinue;
  double tol;
  if (P.stop_rule == YS_STOP_RESIDUAL) {
    tol = P.st[kTolParam] * P.st[kTolParam] * v[2];
    if (!(isfinite(v[1]) && isfinite(v[2]))) status = kInvalidInit;
    else if (v[1] <= tol) status = kConverged;
    else if (!(isfinite(delta_new) && delta_new > 0.0)) status = kInvalidInit;
  } else {
    // solverKernel.pyx:588-604
    tol = P.st[kTolParam] * delta0;
    if (!(isfinite(delta0) && delta0 >= 0.0 && isfinite(delta_new) && delta_new >= 0.0)) status = kInvalidInit;
    else if (!(isfinite(tol) && tol >= 0.0)) status = kInvalidInit;
    else if (delta_new <= tol) status = kConverged;
  }
  if (status == kContinue && P.st[kMaxItParam] < 1.0) status = kMaxIter;
  st[kTolAbs] = tol;
  st[kStatus] = (double)status;
  cudaGraphSetConditional(P.cond, status == kContinue ? 1u : 0u);
}

// Iteration bookkeeping from v = (r.z, r.r) (thread 0 of the last block).
__device__ __forceinline__ void pcg_update_finish(const PcgParams& P, const double (&v)[2]) {
  double* st = P.st;
  const double delta_new = v[0], delta_old = st[kDeltaOld];
  const double it = st[kIter] + 1.0;
  st[kIter] = it;
  st[kDeltaNew] = delta_new;
  st[kRR] = v[1];
  int status = kContinue;
  // finishCgIteration (solverKernel.pyx:420-438)
  if (!isfinite(delta_new) || delta_new < 0.0 || !isfinite(delta_old) || delta_old <= 0.0) {
    st[kBeta] = 0.0;
    status = kNonSpd;
  } else {
    st[kBeta] = delta_new / delta_old;
    if (stop_reached(P, delta_new, v[1])) status = kConverged;
    else if (it >= P.st[kMaxItParam]) status = kMaxIter;
  }
  st[kStatus] = (double)status;
  cudaGraphSetConditional(P.cond, status == kContinue ? 1u : 0u);
}

// Initial residual, preconditioned residual and the stop threshold.
__global__ void __launch_bounds__(kPcgBlock) pcg_init_bj(PcgParams P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0.0, 0.0, 0.0, 0.0};  // r.z, r.r, g.g, g.M^-1 g
  if (i < P.nv) {
    const double g0 = P.rhs[3ull * i], g1 = P.rhs[3ull * i + 1], g2 = P.rhs[3ull * i + 2];
    double r0 = g0, r1 = g1, r2 = g2;
    if (P.zero_guess) {
      P.x[3ull * i] = 0.0; P.x[3ull * i + 1] = 0.0; P.x[3ull * i + 2] = 0.0;
    } else {
      double h0, h1, h2;
      spmv3_row(P.sets, P.nsets, P.fp32, i, P.x, h0, h1, h2);
      r0 = g0 - h0; r1 = g1 - h1; r2 = g2 - h2;
    }
    double z0, z1, z2;
    jacobi3(P.jinv, i, r0, r1, r2, z0, z1, z2);
    P.r[3ull * i] = r0; P.r[3ull * i + 1] = r1; P.r[3ull * i + 2] = r2;
    P.z[3ull * i] = z0; P.z[3ull * i + 1] = z1; P.z[3ull * i + 2] = z2;
    P.p[3ull * i] = z0; P.p[3ull * i + 1] = z1; P.p[3ull * i + 2] = z2;
    if (P.p32) P.p32[i] = make_float4((float)z0, (float)z1, (float)z2, 0.0f);
    v[0] = r0 * z0 + r1 * z1 + r2 * z2;
    v[1] = r0 * r0 + r1 * r1 + r2 * r2;
    v[2] = g0 * g0 + g1 * g1 + g2 * g2;
    if (!P.zero_guess) {
      double y0, y1, y2;
      jacobi3(P.jinv, i, g0, g1, g2, y0, y1, y2);
      v[3] = g0 * y0 + g1 * y1 + g2 * y2;
    }
  }
  if (!grid_reduce_last<4>(v, P.partials, P.tickets)) return;
  if (threadIdx.x != 0) return;
  pcg_init_finish(P, v);
}

// Curvature p^T q (grid reduction) and the step length; the last block of
// the grid decides.
template <int BLOCK = kPcgBlock>
__device__ __forceinline__ void spmv_dot_finish(const PcgParams& P, double (&v)[1]) {
  if (!grid_reduce_last<1, BLOCK>(v, P.partials, P.tickets + 1)) return;
  if (threadIdx.x != 0) return;
  double* st = P.st;
  const double curv = v[0];
  st[kCurv] = curv;
  st[kDeltaOld] = st[kDeltaNew];
  const double rz = st[kDeltaNew];
  if (P.restart_on_curvature && isfinite(curv) && curv <= 0.0 && isfinite(rz) && rz > 0.0) {
    // The reference's MAS PCG (mas/cuda/pcg.cu:183-189): rounding can break
    // conjugacy on an ill-conditioned SPD system, so a finite non-positive
    // curvature takes a zero step and restarts from M^-1 r (beta = 0 in the
    // collect kernel) instead of ending the solve as non-SPD.
    st[kAlpha] = 0.0;
    st[kRestart] = 1.0;
  } else if (!isfinite(curv) || curv <= 0.0) {
    // prepareCgIteration (solverKernel.pyx:388-404)
    st[kAlpha] = 0.0;
    st[kStatus] = (double)kNonSpd;
    st[kIter] = st[kIter] + 1.0;
    cudaGraphSetConditional(P.cond, 0u);
  } else {
    st[kAlpha] = rz / curv;
  }
}

// kRowLanes threads per row (see spmv3_group).
// One instantiation per precision of the block values (the FP32 one keeps
// fewer registers: higher occupancy for the latency-bound gathers).
// A grid of resident size strides over the groups of kPcgBlock / kRowLanes
// rows: the dot product then ends in a few hundred block partials (each
// block's fence and ticket, and the last block's sum, are per block, so a
// CTA per row group would pay them thousands of times).
template <bool FP32>
__global__ void __launch_bounds__(kPcgBlock) pcg_spmv_dot(PcgParams P) {
  constexpr uint32_t kRows = kPcgBlock / kRowLanes;
  const uint32_t groups = (P.nv + kRows - 1) / kRows;
  const int lane = (int)(threadIdx.x % kRowLanes);
  double v[1] = {0.0};
  for (uint32_t gb = blockIdx.x; gb < groups; gb += gridDim.x) {  // block-uniform
    const uint32_t i = gb * kRows + threadIdx.x / kRowLanes;
    double q0, q1, q2;
    if (FP32) spmv3_group_x32(P.sets, P.nsets, i, i < P.nv, lane, P.p32, q0, q1, q2);
    else spmv3_group(P.sets, P.nsets, false, i, i < P.nv, lane, P.p, q0, q1, q2);
    if (i < P.nv && lane == 0) {
      P.q[3ull * i] = q0; P.q[3ull * i + 1] = q1; P.q[3ull * i + 2] = q2;
      v[0] += P.p[3ull * i] * q0 + P.p[3ull * i + 1] * q1 + P.p[3ull * i + 2] * q2;
    }
  }
  spmv_dot_finish(P, v);
}

// The SpMV + dot of the FP32 loop over the tile plan: each persistent CTA
// stages its tiles' blocks into shared memory by bulk copies (see
// ys_spmv_tiled.cuh); lane 0 of a row group writes q and adds p . q.
__global__ void __launch_bounds__(kTileThreads, 3) pcg_spmv_dot_tiled(PcgParams P) {
  double v[1] = {0.0};
  spmv3_tiles_x32(P.tiled, P.p32, P.tickets + 6, [&](uint32_t i, bool valid, int lane, double q0, double q1,
                                                     double q2) {
    if (!valid || lane != 0) return;
    P.q[3ull * i] = q0; P.q[3ull * i + 1] = q1; P.q[3ull * i + 2] = q2;
    v[0] += P.p[3ull * i] * q0 + P.p[3ull * i + 1] * q1 + P.p[3ull * i + 2] * q2;
  });
  spmv_dot_finish<kTileThreads>(P, v);
}

// The same over the streamed-tile plan (see ys_spmv_stream.cuh).
__global__ void __launch_bounds__(kTileThreads, 2) pcg_spmv_dot_streamed(PcgParams P) {
  double v[1] = {0.0};
  double pp[3] = {0.0, 0.0, 0.0};  // p of the row, loaded before its products
  spmv3_stream_x32(
      P.streamed, P.p32, P.tickets + 6,
      [&](uint32_t i, bool valid, int lane) {
        if (valid && lane == 0)
          for (int c = 0; c < 3; ++c) pp[c] = P.p[3ull * i + c];
      },
      [&](uint32_t i, bool valid, int lane, double q0, double q1, double q2) {
        if (!valid || lane != 0) return;
        P.q[3ull * i] = q0; P.q[3ull * i + 1] = q1; P.q[3ull * i + 2] = q2;
        v[0] += pp[0] * q0 + pp[1] * q1 + pp[2] * q2;
      });
  spmv_dot_finish<kTileThreads>(P, v);
}

__global__ void __launch_bounds__(kPcgBlock) pcg_update_bj(PcgParams P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = P.st[kStatus] == (double)kContinue;
  double v[2] = {0.0, 0.0};
  if (i < P.nv && live) {
    const double alpha = P.st[kAlpha];
    double r[3], z[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      P.x[3ull * i + k] = P.x[3ull * i + k] + P.p[3ull * i + k] * alpha;
      r[k] = P.r[3ull * i + k] - P.q[3ull * i + k] * alpha;
      P.r[3ull * i + k] = r[k];
    }
    jacobi3(P.jinv, i, r[0], r[1], r[2], z[0], z[1], z[2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) P.z[3ull * i + k] = z[k];
    v[0] = r[0] * z[0] + r[1] * z[1] + r[2] * z[2];
    v[1] = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  }
  if (!grid_reduce_last<2>(v, P.partials, P.tickets + 2)) return;
  if (threadIdx.x != 0 || !live) return;
  pcg_update_finish(P, v);
}

// ---- block-Jacobi over variable groups ----------------------------------------
// A target wider than 3 (the 9-DoF affine matrix of a body, stored as three
// 3-DoF rows) has one diagonal block of 9x9 whose pseudo-inverse couples its
// three rows (diagonalBlockInverseKernel.pyx:40-215 inverts per attribute
// block).  With jgroup, jinv holds for every 3-DoF variable the 3 x 9 strip of
// its group's inverse (27 doubles, row-major; columns of the group's
// variables in order) and jgroup[i] = first variable of i's group | (group
// size << 30).  The thread of a group's first variable updates the whole
// group, so every z of the group sees the group's new residual.
constexpr uint32_t kGroupShift = 30;

__device__ __forceinline__ void group_apply(const double* __restrict__ jinv, uint32_t g, int gs, const double* rr,
                                            double* zz) {
  for (int s = 0; s < gs; ++s) {
    const double* strip = jinv + 27ull * (g + s);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double acc = 0.0;
      for (int t = 0; t < 3 * gs; ++t) acc += strip[9 * k + t] * rr[t];
      zz[3 * s + k] = acc;
    }
  }
}

__global__ void __launch_bounds__(kPcgBlock) pcg_init_bjw(PcgParams P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0.0, 0.0, 0.0, 0.0};  // r.z, r.r, g.g, g.M^-1 g
  if (i < P.nv && (P.jgroup[i] & ((1u << kGroupShift) - 1)) == i) {
    const int gs = (int)(P.jgroup[i] >> kGroupShift);
    double gg[9], rr[9], zz[9], yy[9];
    for (int s = 0; s < gs; ++s) {
      const uint32_t j = i + s;
#pragma unroll
      for (int k = 0; k < 3; ++k) gg[3 * s + k] = rr[3 * s + k] = P.rhs[3ull * j + k];
      if (P.zero_guess) {
#pragma unroll
        for (int k = 0; k < 3; ++k) P.x[3ull * j + k] = 0.0;
      } else {
        double h0, h1, h2;
        spmv3_row(P.sets, P.nsets, P.fp32, j, P.x, h0, h1, h2);
        rr[3 * s] -= h0; rr[3 * s + 1] -= h1; rr[3 * s + 2] -= h2;
      }
    }
    group_apply(P.jinv, i, gs, rr, zz);
    if (!P.zero_guess) group_apply(P.jinv, i, gs, gg, yy);
    for (int s = 0; s < gs; ++s) {
      const uint32_t j = i + s;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int q = 3 * s + k;
        P.r[3ull * j + k] = rr[q];
        P.z[3ull * j + k] = zz[q];
        P.p[3ull * j + k] = zz[q];
        v[0] += rr[q] * zz[q];
        v[1] += rr[q] * rr[q];
        v[2] += gg[q] * gg[q];
        if (!P.zero_guess) v[3] += gg[q] * yy[q];
      }
      if (P.p32) P.p32[j] = make_float4((float)zz[3 * s], (float)zz[3 * s + 1], (float)zz[3 * s + 2], 0.0f);
    }
  }
  if (!grid_reduce_last<4>(v, P.partials, P.tickets)) return;
  if (threadIdx.x != 0) return;
  pcg_init_finish(P, v);
}

__global__ void __launch_bounds__(kPcgBlock) pcg_update_bjw(PcgParams P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = P.st[kStatus] == (double)kContinue;
  double v[2] = {0.0, 0.0};
  if (i < P.nv && live && (P.jgroup[i] & ((1u << kGroupShift) - 1)) == i) {
    const int gs = (int)(P.jgroup[i] >> kGroupShift);
    const double alpha = P.st[kAlpha];
    double rr[9], zz[9];
    for (int s = 0; s < gs; ++s) {
      const uint32_t j = i + s;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        P.x[3ull * j + k] = P.x[3ull * j + k] + P.p[3ull * j + k] * alpha;
        rr[3 * s + k] = P.r[3ull * j + k] - P.q[3ull * j + k] * alpha;
        P.r[3ull * j + k] = rr[3 * s + k];
      }
    }
    group_apply(P.jinv, i, gs, rr, zz);
    for (int s = 0; s < gs; ++s) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int q = 3 * s + k;
        P.z[3ull * (i + s) + k] = zz[q];
        v[0] += rr[q] * zz[q];
        v[1] += rr[q] * rr[q];
      }
    }
  }
  if (!grid_reduce_last<2>(v, P.partials, P.tickets + 2)) return;
  if (threadIdx.x != 0 || !live) return;
  pcg_update_finish(P, v);
}

__global__ void __launch_bounds__(kPcgBlock) pcg_direction(PcgParams P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.nv) return;
  if (P.st[kStatus] == (double)kNonSpd) return;
  const double beta = P.st[kBeta];
  double p[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    p[k] = P.z[3ull * i + k] + P.p[3ull * i + k] * beta;
    P.p[3ull * i + k] = p[k];
  }
  if (P.p32) P.p32[i] = make_float4((float)p[0], (float)p[1], (float)p[2], 0.0f);
}

// Iterative refinement step in FP64: x += delta, then r = rhs - H x with the
// FP64 blocks and the deterministic norms ||r||^2, ||rhs||^2 in out[0..1].
__global__ void __launch_bounds__(kPcgBlock) refine_add(uint32_t nv, double* __restrict__ x,
                                                        const double* __restrict__ delta) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
#pragma unroll
  for (int k = 0; k < 3; ++k) x[3ull * i + k] += delta[3ull * i + k];
}

struct RefineParams {
  SpmvSet sets[2];
  int nsets;
  uint32_t nv;
  const double* rhs;
  const double* x;
  double* r;
  double* out;
  double* partials;
  unsigned* ticket;
};

// kRowLanes threads a row on a resident-size grid striding over the row
// groups (as pcg_spmv_dot), FP64 blocks.
__global__ void __launch_bounds__(kPcgBlock) refine_residual(RefineParams P) {
  constexpr uint32_t kRows = kPcgBlock / kRowLanes;
  const uint32_t groups = (P.nv + kRows - 1) / kRows;
  const int lane = (int)(threadIdx.x % kRowLanes);
  double v[2] = {0.0, 0.0};
  for (uint32_t gb = blockIdx.x; gb < groups; gb += gridDim.x) {  // block-uniform
    const uint32_t i = gb * kRows + threadIdx.x / kRowLanes;
    double h[3] = {0.0, 0.0, 0.0};
    // x == NULL is the zero vector: r = g without the product
    if (P.x) spmv3_group(P.sets, P.nsets, false, i, i < P.nv, lane, P.x, h[0], h[1], h[2]);
    if (i < P.nv && lane == 0) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double g = P.rhs[3ull * i + k];
        const double r = g - h[k];
        P.r[3ull * i + k] = r;
        v[0] += r * r;
        v[1] += g * g;
      }
    }
  }
  if (!grid_reduce_last<2>(v, P.partials, P.ticket)) return;
  if (threadIdx.x == 0) {
    P.out[0] = v[0];
    P.out[1] = v[1];
  }
}

struct PcgHandle {
  PcgParams P;
  int preconditioner;
  MasPcgHooks mas;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double* slots_host = nullptr;
  // tolerance, iteration budget, grid-barrier poll limit (copied to the
  // device per launch)
  double params[3] = {0.0, 0.0, (double)kDefaultPollLimit};
};

static cudaError_t add_kernel(cudaGraph_t g, cudaGraphNode_t* node, const cudaGraphNode_t* deps, size_t ndeps,
                              const void* fn, unsigned grid, unsigned block, void** args, size_t smem = 0) {
  cudaKernelNodeParams kp{};
  kp.func = const_cast<void*>(fn);
  kp.gridDim = dim3(grid);
  kp.blockDim = dim3(block);
  kp.sharedMemBytes = (unsigned)smem;
  kp.kernelParams = args;
  kp.extra = nullptr;
  return cudaGraphAddKernelNode(node, g, deps, ndeps, &kp);
}

}  // namespace ys

extern "C" {

uint64_t ys_pcg_workspace_doubles(uint32_t n) {
  const uint64_t nv = (n + 2) / 3;
  const uint64_t grid = (nv + ys::kPcgBlock - 1) / ys::kPcgBlock;
  // r, p, q, z (n each) + the FP32 copy of p (4 floats per variable) +
  // slots + partials + tickets
  // partials: up to 4 values per block of the row kernels, or 1 per block of
  // the kRowLanes-per-row SpMV (kRowLanes times more blocks)
  return 4ull * 3 * nv + 2 * nv + ys::kSlots + (uint64_t)ys::kRowLanes * (grid + 2) + 8;
}

int32_t ys_pcg_create(const ys_pcg_args* args, void** handle) {
  YS_REQUIRE(args && handle, YS_ERR_INVALID, "null argument");
  const ys_pcg_args& a = *args;
  YS_REQUIRE(a.matrix.num_sets >= 1 && a.matrix.num_sets <= 2, YS_ERR_INVALID, "1 or 2 block sets");
  YS_REQUIRE(a.preconditioner == YS_PREC_BLOCK_JACOBI ? a.jacobi_inverse != nullptr : a.mas != nullptr,
             YS_ERR_INVALID, "missing preconditioner data");
  auto* h = new ys::PcgHandle();
  ys::PcgParams& P = h->P;
  P.nsets = (int)a.matrix.num_sets;
  P.fp32 = a.precision == 1;
  for (int s = 0; s < P.nsets; ++s) {
    P.sets[s] = ys::SpmvSet{a.matrix.values[s], a.matrix.values32[s], a.matrix.row_ptr[s], a.matrix.entry_block[s],
                            a.matrix.entry_col[s]};
    if (P.fp32 && !P.sets[s].values32) { delete h; YS_REQUIRE(false, YS_ERR_INVALID, "FP32 PCG needs values32"); }
    if (!P.fp32 && !P.sets[s].values) { delete h; YS_REQUIRE(false, YS_ERR_INVALID, "FP64 PCG needs values"); }
  }
  P.nv = a.matrix.num_vars;
  const uint64_t n = 3ull * P.nv;
  P.rhs = a.rhs;
  P.x = a.solution;
  double* w = a.workspace;
  P.r = w; w += n;
  P.p = w; w += n;
  P.q = w; w += n;
  P.z = w; w += n;
  // 12 doubles per variable before it: 16-byte aligned with the workspace
  P.p32 = P.fp32 ? reinterpret_cast<float4*>(w) : nullptr;
  w += 2ull * P.nv;
  P.st = w; w += ys::kSlots;
  const unsigned grid = ys::grid_for(P.nv, ys::kPcgBlock);
  unsigned grid_rows = ys::grid_for((uint64_t)P.nv * ys::kRowLanes, ys::kPcgBlock);
  {
    // resident-size grid for the SpMV + dot (see pcg_spmv_dot)
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, P.fp32 ? (const void*)ys::pcg_spmv_dot<true> : (const void*)ys::pcg_spmv_dot<false>, ys::kPcgBlock,
            0) == cudaSuccess &&
        sms > 0 && per_sm > 0)
      grid_rows = std::min<unsigned>(grid_rows, (unsigned)(sms * per_sm));
  }
  // the FP32 loop of a single block set with a tile plan runs the tiled
  // SpMV (persistent CTAs, shared-memory stages)
  bool tiled = false, streamed = false;
  size_t tile_smem = 0;
  unsigned grid_tiles = 0;
  const ys_spmv_stream& sp = a.matrix.stream[0];
  if (P.fp32 && P.nsets == 1 && sp.blocks32 && sp.desc && sp.rows && sp.words && sp.halo && sp.block_cap > 0 &&
      sp.entry_cap > 0 && sp.halo_cap > 0 && sp.halo_cap <= ys::kStreamMaxHalo && sp.block_cap % 4 == 0 &&
      sp.entry_cap % 4 == 0 && sp.halo_cap % 4 == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    const uint32_t stages = ys::stream_pick_stages((const void*)ys::pcg_spmv_dot_streamed, sp.block_cap,
                                                   sp.entry_cap, sp.halo_cap, &per_sm);
    tile_smem = ys::stream_smem_bytes(sp.block_cap, sp.entry_cap, sp.halo_cap, stages ? stages : 2);
    if (stages && cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaFuncSetAttribute(ys::pcg_spmv_dot_streamed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tile_smem) == cudaSuccess &&
        sms > 0 && per_sm > 0) {
      const unsigned ntiles = (P.nv + ys::kTileRows - 1) / ys::kTileRows;
      grid_tiles = std::min<unsigned>(ntiles, (unsigned)(sms * per_sm));
      streamed = true;
      P.streamed = ys::stream_set(sp, P.sets[0], P.nv, stages);
    }
  }
  if (!streamed && P.fp32 && P.nsets == 1 && a.matrix.row_block[0] && a.matrix.tile_cap[0] > 0 &&
      a.matrix.entry_cap[0] > 0) {
    int dev = 0, sms = 0, per_sm = 0, smem_sm = 0;
    uint32_t stages = 2;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess)
      stages = ys::tile_auto_stages(a.matrix.tile_cap[0], a.matrix.entry_cap[0], (size_t)smem_sm);
    tile_smem = ys::tile_smem_bytes(a.matrix.tile_cap[0], a.matrix.entry_cap[0], stages);
    if (tile_smem <= 200u * 1024u &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaFuncSetAttribute(ys::pcg_spmv_dot_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem) ==
            cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ys::pcg_spmv_dot_tiled, ys::kTileThreads, tile_smem) ==
            cudaSuccess &&
        sms > 0 && per_sm > 0) {
      const unsigned ntiles = (P.nv + ys::kTileRows - 1) / ys::kTileRows;
      grid_tiles = std::min<unsigned>(ntiles, (unsigned)(sms * per_sm));
      tiled = true;
      P.tiled = ys::TiledSet{a.matrix.values32[0], a.matrix.row_ptr[0], a.matrix.entry_block[0],
                             a.matrix.entry_col[0], a.matrix.row_block[0], P.nv, a.matrix.tile_cap[0],
                             a.matrix.entry_cap[0], stages};
    }
  }
  P.partials = w; w += (uint64_t)ys::kRowLanes * (grid + 2);
  P.tickets = reinterpret_cast<unsigned*>(w);
  P.jinv = a.jacobi_inverse;
  P.jgroup = a.jacobi_group;
  P.stop_rule = a.stop_rule;
  P.zero_guess = a.zero_initial_guess;
  P.restart_on_curvature = a.preconditioner == YS_PREC_MAS;
  P.tolerance = a.tolerance;
  P.max_it = a.max_iterations;
  h->params[0] = a.tolerance;
  h->params[1] = (double)a.max_iterations;
  h->preconditioner = a.preconditioner;

  cudaError_t e = cudaGraphCreate(&h->graph, 0);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&P.cond, h->graph, 0, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) e = cudaMallocHost(&h->slots_host, sizeof(double) * ys::kSlots);
  cudaGraphNode_t reset = nullptr, init = nullptr, loop = nullptr;
  if (e == cudaSuccess) {
    cudaMemsetParams mp{};
    mp.dst = P.tickets;
    mp.value = 0;
    mp.pitch = 0;
    mp.elementSize = 4;
    mp.width = 8;
    mp.height = 1;
    e = cudaGraphAddMemsetNode(&reset, h->graph, nullptr, 0, &mp);
  }
  if (e == cudaSuccess) {
    if (a.preconditioner == YS_PREC_BLOCK_JACOBI) {
      void* args0[] = {&P};
      e = ys::add_kernel(h->graph, &init, &reset, 1,
                         P.jgroup ? (const void*)ys::pcg_init_bjw : (const void*)ys::pcg_init_bj, grid, ys::kPcgBlock,
                         args0);
    } else {
      e = ys::mas_add_init_nodes(a.mas, h->graph, &reset, 1, &init, P.nv, P.rhs, P.x, P.r, P.p, P.p32, P.q, P.z, P.st, P.partials,
                                 P.tickets, P.sets, P.nsets, P.fp32, P.stop_rule, P.zero_guess, P.tolerance, P.max_it,
                                 P.cond, &h->mas);
    }
  }
  if (e == cudaSuccess) {
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = P.cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&loop, h->graph, &init, 1, &cp);
    if (e == cudaSuccess) {
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      cudaGraphNode_t n1 = nullptr, n2 = nullptr, n3 = nullptr;
      void* args1[] = {&P};
      if (streamed)
        e = ys::add_kernel(body, &n1, nullptr, 0, (const void*)ys::pcg_spmv_dot_streamed, grid_tiles,
                           ys::kTileThreads, args1, tile_smem);
      else if (tiled)
        e = ys::add_kernel(body, &n1, nullptr, 0, (const void*)ys::pcg_spmv_dot_tiled, grid_tiles, ys::kTileThreads,
                           args1, tile_smem);
      else
        e = ys::add_kernel(body, &n1, nullptr, 0,
                           P.fp32 ? (const void*)ys::pcg_spmv_dot<true> : (const void*)ys::pcg_spmv_dot<false>,
                           grid_rows, ys::kPcgBlock, args1);
      if (e == cudaSuccess) {
        if (a.preconditioner == YS_PREC_BLOCK_JACOBI) {
          e = ys::add_kernel(body, &n2, &n1, 1,
                             P.jgroup ? (const void*)ys::pcg_update_bjw : (const void*)ys::pcg_update_bj, grid,
                             ys::kPcgBlock, args1);
        } else {
          e = ys::mas_add_update_nodes(a.mas, body, &n1, 1, &n2, &h->mas);
        }
      }
      if (e == cudaSuccess && a.preconditioner != YS_PREC_BLOCK_JACOBI && h->mas.fused_direction)
        n3 = n2;  // the MAS collect kernel updated p already
      else if (e == cudaSuccess)
        e = ys::add_kernel(body, &n3, &n2, 1, (const void*)ys::pcg_direction, grid, ys::kPcgBlock, args1);
    }
  }
  // per-node priorities (the MAS coarse chain) take effect only with this flag
  if (e == cudaSuccess) e = cudaGraphInstantiate(&h->exec, h->graph, cudaGraphInstantiateFlagUseNodePriority);
  if (e != cudaSuccess) {
    ys_set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->slots_host) cudaFreeHost(h->slots_host);
    delete h;
    return YS_ERR_CUDA;
  }
  *handle = h;
  return YS_OK;
}

int32_t ys_pcg_launch(void* handle, void* stream) {
  YS_REQUIRE(handle, YS_ERR_INVALID, "null handle");
  auto* h = static_cast<ys::PcgHandle*>(handle);
  // Pageable source: the copy is staged before the call returns, so the
  // parameters may change for the next launch right away.
  const double params[3] = {h->params[0], h->params[1], h->params[2]};
  YS_CUDA_TRY(cudaMemcpyAsync(h->P.st + ys::kTolParam, params, sizeof(params), cudaMemcpyHostToDevice,
                              (cudaStream_t)stream));
  YS_CUDA_TRY(cudaGraphLaunch(h->exec, (cudaStream_t)stream));
  return YS_OK;
}

int32_t ys_pcg_set_params(void* handle, double tolerance, uint32_t max_iterations) {
  YS_REQUIRE(handle, YS_ERR_INVALID, "null handle");
  auto* h = static_cast<ys::PcgHandle*>(handle);
  h->params[0] = tolerance;
  h->params[1] = (double)max_iterations;
  return YS_OK;
}

int32_t ys_pcg_set_barrier_poll_limit(void* handle, uint32_t polls) {
  YS_REQUIRE(handle, YS_ERR_INVALID, "null handle");
  static_cast<ys::PcgHandle*>(handle)->params[2] = (double)polls;
  return YS_OK;
}

int32_t ys_pcg_status(void* handle, void* stream, ys_pcg_result* result) {
  YS_REQUIRE(handle && result, YS_ERR_INVALID, "null argument");
  auto* h = static_cast<ys::PcgHandle*>(handle);
  cudaStream_t s = (cudaStream_t)stream;
  YS_CUDA_TRY(cudaMemcpyAsync(h->slots_host, h->P.st, sizeof(double) * ys::kSlots, cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaStreamSynchronize(s));
  const double* st = h->slots_host;
  const int status = (int)st[ys::kStatus];
  const uint32_t it = (uint32_t)st[ys::kIter];
  result->iterations = it;
  result->delta0 = st[ys::kDelta0];
  result->delta = st[ys::kDeltaNew];
  result->residual0 = sqrt(st[ys::kRR0]);
  result->residual = sqrt(st[ys::kRR]);
  if (st[ys::kBarrierFail] != 0.0) {
    // a grid barrier of the loop gave up waiting (it never does when the
    // grid is co-resident); nothing of the solve is valid
    result->status = YS_ERR_CUDA;
    ys_set_last_error("PCG grid barrier wait ran out", __FILE__, __LINE__);
    return YS_ERR_CUDA;
  }
  switch (status) {
    case ys::kConverged: result->status = (int32_t)it; break;
    case ys::kNonSpd: result->status = -(int32_t)it - 4; break;
    case ys::kInvalidInit: result->status = YS_ERR_INVALID_RESIDUAL; break;
    case ys::kMaxIter: result->status = YS_ERR_NOT_CONVERGED; break;
    default: result->status = YS_ERR_NOT_CONVERGED; break;
  }
  return YS_OK;
}

int32_t ys_pcg_run(void* handle, void* stream, ys_pcg_result* result) {
  int32_t rc = ys_pcg_launch(handle, stream);
  if (rc != YS_OK) return rc;
  return ys_pcg_status(handle, stream, result);
}

uint64_t ys_refine_workspace_doubles(uint32_t num_vars) {
  // norms (2) + ticket (2) + 2 partials per block, at most one block a row group
  const uint64_t groups = (num_vars + ys::kPcgBlock / ys::kRowLanes - 1) / (ys::kPcgBlock / ys::kRowLanes);
  return 4 + 2 * (groups + 1);
}

int32_t ys_refine_residual(const ys_matrix3* m, const double* rhs, double* x, const double* delta, double* r,
                           double* workspace, double* norms_host, void* stream) {
  YS_REQUIRE(m && m->num_sets >= 1 && m->num_sets <= 2, YS_ERR_INVALID, "bad matrix");
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t nv = m->num_vars;
  const unsigned grid = ys::grid_for(nv, ys::kPcgBlock);
  YS_REQUIRE(x || !delta, YS_ERR_INVALID, "a correction needs the solution vector");
  if (delta) {
    ys::refine_add<<<grid, ys::kPcgBlock, 0, s>>>(nv, x, delta);
    YS_CHECK_LAUNCH();
  }
  ys::RefineParams P{};
  P.nsets = (int)m->num_sets;
  for (int k = 0; k < P.nsets; ++k)
    P.sets[k] = ys::SpmvSet{m->values[k], nullptr, m->row_ptr[k], m->entry_block[k], m->entry_col[k]};
  P.nv = nv;
  P.rhs = rhs;
  P.x = x;
  P.r = r;
  P.out = workspace;
  P.ticket = reinterpret_cast<unsigned*>(workspace + 2);
  P.partials = workspace + 4;
  unsigned rgrid = ys::grid_for((uint64_t)nv * ys::kRowLanes, ys::kPcgBlock);
  {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ys::refine_residual, ys::kPcgBlock, 0) == cudaSuccess &&
        sms > 0 && per_sm > 0)
      rgrid = std::min<unsigned>(rgrid, (unsigned)(sms * per_sm));
  }
  YS_CUDA_TRY(cudaMemsetAsync(P.ticket, 0, sizeof(unsigned), s));
  ys::refine_residual<<<rgrid, ys::kPcgBlock, 0, s>>>(P);
  YS_CHECK_LAUNCH();
  if (norms_host) {
    YS_CUDA_TRY(cudaMemcpyAsync(norms_host, workspace, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    YS_CUDA_TRY(cudaStreamSynchronize(s));
  }
  return YS_OK;
}

int32_t ys_pcg_destroy(void* handle) {
  if (!handle) return YS_OK;
  auto* h = static_cast<ys::PcgHandle*>(handle);
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  if (h->slots_host) cudaFreeHost(h->slots_host);
  delete h;
  return YS_OK;
}

}  // extern "C"
