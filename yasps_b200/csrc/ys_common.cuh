// Shared helpers of the yasps_b200 CUDA library (sm_100a).
#pragma once

#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "../../include/ys_newton.h"

#define YS_CUDA_TRY(expr)                                                     \
  do {                                                                        \
    cudaError_t ys_err_ = (expr);                                             \
    if (ys_err_ != cudaSuccess) {                                             \
      ys_set_last_error(cudaGetErrorString(ys_err_), __FILE__, __LINE__);     \
      return YS_ERR_CUDA;                                                     \
    }                                                                         \
  } while (0)

#define YS_CHECK_LAUNCH() YS_CUDA_TRY(cudaGetLastError())

#define YS_REQUIRE(cond, code, msg)                                           \
  do {                                                                        \
    if (!(cond)) {                                                            \
      ys_set_last_error(msg, __FILE__, __LINE__);                             \
      return code;                                                            \
    }                                                                         \
  } while (0)

void ys_set_last_error(const char* msg, const char* file, int line);

namespace ys {

constexpr int kSMs = 148;  // B200: 2 dies x 74 SMs

inline unsigned grid_for(uint64_t n, unsigned block) {
  uint64_t g = (n + block - 1) / block;
  return g == 0 ? 1u : (unsigned)(g > 0x7fffffffULL ? 0x7fffffffULL : g);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum (fixed tree): every thread receives the result.
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double* smem /*[BLOCK/32]*/) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) {
    t = lane < BLOCK / 32 ? smem[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) smem[0] = t;
  }
  __syncthreads();
  t = smem[0];
  return t;
}

}  // namespace ys
