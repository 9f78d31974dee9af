// MAS device state and the per-node / per-domain bodies of its application,
// shared by the single-solve kernels (ys_mas.cu) and the batched serving
// kernels (ys_serve.cu).
//
// Application z = sum_l w_l P_l A_l^-1 R_l r (PKG/solver/mas/preconditioner.py:128-154):
//   restriction : a level-l node sums its children of level l-1 (FP64, fixed
//                 order; children of level 1 are fine nodes read from r);
//   domain GEMV : z_d = A_d^-1 r_d from the packed FP32 upper triangle;
//   collect     : z_i = sum_l w_l z_l(map_l(i)).
#pragma once

#include "ys_common.cuh"

namespace ys {

constexpr int kMaxLevels = 8;

struct MasDev {
  uint32_t nv;              // fine 3-DoF nodes
  uint32_t levels;
  uint32_t packed_nodes;    // total nodes over all levels
  uint32_t level_node_offset[kMaxLevels + 1];
  float weight[kMaxLevels];
  const uint32_t* cmap;     // [levels x nv] packed node index per fine node and level
  const uint32_t* child_ptr;   // [packed_nodes - nv + 1] children (packed ids of level l-1) of coarse nodes
  const uint32_t* child_fine;
  // domains (all levels)
  uint32_t num_domains;
  const uint32_t* dom_node_ptr;   // [D+1]
  const uint32_t* dom_nodes;      // packed node ids in local order
  const uint64_t* inv_offset;     // [D]
  const uint32_t* dom_entry_ptr;  // [D+1] dense assembly entries of each domain
  const uint32_t* dom_entry;      // [E*3] (local i, local j, level block index)
  // level blocks: level 0 = fine upper blocks (values supplied per update)
  uint32_t fine_blocks;
  uint32_t coarse_blocks;         // blocks of levels >= 1 (stored after the fine ones)
  const uint32_t* cb_src_ptr;     // [coarse_blocks+1]
  const uint32_t* cb_src;         // source block index (into level values) | mode << 30
  uint32_t cb_level_begin[kMaxLevels + 1];  // coarse block ranges per level (relative)
  double* coarse_values;          // [coarse_blocks * 9]
  float* inverse;                 // FP32 inverses (packed upper triangles)
  float* rl;                      // packed level residuals [3 * packed_nodes]
  double* rl64;                   // FP64 restriction chain (levels >= 1)
  float* zl;                      // packed level corrections
  int* status;                    // [1] failing domain count
  uint32_t max_dofs;
  const double* fine_values;      // set at numeric update
};

__device__ __forceinline__ const double* level_block(const MasDev& M, uint32_t idx) {
  return idx < M.fine_blocks ? M.fine_values + 9ull * idx : M.coarse_values + 9ull * (idx - M.fine_blocks);
}

// Level-l (l >= 1) node p by one warp (p warp-uniform): lane k sums children
// k, k+32, ... of level l-1 (FP64), a fixed xor-shuffle tree adds the lanes.
__device__ __forceinline__ void restrict_node_warp(const MasDev& M, const double* __restrict__ r, uint32_t level,
                                                   uint32_t p, int lane) {
  const double* src = level == 1 ? r : M.rl64;
  const uint32_t c = p - M.nv;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (uint32_t q = M.child_ptr[c] + lane; q < M.child_ptr[c + 1]; q += 32) {
    const uint32_t f = M.child_fine[q];
    s0 += src[3ull * f]; s1 += src[3ull * f + 1]; s2 += src[3ull * f + 2];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    M.rl64[3ull * p] = s0;
    M.rl64[3ull * p + 1] = s1;
    M.rl64[3ull * p + 2] = s2;
    M.rl[3ull * p] = (float)s0;
    M.rl[3ull * p + 1] = (float)s1;
    M.rl[3ull * p + 2] = (float)s2;
  }
}

// Levels first..coarsest by one CTA, level by level (a warp per node).
__device__ __forceinline__ void restrict_tail_levels(const MasDev& M, const double* __restrict__ r,
                                                     uint32_t first) {
  const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  for (uint32_t level = first; level < M.levels; ++level) {
    const uint32_t begin = M.level_node_offset[level], end = M.level_node_offset[level + 1];
    for (uint32_t p = begin + warp; p < end; p += nwarps) restrict_node_warp(M, r, level, p, lane);
    __syncthreads();
  }
}

// First level handled by the one-CTA tail restriction: every level from
// there on has at most kTailNodes nodes.
constexpr uint32_t kTailNodes = 512;

__host__ __device__ inline uint32_t restrict_tail_first(const MasDev& M) {
  uint32_t first = M.levels;
  while (first > 1 && M.level_node_offset[first] - M.level_node_offset[first - 1] <= kTailNodes) --first;
  return first;
}

// z_d = A_d^-1 r_d for domain d by one CTA.  The FP32 inverse is stored as
// its packed upper triangle (n(n+1)/2 floats from a 16-byte aligned offset):
// it is staged in shared memory with coalesced 16-byte loads, so every byte
// crosses HBM once and half as many bytes cross as for a full n x n inverse.
// Thread i owns output row i; S(i, j) for j < i is read from column i of the
// upper triangle (consecutive threads, consecutive words).
__host__ __device__ inline uint32_t gemv_rloc_offset(uint32_t max_dofs) {
  return (max_dofs * (max_dofs + 1) / 2 + 3) & ~3u;
}
inline size_t gemv_smem_bytes(uint32_t max_dofs) { return 4ull * (gemv_rloc_offset(max_dofs) + max_dofs); }

__device__ __forceinline__ void gemv_domain(const MasDev& M, uint32_t d, float4* smem) {
  float* S = reinterpret_cast<float*>(smem);
  float* rloc = S + gemv_rloc_offset(M.max_dofs);
  const uint32_t nb = M.dom_node_ptr[d], nn = M.dom_node_ptr[d + 1] - nb;
  const uint32_t n = 3 * nn;
  const uint32_t packed4 = (n * (n + 1) / 2 + 3) / 4;
  const float4* src = reinterpret_cast<const float4*>(M.inverse + M.inv_offset[d]);
  for (uint32_t t = threadIdx.x; t < packed4; t += blockDim.x) smem[t] = __ldg(src + t);
  for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
    const uint32_t node = M.dom_nodes[nb + t / 3];
    rloc[t] = M.rl[3ull * node + t % 3];
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t bi = i * n - i * (i - 1) / 2 - i;  // S(i, j) = S[bi + j], j >= i
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t bj = 0;  // start of packed row j
    uint32_t j = 0;
    for (; j + 4 <= n; j += 4) {
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint32_t jj = j + u;
        const uint32_t idx = jj < i ? bj + (i - jj) : bi + jj;
        acc[u] += S[idx] * rloc[jj];
        bj += n - jj;
      }
    }
    for (; j < n; ++j) {
      const uint32_t idx = j < i ? bj + (i - j) : bi + j;
      acc[0] += S[idx] * rloc[j];
      bj += n - j;
    }
    const float s = (acc[0] + acc[1]) + (acc[2] + acc[3]);
    const uint32_t node = M.dom_nodes[nb + i / 3];
    M.zl[3ull * node + i % 3] = s;
  }
}

// z_i = sum_l w_l z_l(map_l(i)) for fine node i (FP64 sum in level order).
__device__ __forceinline__ void collect_levels(const MasDev& M, uint32_t nv, uint32_t i, double (&z)[3]) {
  z[0] = z[1] = z[2] = 0.0;
  for (uint32_t l = 0; l < M.levels; ++l) {
    const uint32_t node = M.cmap[(uint64_t)l * nv + i];
    const double w = (double)M.weight[l];
    z[0] += w * (double)M.zl[3ull * node];
    z[1] += w * (double)M.zl[3ull * node + 1];
    z[2] += w * (double)M.zl[3ull * node + 2];
  }
}

// Device state of a MAS handle created by ys_mas_create (host side).
const MasDev* mas_device_state(void* handle);

}  // namespace ys
