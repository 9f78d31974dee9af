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
constexpr uint32_t kTailNodes = 64;

__host__ __device__ inline uint32_t restrict_tail_first(const MasDev& M) {
  uint32_t first = M.levels;
  while (first > 1 && M.level_node_offset[first] - M.level_node_offset[first - 1] <= kTailNodes) --first;
  return first;
}

// FP32 domain inverses are stored as 4x4 tiles: the n x n inverse is padded
// to 4T rows (T = ceil(n / 4) rounded up to even, zero padding) and its upper
// tiles (A <= B, diagonal tiles in full) are kept, 16 floats a tile, row-major
// inside the tile.  Tile order folds the triangle into a T/2 x (T+1)
// rectangle: rectangle row q holds tile row q (B = q..T-1) followed by tile
// row T-1-q, so a tile's slot and its (A, B) convert with one division.
__host__ __device__ inline uint32_t inv_tiles(uint32_t n) {
  const uint32_t t = (n + 3) / 4;
  return t + (t & 1u);
}
__host__ __device__ inline uint64_t inv_floats(uint32_t n) {
  const uint64_t t = inv_tiles(n);
  return 8ull * t * (t + 1);
}
// slot of tile (A, B) = inv_tile_rowbase(T, A) + B
__host__ __device__ inline uint32_t inv_tile_rowbase(uint32_t T, uint32_t A) {
  if (A < T / 2) return A * T;
  const uint32_t q = T - 1 - A;
  return q * (T + 1) + (T - q) - A;
}
__host__ __device__ inline uint32_t inv_tile_slot(uint32_t T, uint32_t A, uint32_t B) {
  return inv_tile_rowbase(T, A) + B;
}
// Row stride (in float4) of the partial-product grid: >= T and 1 mod 8, so
// the reads of the final row sums and the transposed writes are free of
// shared-memory bank conflicts.
__host__ __device__ inline uint32_t gemv_partial_ld(uint32_t T) { return (T + 6) / 8 * 8 + 1; }
inline size_t gemv_smem_bytes(uint32_t max_dofs) {
  const uint32_t T = inv_tiles(max_dofs);
  return 16ull * (T * gemv_partial_ld(T) + T);
}

// Products of one tile (A, B) (slot `slot`, rows t0..t3) with the staged
// residual: T_AB r_B into cell (A, B) and, off the diagonal, T_AB^T r_A into
// cell (B, A) of the partial grid.
__device__ __forceinline__ void gemv_tile(uint32_t T, uint32_t ld, uint32_t slot, const float4 (&t)[4],
                                          const float4* r4, float4* part) {
  // slot = q (T + 1) + c; the +0.5 keeps the float quotient off integers
  const uint32_t q = (uint32_t)(((float)slot + 0.5f) * (1.0f / (float)(T + 1)));
  const uint32_t c = slot - q * (T + 1);
  const bool first = c < T - q;
  const uint32_t A = first ? q : T - 1 - q;
  const uint32_t B = first ? q + c : A + (c - (T - q));
  const float4 rb = r4[B];
  float4 u;
  u.x = fmaf(t[0].w, rb.w, fmaf(t[0].z, rb.z, fmaf(t[0].y, rb.y, t[0].x * rb.x)));
  u.y = fmaf(t[1].w, rb.w, fmaf(t[1].z, rb.z, fmaf(t[1].y, rb.y, t[1].x * rb.x)));
  u.z = fmaf(t[2].w, rb.w, fmaf(t[2].z, rb.z, fmaf(t[2].y, rb.y, t[2].x * rb.x)));
  u.w = fmaf(t[3].w, rb.w, fmaf(t[3].z, rb.z, fmaf(t[3].y, rb.y, t[3].x * rb.x)));
  part[A * ld + B] = u;
  if (A != B) {
    const float4 ra = r4[A];
    float4 v;
    v.x = fmaf(t[3].x, ra.w, fmaf(t[2].x, ra.z, fmaf(t[1].x, ra.y, t[0].x * ra.x)));
    v.y = fmaf(t[3].y, ra.w, fmaf(t[2].y, ra.z, fmaf(t[1].y, ra.y, t[0].y * ra.x)));
    v.z = fmaf(t[3].z, ra.w, fmaf(t[2].z, ra.z, fmaf(t[1].z, ra.y, t[0].z * ra.x)));
    v.w = fmaf(t[3].w, ra.w, fmaf(t[2].w, ra.z, fmaf(t[1].w, ra.y, t[0].w * ra.x)));
    part[B * ld + A] = v;
  }
}

// Threads of a domain-GEMV CTA, and the tiles a thread loads before the
// residual is staged (their HBM reads overlap the residual gather); 160 x 2
// covers the 300 tiles of a 96-DoF domain.
constexpr int kGemvThreads = 160;
constexpr int kGemvPrefetch = 2;

// z_d = A_d^-1 r_d for domain d by one CTA.  A thread takes whole tiles
// (four coalesced 16-byte loads straight from HBM, every byte read once):
// tile (A, B) gives T_AB r_B for output tile row A and, off the diagonal,
// T_AB^T r_A for output tile row B.  Every (output row, source tile) pair is
// produced by exactly one tile, into its own cell of a shared-memory grid,
// and each output entry sums its grid row in a fixed order: deterministic.
__device__ __forceinline__ void gemv_domain(const MasDev& M, uint32_t d, float4* smem) {
  const uint32_t nb = M.dom_node_ptr[d], nn = M.dom_node_ptr[d + 1] - nb;
  const uint32_t n = 3 * nn;
  const uint32_t T = inv_tiles(n);
  const uint32_t ld = gemv_partial_ld(T);
  const uint32_t tiles = T * (T + 1) / 2;
  float4* part = smem;         // [T][ld] partial products
  float4* r4 = smem + T * ld;  // r_d, zero beyond n
  const float4* src = reinterpret_cast<const float4*>(M.inverse + M.inv_offset[d]);
  float4 pre[kGemvPrefetch][4];
#pragma unroll
  for (int k = 0; k < kGemvPrefetch; ++k) {
    const uint32_t slot = threadIdx.x + k * blockDim.x;
    if (slot < tiles) {
#pragma unroll
      for (int m = 0; m < 4; ++m) pre[k][m] = __ldg(src + 4ull * slot + m);
    }
  }
  float* rloc = reinterpret_cast<float*>(r4);
  // A domain's node list is normally the consecutive packed ids from nb
  // (domains are numbered level by level over the packed node order): the
  // residual is read there at once, beside the list entry that confirms it
  // (a mismatch takes the listed node), so the gather is not a chain of two
  // dependent loads.  The first entry's node is kept for the store below.
  uint32_t own_node = 0;
  for (uint32_t t = threadIdx.x; t < 4 * T; t += blockDim.x) {
    float v = 0.0f;
    if (t < n) {
      const uint32_t guess = nb + t / 3;
      const float vs = M.rl[3ull * guess + t % 3];
      const uint32_t node = M.dom_nodes[nb + t / 3];
      v = node == guess ? vs : M.rl[3ull * node + t % 3];
      if (t == threadIdx.x) own_node = node;
    }
    rloc[t] = v;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kGemvPrefetch; ++k) {
    const uint32_t slot = threadIdx.x + k * blockDim.x;
    if (slot < tiles) gemv_tile(T, ld, slot, pre[k], r4, part);
  }
  for (uint32_t slot = threadIdx.x + kGemvPrefetch * blockDim.x; slot < tiles; slot += blockDim.x) {
    float4 t[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) t[m] = __ldg(src + 4ull * slot + m);
    gemv_tile(T, ld, slot, t, r4, part);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const float* row = reinterpret_cast<const float*>(part + (i / 4) * ld) + (i % 4);
    float s0 = 0.0f, s1 = 0.0f;
    for (uint32_t y = 0; y < T; y += 2) {  // T is even
      s0 += row[4 * y];
      s1 += row[4 * y + 4];
    }
    const uint32_t node = i == threadIdx.x ? own_node : M.dom_nodes[nb + i / 3];
    M.zl[3ull * node + i % 3] = s0 + s1;
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
