// Tiled symmetric 3x3-block SpMV with FP32 blocks staged in shared memory by
// bulk copies (cp.async.bulk + mbarrier, a ring of stage buffers, persistent
// CTAs).
//
// In the reference's storage every off-diagonal block is stored once (upper)
// and used twice: by its row (B x_c) and, transposed, by its column
// (B^T x_r).  The stored blocks are sorted by (row, col), so the blocks whose
// row lies in a tile of kTileRows consecutive rows form one contiguous range
// [row_block[r0], row_block[r1]) of the value array.  One bulk copy moves that
// range into shared memory; every row of the tile then reads its direct
// blocks and the transposed blocks of rows inside the tile from shared
// memory, and only the transposed blocks of earlier tiles from global memory
// (recent, so mostly L2 hits).  A tile's blocks therefore cross HBM once per
// SpMV instead of once per use, and the scattered 16-byte gathers of the row
// plan become shared-memory loads.
//
// The arithmetic is that of spmv3_group_accumulate (ys_spmv.cuh): kRowLanes
// lanes a row, lane l takes entries l, l + 8, ... of the row plan in order,
// the same fused multiply-add chains and the same shuffle tree, so the
// result is bit-identical to ys_spmv3_x32.
#pragma once

#include "ys_spmv.cuh"

namespace ys {

constexpr uint32_t kTileRows = YS_SPMV_TILE_ROWS;
constexpr int kTileThreads = kTileRows * kRowLanes;  // a thread group of kRowLanes a row
constexpr uint32_t kTileSlotBytes = 4 * kFp32BlockStride;  // one FP32 block slot (48 B)
// try_wait polls before a CTA stops using shared memory (the copies are a
// few tens of KB and land within microseconds; the bound only keeps a stuck
// copy from hanging the device)
constexpr uint32_t kTileWaitPolls = 1u << 22;

struct TiledSet {
  const float* values32;       // 12-float slots, (row, col)-sorted upper blocks
  const uint32_t* row_ptr;     // row plan (ys_spmv_plan_build), num_vars + 4 entries
  const uint32_t* entry_block; // both hold (row_ptr[nv] + 3) & ~3 entries at least
  const uint32_t* entry_col;
  const uint32_t* row_block;   // [nv + 4] first stored block of each row
  uint32_t nv;
  uint32_t tile_cap;           // most blocks of one tile
  uint32_t entry_cap;          // most plan entries of one tile, 4-aligned range
  uint32_t stages;             // stage buffers in shared memory (2 .. kMaxStages)
};

// Words of row_ptr / row_block staged per tile: rows r0 .. r0 + kTileRows
// rounded up to a 16-byte multiple.
constexpr uint32_t kTileRowWords = (kTileRows + 1 + 3) & ~3u;

// Bytes of one stage buffer: the tile's block slots, its plan entries
// (columns, then blocks) and its row pointers (row_ptr, then row_block).
__host__ __device__ inline uint64_t tile_stage_bytes(uint32_t tile_cap, uint32_t entry_cap) {
  return (uint64_t)tile_cap * kTileSlotBytes + 8ull * entry_cap + 8ull * kTileRowWords;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the phase of the given parity.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t k = 0; k < kTileWaitPolls; ++k)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Order this CTA's earlier generic-proxy reads of shared memory before a bulk
// copy (async proxy) overwrites it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Global -> shared bulk copy of `bytes` (multiple of 16, both addresses
// 16-byte aligned) completing on `bar`.  No multicast: the source is this
// GPU's own memory and only this CTA reads the copy.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// A staged block slot: three 16-byte shared loads (the 12-word slot stride
// spreads the 8 lanes of a row group over distinct banks).
__device__ __forceinline__ void load_slot(const float* __restrict__ p, float (&b)[9]) {
  const float4* q = reinterpret_cast<const float4*>(p);
  const float4 v0 = q[0], v1 = q[1], v2 = q[2];
  b[0] = v0.x; b[1] = v0.y; b[2] = v0.z; b[3] = v0.w;
  b[4] = v1.x; b[5] = v1.y; b[6] = v1.z; b[7] = v1.w;
  b[8] = v2.x;
}

// One staged tile: pointers into a stage buffer and the global ranges they
// hold (blocks [b0, ...), plan entries [e0a, ...), rows [r0, ...]).
struct TileStage {
  const float* blocks;
  const uint32_t* cols;
  const uint32_t* eblocks;
  const uint32_t* rptr;
  const uint32_t* rblock;
  uint32_t b0, e0a, r0;
};

__device__ __forceinline__ TileStage stage_view(const TiledSet& T, const float* base, uint32_t r0, uint32_t b0,
                                                uint32_t e0a) {
  TileStage S;
  S.blocks = base;
  S.cols = reinterpret_cast<const uint32_t*>(base + (uint64_t)kFp32BlockStride * T.tile_cap);
  S.eblocks = S.cols + T.entry_cap;
  S.rptr = S.eblocks + T.entry_cap;
  S.rblock = S.rptr + kTileRowWords;
  S.b0 = b0;
  S.e0a = e0a;
  S.r0 = r0;
  return S;
}

// One row of a staged tile by kRowLanes lanes (the arithmetic and entry
// order of spmv3_group_accumulate); every lane of the warp calls it, rows
// beyond the tile with valid == false.  Only the neighbour vector and the
// transposed blocks of earlier tiles come from global memory.
__device__ __forceinline__ void tile_row_staged(const TiledSet& T, const TileStage& S,
                                                const float4* __restrict__ x32, uint32_t i, bool valid, int lane,
                                                double& y0, double& y1, double& y2) {
  uint32_t e0 = 0, e1 = 0, ub = 0, nt = 0;
  if (valid) {
    const uint32_t k = i - S.r0;
    e0 = S.rptr[k];
    e1 = S.rptr[k + 1];
    ub = S.rblock[k];
    nt = (e1 - e0) - (S.rblock[k + 1] - ub);  // transposed entries come first
  }
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  // entries lane, lane + 8, ... in order (the order of the row-plan gather);
  // the next entry's column and neighbour vector are loaded before this
  // entry's product, so one gather is always in flight
  uint32_t e = e0 + lane;
  float xn[3] = {0.f, 0.f, 0.f};
  if (e < e1) load_x(x32, S.cols[e - S.e0a], xn);
#pragma unroll 1
  for (; e < e1; e += kRowLanes) {
    const uint32_t kk = e - e0;
    const bool tr = kk < nt;
    const uint32_t b = tr ? (S.eblocks[e - S.e0a] & 0x7fffffffu) : ub + (kk - nt);
    const float xv[3] = {xn[0], xn[1], xn[2]};
    if (e + kRowLanes < e1) load_x(x32, S.cols[e + kRowLanes - S.e0a], xn);
    float bv[9];
    if (b >= S.b0) load_slot(S.blocks + (uint64_t)kFp32BlockStride * (b - S.b0), bv);
    else load_block(T.values32, b, bv);
    block_mac(bv, xv, tr, a0, a1, a2);
  }
#pragma unroll
  for (int o = kRowLanes / 2; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o, kRowLanes);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o, kRowLanes);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o, kRowLanes);
  }
  y0 = (double)a0;
  y1 = (double)a1;
  y2 = (double)a2;
}

// Stage buffers of a tiled launch (2 .. kMaxStages) and their shared memory.
constexpr uint32_t kMaxStages = 4;
inline size_t tile_smem_bytes(uint32_t tile_cap, uint32_t entry_cap, uint32_t stages) {
  return (size_t)stages * tile_stage_bytes(tile_cap, entry_cap);
}

// Stage count of a launch: the kernel is bound by the latency of its
// gathers, so resident warps come first: the most stages (up to kMaxStages,
// at least two) that still let the thread limit's worth of CTAs share an SM.
inline uint32_t tile_auto_stages(uint32_t tile_cap, uint32_t entry_cap, size_t smem_per_sm) {
  const size_t one = tile_stage_bytes(tile_cap, entry_cap);
  const size_t ctas = 2048 / kTileThreads;
  uint32_t s = kMaxStages;
  while (s > 2 && ctas * (s * one + 1024) > smem_per_sm) --s;
  return s;
}

// Runs every tile t = blockIdx.x + k gridDim.x of the set through a ring of
// `stages` stage buffers (tile k is staged in buffer k % stages, up to
// stages - 1 tiles ahead of the one being computed);
// out(i, valid, lane, y0, y1, y2) receives each row (all lanes call it, lane
// 0 of a row group owns the result).  A bulk-copy wait that runs out sets
// *err and the CTA reads global memory from then on through the row-plan
// gather (the same values and order: the result stays exact).
template <class Out>
__device__ __forceinline__ void spmv3_tiles_x32(const TiledSet& T, const float4* __restrict__ x32, unsigned* err,
                                                Out&& out) {
  const uint32_t stages = T.stages;
  extern __shared__ float4 tile_stage4[];
  float* stage_base = reinterpret_cast<float*>(tile_stage4);
  const uint64_t buf_floats = tile_stage_bytes(T.tile_cap, T.entry_cap) / 4;
  __shared__ uint64_t bars[kMaxStages];
  __shared__ int dead;
  const uint32_t ntiles = (T.nv + kTileRows - 1) / kTileRows;
  if (threadIdx.x == 0) {
    for (uint32_t b = 0; b < stages; ++b) mbar_init(&bars[b], 1);
    mbar_fence_init();
    dead = 0;
  }
  __syncthreads();
  const uint32_t mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // thread 0's pipeline state lives in shared memory (the other threads need
  // no registers for it): tiles issued so far, and the bounds of the next
  // tile to issue, loaded one issue ahead so the copy is not held up by
  // their latency
  __shared__ uint32_t issued;
  __shared__ uint32_t nxt[4];  // row_block[r0], row_block[r1], row_ptr[r0], row_ptr[r1]
  auto load_bounds = [&](uint32_t q) {
    if (q >= mine) return;
    const uint32_t r0 = (blockIdx.x + q * gridDim.x) * kTileRows, r1 = min(r0 + kTileRows, T.nv);
    nxt[0] = __ldg(T.row_block + r0);
    nxt[1] = __ldg(T.row_block + r1);
    nxt[2] = __ldg(T.row_ptr + r0);
    nxt[3] = __ldg(T.row_ptr + r1);
  };
  if (threadIdx.x == 0) {
    issued = 0;
    load_bounds(0);
  }
  // thread 0: stage this CTA's tile number `q` (t = blockIdx.x + q gridDim.x)
  // into buffer q % stages: its blocks, its plan entries (a 16-byte aligned
  // range) and its row pointers, one mbarrier phase
  auto issue = [&]() {
    const uint32_t q = issued;
    const uint32_t t = blockIdx.x + q * gridDim.x;
    const uint32_t buf = q % stages;
    const uint32_t r0 = t * kTileRows, r1 = min(r0 + kTileRows, T.nv);
    // block slots are 48 bytes; entries move in 4-entry groups: 16-byte aligned
    const uint32_t b0 = nxt[0], b1 = nxt[1], e0a = nxt[2] & ~3u, e1a = (nxt[3] + 3u) & ~3u;
    // rows r0 .. r1 (inclusive) rounded up to 4 words: at most num_vars + 4
    const uint32_t vb = (b1 - b0) * kTileSlotBytes, eb = (e1a - e0a) * 4u, rb = ((r1 - r0 + 4u) & ~3u) * 4u;
    float* dst = stage_base + buf * buf_floats;
    const TileStage S = stage_view(T, dst, r0, b0, e0a);
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bars[buf], vb + 2 * eb + 2 * rb);
    if (vb) bulk_copy_g2s(dst, T.values32 + (uint64_t)kFp32BlockStride * b0, vb, &bars[buf]);
    if (eb) {
      bulk_copy_g2s((void*)S.cols, T.entry_col + e0a, eb, &bars[buf]);
      bulk_copy_g2s((void*)S.eblocks, T.entry_block + e0a, eb, &bars[buf]);
    }
    bulk_copy_g2s((void*)S.rptr, T.row_ptr + r0, rb, &bars[buf]);
    bulk_copy_g2s((void*)S.rblock, T.row_block + r0, rb, &bars[buf]);
    issued = q + 1;
    load_bounds(q + 1);
  };
  if (threadIdx.x == 0)
    while (issued < mine && issued + 1 < stages) issue();
  __syncthreads();
  static_assert(kTileRows * kRowLanes == kTileThreads, "one row a thread group");
  const int lane = (int)(threadIdx.x % kRowLanes);
  for (uint32_t k = 0; k < mine; ++k) {
    const uint32_t t = blockIdx.x + k * gridDim.x;
    const uint32_t buf = k % stages;
    // buffer (k + stages - 1) % stages was last read in iteration k - 1
    if (threadIdx.x == 0 && issued < mine && !dead) issue();
    const uint32_t r0 = t * kTileRows, r1 = min(r0 + kTileRows, T.nv);
    const uint32_t iA = r0 + threadIdx.x / kRowLanes;
    double yA[3];
    // tile k is the (k / stages)-th phase of its buffer
    bool staged = !dead;
    if (staged && !mbar_wait_bounded(&bars[buf], (k / stages) & 1u)) {
      staged = false;
      dead = 1;  // no further copies into this CTA's buffers
      atomicOr(err, 1u);
    }
    if (staged) {
      const float* base = stage_base + buf * buf_floats;
      const uint32_t* rblk = reinterpret_cast<const uint32_t*>(base + (uint64_t)kFp32BlockStride * T.tile_cap) +
                             2ull * T.entry_cap + kTileRowWords;
      const uint32_t* rp = rblk - kTileRowWords;
      const TileStage S = stage_view(T, base, r0, rblk[0], rp[0] & ~3u);
      tile_row_staged(T, S, x32, iA, iA < r1, lane, yA[0], yA[1], yA[2]);
    } else {
      SpmvSet g{nullptr, T.values32, T.row_ptr, T.entry_block, T.entry_col};
      spmv3_group_x32(&g, 1, iA, iA < r1, lane, x32, yA[0], yA[1], yA[2]);
    }
    out(iA, iA < r1, lane, yA[0], yA[1], yA[2]);
    __syncthreads();
  }
  // a CTA that stopped staging waits (bounded) for every copy it issued
  // before its shared memory goes away: the last phase of each buffer
  if (dead && threadIdx.x == 0) {
    const uint32_t n = issued;
    for (uint32_t q = n > stages ? n - stages : 0; q < n; ++q)
      mbar_wait_bounded(&bars[q % stages], (q / stages) & 1u);
  }
}

}  // namespace ys
