// Streamed-tile symmetric 3x3-block SpMV: every tile of kTileRows rows reads
// one contiguous run of packed FP32 blocks, one run of entry words and the
// tile's distinct neighbour variables, so the product's only scattered reads
// are the distinct neighbour vectors of each tile, gathered once per tile.
//
// Tile t's stream holds its own stored (upper) blocks [row_block[r0],
// row_block[r1]) in storage order, then the blocks of earlier tiles that its
// rows use transposed (the "cross" blocks, in first-use order), as 9 packed
// floats each (36 bytes: no padding crosses HBM).  An entry word names, for
// one row-plan entry, the entry's neighbour as an index into the tile's
// distinct-column list (bits 0-15), its block as a slot of the tile's stream
// (bits 16-30) and whether the block is used transposed (bit 31).  Blocks,
// entry words and distinct columns of tile t all start at the same base
//   base_t = (row_ptr[r0] + 4 t + 3) & ~3
// in their arrays (each tile holds at most as many stream blocks and
// distinct columns as entries, so the runs never overlap and every run
// starts on a 16-byte boundary); rows[68 t .. 68 t + 64] are the tile's
// local row offsets into its entry words, rows[68 t + 65] its distinct-column
// count.
//
// The kernel: persistent CTAs, a ring of two or three stage buffers (blocks,
// entry words, rows) filled by bulk copies (cp.async.bulk, mbarrier
// completion) one or two tiles ahead; while tile k is computed, the neighbour vectors of tile
// k + 1 are gathered into a second shared-memory buffer by 16-byte cp.async
// copies, one distinct column a thread.  The rows of tile k then read
// blocks, entry words and neighbour vectors from shared memory only.
//
// The arithmetic is that of spmv3_group_accumulate (ys_spmv.cuh): kRowLanes
// lanes a row, lane l takes entries l, l + 8, ... of the row plan in order,
// the same fused multiply-add chains and the same shuffle tree, so the
// result is bit-identical to ys_spmv3_x32.
#pragma once

#include "ys_spmv_tiled.cuh"

namespace ys {

constexpr uint32_t kStreamRowWords = 68;          // 65 row offsets, the distinct-column count, 2 spare
constexpr uint32_t kStreamHaloWord = 65;
constexpr uint32_t kStreamFloats = 9;             // packed block
constexpr uint32_t kStreamMaxStages = 3;
constexpr uint32_t kStreamMaxEntries = 4096;      // plan build: a tile's entries sorted in shared memory
constexpr uint32_t kStreamMaxHalo = kTileThreads; // one distinct column a thread
constexpr uint32_t kStreamMaxSlots = 1u << 15;
constexpr uint32_t kStreamEmpty = 0xffffffffu;    // stream slot without a block (fill leaves it)

static_assert(kTileRows + 1 <= kStreamHaloWord, "row offsets and the distinct-column count share 68 words");

__host__ __device__ inline uint32_t round4(uint32_t x) { return (x + 3u) & ~3u; }

// Words (and stream slots) each per-tile array needs for num_entries
// row-plan entries over num_vars variables.
__host__ __device__ inline uint64_t stream_words(uint64_t num_entries, uint32_t num_vars) {
  const uint64_t ntiles = (num_vars + kTileRows - 1) / kTileRows;
  return (num_entries + 4 * ntiles + 8 + 3) & ~3ull;  // a multiple of 4 (the fill packs four slots a thread)
}

struct StreamSet {
  const float* stream32;    // packed FP32 blocks, tile t's run at base_t
  const uint4* desc;        // per tile: base, stream blocks, entries, distinct columns
  const uint32_t* rows;     // kStreamRowWords per tile
  const uint32_t* words;    // entry words, tile t's at base_t
  const uint32_t* halo;     // distinct columns, tile t's at base_t
  SpmvSet plan;             // the row plan (values32): read instead after a copy wait runs out
  uint32_t nv;
  uint32_t block_cap;       // most stream blocks of one tile, a multiple of 4
  uint32_t entry_cap;       // most entries of one tile, a multiple of 4
  uint32_t halo_cap;        // most distinct columns of one tile, a multiple of 4, <= kStreamMaxHalo
  uint32_t stages;          // stage buffers, 2 or 3
};

inline StreamSet stream_set(const ys_spmv_stream& p, const SpmvSet& plan, uint32_t nv, uint32_t stages) {
  return StreamSet{p.blocks32, reinterpret_cast<const uint4*>(p.desc), p.rows, p.words, p.halo, plan, nv,
                   p.block_cap, p.entry_cap, p.halo_cap, stages};
}

// Bytes of one stage buffer: blocks, entry words, rows.
__host__ __device__ inline uint32_t stream_stage_bytes(uint32_t block_cap, uint32_t entry_cap) {
  return block_cap * 4u * kStreamFloats + 4u * entry_cap + 4u * kStreamRowWords;
}

// Dynamic shared memory of a launch: the stage ring and two neighbour buffers.
inline size_t stream_smem_bytes(uint32_t block_cap, uint32_t entry_cap, uint32_t halo_cap, uint32_t stages) {
  return (size_t)stages * stream_stage_bytes(block_cap, entry_cap) + 2ull * 16u * halo_cap;
}

// Stage count of a launch of `kernel`: the one with more resident CTAs (the
// rows' shared-memory reads are latency-bound, so resident warps come
// first), three on a tie (copies issued two tiles ahead); 0 when neither
// fits.  *per_sm gets the resident CTAs of the choice.
inline uint32_t stream_pick_stages(const void* kernel, uint32_t block_cap, uint32_t entry_cap, uint32_t halo_cap,
                                   int* per_sm) {
  int best = 0;
  uint32_t pick = 0;
  for (uint32_t s = 3; s >= 2; --s) {
    const size_t smem = stream_smem_bytes(block_cap, entry_cap, halo_cap, s);
    int n = 0;
    if (smem > 220u * 1024u || cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                                   cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kTileThreads, smem) != cudaSuccess)
      n = 0;
    if (n > best) {
      best = n;
      pick = s;
    }
  }
  *per_sm = best;
  return pick;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// One row of a staged tile by kRowLanes lanes (every lane of the warp calls
// it; rows beyond the tile with valid == false).
__device__ __forceinline__ void stream_row(const float* __restrict__ blocks, const uint32_t* __restrict__ words,
                                           const uint32_t* __restrict__ rws, const float4* __restrict__ hx,
                                           uint32_t k, bool valid, int lane, double& y0, double& y1, double& y2) {
  const uint32_t e0 = valid ? rws[k] : 0u, e1 = valid ? rws[k + 1] : 0u;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll 2
  for (uint32_t e = e0 + lane; e < e1; e += kRowLanes) {
    const uint32_t w = words[e];
    const float4 xv4 = hx[w & 0xffffu];
    const float* b = blocks + kStreamFloats * ((w >> 16) & 0x7fffu);
    float bv[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) bv[j] = b[j];
    const float xv[3] = {xv4.x, xv4.y, xv4.z};
    block_mac(bv, xv, (w >> 31) != 0u, a0, a1, a2);
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

// Runs every tile t = blockIdx.x + k gridDim.x of the set.  For each row,
// pre(i, valid, lane) runs before the row's products (loads the caller
// needs afterwards are issued early) and out(i, valid, lane, y0, y1, y2)
// after them (all lanes call both; lane 0 of a row group owns the result).
//
// Pipeline of iteration k (S = 2 or 3 stage buffers): thread 0 stages tile
// k + S - 1 (bulk copies into buffer (k + S - 1) % S, last read in
// iteration k - 1); every thread gathers
// its distinct column of tile k + 1 (cp.async, the column read from global
// memory in iteration k - 1, the tile's descriptor in iteration k - 2);
// the rows of tile k run on buffer k % S (its copies waited for here, S - 1
// iterations after their issue) and neighbour buffer k & 1 (gathered in
// iteration k - 1, complete at its closing barrier).
//
// A copy wait that runs out sets *err; the CTA issues no further copies and
// the warps without a completed stage read the row plan from global memory
// (the same values and order: the result stays exact).
template <class Pre, class Out>
__device__ __forceinline__ void spmv3_stream_x32(const StreamSet& T, const float4* __restrict__ x32, unsigned* err,
                                                 Pre&& pre, Out&& out) {
  extern __shared__ float4 stream_smem4[];
  char* const smem = reinterpret_cast<char*>(stream_smem4);
  const uint32_t stage = stream_stage_bytes(T.block_cap, T.entry_cap);
  const uint32_t off_words = T.block_cap * 4u * kStreamFloats;
  const uint32_t off_rows = off_words + 4u * T.entry_cap;
  float4* const hx = reinterpret_cast<float4*>(smem + T.stages * stage);
  __shared__ uint64_t bars[kStreamMaxStages];
  __shared__ int dead;
  __shared__ uint32_t issued;
  __shared__ uint4 nxt;  // descriptor of the next tile to issue (loaded one issue ahead)
  const uint32_t ntiles = (T.nv + kTileRows - 1) / kTileRows;
  const uint32_t mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint32_t g = gridDim.x;
  const uint32_t S = T.stages;
  if (threadIdx.x == 0) {
    for (uint32_t b = 0; b < S; ++b) mbar_init(&bars[b], 1);
    mbar_fence_init();
    dead = 0;
    issued = 0;
    if (mine) nxt = T.desc[blockIdx.x];
  }
  __syncthreads();
  // thread 0: stage this CTA's tile number `issued` into buffer issued % 3
  auto issue = [&]() {
    const uint32_t q = issued;
    const uint32_t t = blockIdx.x + q * g;
    const uint32_t buf = q % S;
    const uint4 d = nxt;
    char* dst = smem + buf * stage;
    const uint32_t nb = round4(d.y) * 4u * kStreamFloats, ne = round4(d.z) * 4u;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bars[buf], nb + ne + 4u * kStreamRowWords);
    if (nb) bulk_copy_g2s(dst, T.stream32 + (uint64_t)kStreamFloats * d.x, nb, &bars[buf]);
    if (ne) bulk_copy_g2s(dst + off_words, T.words + d.x, ne, &bars[buf]);
    bulk_copy_g2s(dst + off_rows, T.rows + (uint64_t)kStreamRowWords * t, 4u * kStreamRowWords, &bars[buf]);
    issued = q + 1;
    if (q + 1 < mine) nxt = T.desc[t + g];
  };
  if (threadIdx.x == 0)
    while (issued < mine && issued < S - 1) issue();
  // the neighbour gather pipeline in registers: this thread's column of
  // the next tile (hid, valid below hnh) and the descriptor (hbase, hnh2)
  // of the tile after it
  uint32_t hid = 0, hnh = 0, hbase2 = 0, hnh2 = 0;
  if (mine) {
    const uint4 d0 = T.desc[blockIdx.x];
    if (threadIdx.x < d0.w) cp_async16(hx + threadIdx.x, x32 + T.halo[d0.x + threadIdx.x]);
    cp_async_commit();
    if (mine > 1) {
      const uint4 d1 = T.desc[blockIdx.x + g];
      hnh = d1.w;
      if (threadIdx.x < hnh) hid = T.halo[d1.x + threadIdx.x];
    }
    if (mine > 2) {
      const uint4 d2 = T.desc[blockIdx.x + 2 * g];
      hbase2 = d2.x;
      hnh2 = d2.w;
    }
    cp_async_wait_all();
  }
  __syncthreads();
  const int lane = (int)(threadIdx.x % kRowLanes);
  const uint32_t row = threadIdx.x / kRowLanes;
  for (uint32_t k = 0; k < mine; ++k) {
    const uint32_t t = blockIdx.x + k * g;
    if (threadIdx.x == 0 && issued < mine && !dead) issue();  // tile k + S - 1
    if (k + 1 < mine && threadIdx.x < hnh) cp_async16(hx + ((k + 1) & 1u) * T.halo_cap + threadIdx.x, x32 + hid);
    cp_async_commit();
    if (k + 2 < mine) {
      hnh = hnh2;
      if (threadIdx.x < hnh) hid = T.halo[hbase2 + threadIdx.x];
    }
    if (k + 3 < mine) {
      const uint4 d3 = T.desc[t + 3 * g];
      hbase2 = d3.x;
      hnh2 = d3.w;
    }
    const uint32_t r0 = t * kTileRows, r1 = min(r0 + kTileRows, T.nv);
    const uint32_t i = r0 + row;
    pre(i, i < r1, lane);
    // tile k was issued unless the CTA stopped staging before its turn
    // (issued only grows, and only while no wait has run out)
    const bool have = k < *reinterpret_cast<volatile uint32_t*>(&issued);
    const bool ok = have && mbar_wait_bounded(&bars[k % S], (k / S) & 1u);
    if (have && !ok) {
      dead = 1;
      atomicOr(err, 1u);
    }
    double y[3];
    // warp-uniform: both paths end in full-warp shuffles
    if (__all_sync(0xffffffffu, ok)) {
      const char* st = smem + (k % S) * stage;
      stream_row(reinterpret_cast<const float*>(st), reinterpret_cast<const uint32_t*>(st + off_words),
                 reinterpret_cast<const uint32_t*>(st + off_rows), hx + (k & 1u) * T.halo_cap, row, i < r1, lane,
                 y[0], y[1], y[2]);
    } else {
      spmv3_group_x32(&T.plan, 1, i, i < r1, lane, x32, y[0], y[1], y[2]);
    }
    out(i, i < r1, lane, y[0], y[1], y[2]);
    cp_async_wait_all();
    __syncthreads();
  }
  // a CTA that stopped staging waits (bounded) for every copy it issued
  // before its shared memory goes away: the last phase of each buffer
  if (dead && threadIdx.x == 0) {
    const uint32_t n = issued;
    for (uint32_t q = n > S ? n - S : 0; q < n; ++q)
      mbar_wait_bounded(&bars[q % S], (q / S) & 1u);
  }
}

}  // namespace ys
