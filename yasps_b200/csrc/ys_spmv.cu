// Row plan build and the standalone symmetric 3x3-block SpMV.
#include <cub/cub.cuh>

#include "ys_spmv.cuh"
#include "ys_spmv_stream.cuh"

namespace ys {

__global__ void spmv_entries_kernel(const uint32_t* __restrict__ pos, uint32_t nu, uint64_t* __restrict__ keys,
                                    uint32_t* __restrict__ vals, uint32_t* __restrict__ counts,
                                    uint32_t* __restrict__ bad) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nu) return;
  const uint32_t r = pos[2ull * b], c = pos[2ull * b + 1];
  if ((r % 3) || (c % 3)) { atomicOr(bad, 1u); }
  const uint32_t ri = r / 3, ci = c / 3;
  // Direct entry in row ri at slot 2b, transposed entry in row ci at slot 2b+1.
  keys[2ull * b] = ((uint64_t)ri << 32) | ci;
  vals[2ull * b] = b;
  atomicAdd(counts + ri, 1u);
  if (r != c) {
    keys[2ull * b + 1] = ((uint64_t)ci << 32) | ri;
    vals[2ull * b + 1] = b | 0x80000000u;
    atomicAdd(counts + ci, 1u);
  } else {
    keys[2ull * b + 1] = ~0ull;  // sorts last, dropped
    vals[2ull * b + 1] = 0xffffffffu;
  }
}

__global__ void spmv_split_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals, uint32_t n,
                                  uint32_t* __restrict__ eblock, uint32_t* __restrict__ ecol) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  eblock[p] = vals[p];
  ecol[p] = (uint32_t)(keys[p] & 0xffffffffu);
}

__global__ void __launch_bounds__(256) spmv3_kernel(SpmvSet set, bool fp32, uint32_t nv, const double* __restrict__ x,
                                                    double* __restrict__ y, int beta) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t i = t / kRowLanes;
  const int lane = (int)(t % kRowLanes);
  double y0, y1, y2;
  spmv3_group(&set, 1, fp32, i, i < nv, lane, x, y0, y1, y2);
  if (i >= nv || lane != 0) return;
  if (beta) {
    y0 += y[3ull * i];
    y1 += y[3ull * i + 1];
    y2 += y[3ull * i + 2];
  }
  y[3ull * i] = y0;
  y[3ull * i + 1] = y1;
  y[3ull * i + 2] = y2;
}

// FP32 block values with the float4 copy of x (the layout of the FP32 PCG loop).
__global__ void __launch_bounds__(256) spmv3_x32_kernel(SpmvSet set, uint32_t nv, const float4* __restrict__ x32,
                                                        double* __restrict__ y, int beta) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t i = t / kRowLanes;
  const int lane = (int)(t % kRowLanes);
  double y0, y1, y2;
  spmv3_group_x32(&set, 1, i, i < nv, lane, x32, y0, y1, y2);
  if (i >= nv || lane != 0) return;
  if (beta) {
    y0 += y[3ull * i];
    y1 += y[3ull * i + 1];
    y2 += y[3ull * i + 2];
  }
  y[3ull * i] = y0;
  y[3ull * i + 1] = y1;
  y[3ull * i + 2] = y2;
}

__global__ void pack_x32_kernel(const double* __restrict__ x, uint32_t nv, float4* __restrict__ x32) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  x32[i] = make_float4((float)x[3ull * i], (float)x[3ull * i + 1], (float)x[3ull * i + 2], 0.0f);
}

// row_block[i] = first stored block whose scalar row offset is >= 3 i
// (i = 0 .. nv): a binary search over the (row, col)-sorted positions.
__global__ void tile_row_block_kernel(const uint32_t* __restrict__ pos, uint32_t nu, uint32_t nv,
                                      uint32_t* __restrict__ row_block) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nv) return;
  const uint64_t key = 3ull * i;
  uint32_t lo = 0, hi = nu;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if ((uint64_t)pos[2ull * mid] < key) lo = mid + 1;
    else hi = mid;
  }
  row_block[i] = lo;
}

// Checks that row i's direct plan entries are the blocks row_block[i] ..
// row_block[i+1] - 1 in order after its transposed entries, and records the
// largest tile (scratch[0]: mismatch flag, scratch[1]: most blocks of a tile,
// scratch[2]: most plan entries of a tile's 16-byte aligned entry range).
__global__ void tile_check_kernel(const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ eblock,
                                  const uint32_t* __restrict__ row_block, uint32_t nv,
                                  uint32_t* __restrict__ scratch) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  const uint32_t e0 = row_ptr[i], e1 = row_ptr[i + 1];
  const uint32_t ub = row_block[i], nd = row_block[i + 1] - ub;
  if (row_block[i + 1] < ub || nd > e1 - e0) {
    atomicOr(scratch, 1u);
    return;
  }
  const uint32_t nt = (e1 - e0) - nd;
  for (uint32_t k = 0; k < e1 - e0; ++k) {
    const uint32_t eb = eblock[e0 + k];
    const bool ok = k < nt ? (eb & 0x80000000u) != 0 : eb == ub + (k - nt);
    if (!ok) {
      atomicOr(scratch, 1u);
      return;
    }
  }
  if (i % kTileRows == 0) {
    const uint32_t r1 = min(i + kTileRows, nv);
    atomicMax(scratch + 1, row_block[r1] - ub);
    atomicMax(scratch + 2, ((row_ptr[r1] + 3u) & ~3u) - (e0 & ~3u));
  }
}

// No tile_stage_status given: the flag goes to this word.
__device__ unsigned g_tile_stage_status;

__global__ void __launch_bounds__(kTileThreads) spmv3_x32_tiled_kernel(TiledSet T, const float4* __restrict__ x32,
                                                                      double* __restrict__ y, int beta,
                                                                      unsigned* status) {
  unsigned* err = status ? status : &g_tile_stage_status;
  spmv3_tiles_x32(T, x32, err, [&](uint32_t i, bool valid, int lane, double y0, double y1, double y2) {
    if (!valid || lane != 0) return;
    if (beta) {
      y0 += y[3ull * i];
      y1 += y[3ull * i + 1];
      y2 += y[3ull * i + 2];
    }
    y[3ull * i] = y0;
    y[3ull * i + 1] = y1;
    y[3ull * i + 2] = y2;
  });
}

// ---- streamed tiles (ys_spmv_stream.cuh) ------------------------------------

// Exclusive block-wide prefix sum over kTileThreads threads; *total gets the sum.
__device__ __forceinline__ uint32_t tile_scan_exclusive(uint32_t v, uint32_t* wsum, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int w = 0; w < kTileThreads / 32; ++w) {
      const uint32_t c = wsum[w];
      wsum[w] = acc;
      acc += c;
    }
    wsum[kTileThreads / 32] = acc;
  }
  __syncthreads();
  const uint32_t r = wsum[warp] + x - v;
  *total = wsum[kTileThreads / 32];
  __syncthreads();
  return r;
}

// One CTA a tile: the tile's distinct columns (its entry columns sorted in
// shared memory, duplicates dropped), the cross blocks (transposed entries
// whose block belongs to an earlier tile) numbered in entry order after the
// tile's own blocks, and the entry words, row offsets, stream sources and
// descriptor of the tile.  caps[0] |= 1: a tile has more entries than the
// sort holds; |= 2: more distinct columns or stream slots than the kernel
// takes; |= 4: the blocks are not (row, col)-sorted along the row plan.
// caps[1..3]: the most stream blocks, entries and distinct columns of a
// tile, each rounded up to a multiple of 4.
__global__ void __launch_bounds__(kTileThreads) stream_plan_kernel(
    const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ entry_block,
    const uint32_t* __restrict__ entry_col, const uint32_t* __restrict__ row_block, uint32_t nv,
    uint4* __restrict__ desc, uint32_t* __restrict__ rows, uint32_t* __restrict__ words, uint32_t* __restrict__ halo,
    uint32_t* __restrict__ src, uint32_t* __restrict__ slot_of, uint32_t* __restrict__ caps) {
  __shared__ uint32_t key[kStreamMaxEntries];
  __shared__ uint32_t uniq[kStreamMaxEntries];
  __shared__ uint32_t wsum[kTileThreads / 32 + 1];
  constexpr uint32_t kPer = kStreamMaxEntries / kTileThreads;  // consecutive items a thread
  const uint32_t t = blockIdx.x;
  const uint32_t r0 = t * kTileRows, r1 = min(r0 + kTileRows, nv);
  const uint32_t p0 = row_ptr[r0], ne = row_ptr[r1] - p0;
  const uint32_t base = (p0 + 4u * t + 3u) & ~3u;
  const uint32_t b0 = row_block[r0], b1 = row_block[r1];
  // (a tile holds at most one own block per entry: otherwise the plan does
  // not match the blocks, and nothing is written)
  if (ne > kStreamMaxEntries || b1 < b0 || b1 - b0 > ne) {
    if (threadIdx.x == 0) atomicOr(caps, ne > kStreamMaxEntries ? 1u : 4u);
    return;
  }
  const uint32_t own = b1 - b0;
  uint32_t n = 1;
  while (n < ne) n <<= 1;
  for (uint32_t j = threadIdx.x; j < n; j += kTileThreads) key[j] = j < ne ? entry_col[p0 + j] : 0xffffffffu;
  __syncthreads();
  for (uint32_t size = 2; size <= n; size <<= 1)
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t j = threadIdx.x; j < n; j += kTileThreads) {
        const uint32_t q = j ^ stride;
        if (q > j) {
          const uint32_t a = key[j], b = key[q];
          if ((a > b) == ((j & size) == 0)) {
            key[j] = b;
            key[q] = a;
          }
        }
      }
      __syncthreads();
    }
  // distinct columns in ascending order
  const uint32_t j0 = threadIdx.x * kPer;
  uint32_t cnt = 0;
  for (uint32_t q = 0; q < kPer; ++q) {
    const uint32_t j = j0 + q;
    cnt += (j < ne && (j == 0 || key[j] != key[j - 1])) ? 1u : 0u;
  }
  uint32_t nh = 0;
  uint32_t at = tile_scan_exclusive(cnt, wsum, &nh);
  for (uint32_t q = 0; q < kPer; ++q) {
    const uint32_t j = j0 + q;
    if (j < ne && (j == 0 || key[j] != key[j - 1])) uniq[at++] = key[j];
  }
  // cross blocks, numbered in entry order
  cnt = 0;
  for (uint32_t q = 0; q < kPer; ++q) {
    const uint32_t j = j0 + q;
    if (j < ne) {
      const uint32_t eb = entry_block[p0 + j];
      cnt += ((eb >> 31) && (eb & 0x7fffffffu) < b0) ? 1u : 0u;
    }
  }
  uint32_t ncross = 0;
  uint32_t rank = tile_scan_exclusive(cnt, wsum, &ncross);  // ends with a barrier: uniq is complete
  const uint32_t nslots = own + ncross;
  int bad = 0;
  for (uint32_t q = 0; q < kPer; ++q) {
    const uint32_t j = j0 + q;
    if (j >= ne) break;
    const uint32_t eb = entry_block[p0 + j], col = entry_col[p0 + j];
    const uint32_t tr = eb >> 31, blk = eb & 0x7fffffffu;
    const bool cross = tr && blk < b0;
    if (!cross && (blk < b0 || blk >= b1)) bad = 1;
    const uint32_t slot = cross ? own + rank++ : blk - b0;
    uint32_t lo = 0, hi = nh;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (uniq[mid] < col) lo = mid + 1;
      else hi = mid;
    }
    words[base + j] = lo | ((slot & 0x7fffu) << 16) | (tr << 31);
    if (cross && slot < ne) {
      src[base + slot] = blk;
      slot_of[2ull * blk + 1] = base + slot;  // a block is used transposed by one row only
    }
  }
  if (threadIdx.x < 4 && ne + threadIdx.x < round4(ne)) words[base + ne + threadIdx.x] = 0u;
  for (uint32_t b = b0 + threadIdx.x; b < b1; b += kTileThreads) {
    src[base + (b - b0)] = b;
    slot_of[2ull * b] = base + (b - b0);
  }
  for (uint32_t j = threadIdx.x; j < round4(nh); j += kTileThreads) halo[base + j] = j < nh ? uniq[j] : uniq[0];
  for (uint32_t k = threadIdx.x; k < kStreamRowWords; k += kTileThreads)
    rows[(uint64_t)kStreamRowWords * t + k] =
        k <= kTileRows ? row_ptr[min(r0 + k, r1)] - p0 : (k == kStreamHaloWord ? nh : 0u);
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) {
    desc[t] = make_uint4(base, nslots, ne, nh);
    if (bad) atomicOr(caps, 4u);
    if (nh > kStreamMaxHalo || nslots > kStreamMaxSlots) atomicOr(caps, 2u);
    atomicMax(caps + 1, round4(nslots));
    atomicMax(caps + 2, round4(ne));
    atomicMax(caps + 3, round4(nh));
  }
}

// stream32[9 s + k] = values32[12 src[s] + k] for every slot with a block,
// four slots a thread (36 floats: nine 16-byte stores; slots without a block
// get zeros, which no entry reads).  slots is a multiple of 4.
__global__ void stream_fill_kernel(const float* __restrict__ values32, const uint32_t* __restrict__ src,
                                   uint64_t slots, float* __restrict__ stream32) {
  const uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (4 * q >= slots) return;
  const uint4 b = reinterpret_cast<const uint4*>(src)[q];
  const uint32_t bs[4] = {b.x, b.y, b.z, b.w};
  float v[36];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float w[9];
    if (bs[k] != kStreamEmpty) {
      load_block(values32, bs[k], w);
    } else {
#pragma unroll
      for (int j = 0; j < 9; ++j) w[j] = 0.0f;
    }
#pragma unroll
    for (int j = 0; j < 9; ++j) v[9 * k + j] = w[j];
  }
  float4* o = reinterpret_cast<float4*>(stream32 + 36ull * q);
#pragma unroll
  for (int j = 0; j < 9; ++j) o[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
}

__device__ unsigned g_stream_stage_status;

__global__ void __launch_bounds__(kTileThreads, 3) spmv3_x32_stream_kernel(StreamSet T, const float4* __restrict__ x32,
                                                                          double* __restrict__ y, int beta,
                                                                          unsigned* status) {
  unsigned* err = status ? status : &g_stream_stage_status;
  double old[3] = {0.0, 0.0, 0.0};
  spmv3_stream_x32(
      T, x32, err,
      [&](uint32_t i, bool valid, int lane) {
        if (beta && valid && lane == 0)
          for (int c = 0; c < 3; ++c) old[c] = y[3ull * i + c];
      },
      [&](uint32_t i, bool valid, int lane, double y0, double y1, double y2) {
        if (!valid || lane != 0) return;
        if (beta) {
          y0 += old[0];
          y1 += old[1];
          y2 += old[2];
        }
        y[3ull * i] = y0;
        y[3ull * i + 1] = y1;
        y[3ull * i + 2] = y2;
      });
}

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

static size_t spmv_cub_bytes(uint32_t n2, uint32_t nv) {
  size_t a = 0, b = 0;
  cub::DoubleBuffer<uint64_t> k(nullptr, nullptr);
  cub::DoubleBuffer<uint32_t> v(nullptr, nullptr);
  cub::DeviceRadixSort::SortPairs(nullptr, a, k, v, (int)n2);
  cub::DeviceScan::ExclusiveSum(nullptr, b, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)nv + 1);
  return std::max(a, b);
}

static size_t spmv_ws_bytes(uint32_t nu, uint32_t nv) {
  const uint64_t n2 = 2ull * (nu > 0 ? nu : 1);
  return 2 * align256(8 * n2) + 2 * align256(4 * n2) + align256(4ull * (nv + 1)) + align256(16) +
         align256(spmv_cub_bytes((uint32_t)n2, nv));
}

}  // namespace ys

extern "C" {

int32_t ys_spmv_plan_workspace_bytes(uint32_t nu, uint32_t num_vars, uint64_t* bytes) {
  *bytes = ys::spmv_ws_bytes(nu, num_vars);
  return YS_OK;
}

int32_t ys_spmv_plan_build(const uint32_t* positions, uint32_t nu, uint32_t num_vars, void* workspace,
                           uint64_t workspace_bytes, uint32_t* row_ptr, uint32_t* entry_block, uint32_t* entry_col,
                           void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  YS_REQUIRE(nu < 0x40000000u, YS_ERR_INVALID, "too many blocks");
  YS_REQUIRE(workspace_bytes >= ys::spmv_ws_bytes(nu, num_vars), YS_ERR_CAPACITY, "spmv plan workspace too small");
  YS_CUDA_TRY(cudaMemsetAsync(row_ptr, 0, 4ull * (num_vars + 1), s));
  if (nu == 0) return YS_OK;
  const uint32_t n2 = 2 * nu;
  char* p = (char*)workspace;
  auto take = [&](size_t bytes) { void* r = p; p += ys::align256(bytes); return r; };
  uint64_t* k0 = (uint64_t*)take(8ull * n2);
  uint64_t* k1 = (uint64_t*)take(8ull * n2);
  uint32_t* v0 = (uint32_t*)take(4ull * n2);
  uint32_t* v1 = (uint32_t*)take(4ull * n2);
  uint32_t* counts = (uint32_t*)take(4ull * (num_vars + 1));
  uint32_t* bad = (uint32_t*)take(16);
  size_t cub_bytes = ys::spmv_cub_bytes(n2, num_vars);
  void* tmp = take(cub_bytes);
  YS_CUDA_TRY(cudaMemsetAsync(counts, 0, 4ull * (num_vars + 1), s));
  YS_CUDA_TRY(cudaMemsetAsync(bad, 0, 4, s));
  ys::spmv_entries_kernel<<<ys::grid_for(nu, 256), 256, 0, s>>>(positions, nu, k0, v0, counts, bad);
  YS_CHECK_LAUNCH();
  cub::DoubleBuffer<uint64_t> kb(k0, k1);
  cub::DoubleBuffer<uint32_t> vb(v0, v1);
  size_t tb = cub_bytes;
  YS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, kb, vb, (int)n2, 0, 64, s));
  tb = cub_bytes;
  YS_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tb, counts, row_ptr, (int)num_vars + 1, s));
  uint32_t total = 0, hbad = 0;
  YS_CUDA_TRY(cudaMemcpyAsync(&total, row_ptr + num_vars, 4, cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaStreamSynchronize(s));
  YS_REQUIRE(hbad == 0, YS_ERR_INVALID, "block positions are not 3-aligned");
  ys::spmv_split_kernel<<<ys::grid_for(total, 256), 256, 0, s>>>(kb.Current(), vb.Current(), total, entry_block,
                                                                   entry_col);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_spmv3(const double* values, const float* values32, const uint32_t* row_ptr, const uint32_t* entry_block,
                 const uint32_t* entry_col, uint32_t num_vars, const double* x, double* y, int32_t beta,
                 void* stream) {
  YS_REQUIRE((values == nullptr) != (values32 == nullptr), YS_ERR_INVALID, "pass exactly one of values/values32");
  if (num_vars == 0) return YS_OK;
  ys::SpmvSet set{values, values32, row_ptr, entry_block, entry_col};
  ys::spmv3_kernel<<<ys::grid_for((uint64_t)num_vars * ys::kRowLanes, 256), 256, 0, (cudaStream_t)stream>>>(
      set, values32 != nullptr, num_vars, x, y, beta);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_pack_x32(const double* x, uint32_t num_vars, float* x32, void* stream) {
  YS_REQUIRE((reinterpret_cast<uintptr_t>(x32) & 15) == 0, YS_ERR_INVALID, "x32 must be 16-byte aligned");
  if (num_vars == 0) return YS_OK;
  ys::pack_x32_kernel<<<ys::grid_for(num_vars, 256), 256, 0, (cudaStream_t)stream>>>(
      x, num_vars, reinterpret_cast<float4*>(x32));
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_spmv3_x32(const float* values32, const uint32_t* row_ptr, const uint32_t* entry_block,
                     const uint32_t* entry_col, uint32_t num_vars, const float* x32, double* y, int32_t beta,
                     void* stream) {
  YS_REQUIRE(values32 && x32, YS_ERR_INVALID, "null argument");
  YS_REQUIRE((reinterpret_cast<uintptr_t>(x32) & 15) == 0 && (reinterpret_cast<uintptr_t>(values32) & 15) == 0,
             YS_ERR_INVALID, "values32 and x32 must be 16-byte aligned");
  if (num_vars == 0) return YS_OK;
  ys::SpmvSet set{nullptr, values32, row_ptr, entry_block, entry_col};
  ys::spmv3_x32_kernel<<<ys::grid_for((uint64_t)num_vars * ys::kRowLanes, 256), 256, 0, (cudaStream_t)stream>>>(
      set, num_vars, reinterpret_cast<const float4*>(x32), y, beta);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

}  // extern "C"

extern "C" {

int32_t ys_spmv_tile_plan(const uint32_t* positions, uint32_t nu, const uint32_t* row_ptr,
                          const uint32_t* entry_block, uint32_t num_vars, uint32_t* row_block,
                          uint32_t* tile_cap_host, uint32_t* entry_cap_host, void* stream) {
  YS_REQUIRE(row_block && tile_cap_host && entry_cap_host, YS_ERR_INVALID, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  *tile_cap_host = 0;
  *entry_cap_host = 0;
  uint32_t* scratch = row_block + num_vars + 1;
  YS_CUDA_TRY(cudaMemsetAsync(scratch, 0, 3 * sizeof(uint32_t), s));
  ys::tile_row_block_kernel<<<ys::grid_for(num_vars + 1ull, 256), 256, 0, s>>>(positions, nu, num_vars, row_block);
  YS_CHECK_LAUNCH();
  if (num_vars) {
    ys::tile_check_kernel<<<ys::grid_for(num_vars, 256), 256, 0, s>>>(row_ptr, entry_block, row_block, num_vars,
                                                                      scratch);
    YS_CHECK_LAUNCH();
  }
  uint32_t h[3] = {0, 0, 0};
  YS_CUDA_TRY(cudaMemcpyAsync(h, scratch, sizeof(h), cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaStreamSynchronize(s));
  YS_REQUIRE(h[0] == 0, YS_ERR_INVALID, "blocks are not (row, col)-sorted along the row plan");
  *tile_cap_host = h[1];
  *entry_cap_host = h[2];
  return YS_OK;
}

int32_t ys_spmv3_x32_tiled(const float* values32, const uint32_t* row_ptr, const uint32_t* entry_block,
                           const uint32_t* entry_col, const uint32_t* row_block, uint32_t tile_cap,
                           uint32_t entry_cap, uint32_t stages, uint32_t num_vars, const float* x32, double* y,
                           int32_t beta, uint32_t* stage_status, void* stream) {
  YS_REQUIRE(stages == 0 || (stages >= 2 && stages <= ys::kMaxStages), YS_ERR_INVALID, "stages: 0 (auto) or 2..4");
  YS_REQUIRE(values32 && x32 && row_block && tile_cap > 0 && entry_cap > 0 && (entry_cap & 3u) == 0,
             YS_ERR_INVALID, "null argument or no tile plan");
  YS_REQUIRE((reinterpret_cast<uintptr_t>(x32) & 15) == 0 && (reinterpret_cast<uintptr_t>(values32) & 15) == 0,
             YS_ERR_INVALID, "values32 and x32 must be 16-byte aligned");
  if (num_vars == 0) return YS_OK;
  int dev = 0, sms = 0, per_sm = 0, smem_sm = 0;
  YS_CUDA_TRY(cudaGetDevice(&dev));
  YS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  YS_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  if (stages == 0) stages = ys::tile_auto_stages(tile_cap, entry_cap, (size_t)smem_sm);
  const size_t smem = ys::tile_smem_bytes(tile_cap, entry_cap, stages);
  YS_REQUIRE(smem <= 200u * 1024u, YS_ERR_CAPACITY, "a tile's blocks exceed the shared-memory stage");
  YS_CUDA_TRY(cudaFuncSetAttribute(ys::spmv3_x32_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  YS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ys::spmv3_x32_tiled_kernel, ys::kTileThreads,
                                                            smem));
  YS_REQUIRE(per_sm > 0, YS_ERR_CAPACITY, "tiled SpMV does not fit on an SM");
  const uint32_t ntiles = (num_vars + ys::kTileRows - 1) / ys::kTileRows;
  const unsigned grid = std::min<unsigned>(ntiles, (unsigned)(sms * per_sm));
  ys::TiledSet T{values32, row_ptr, entry_block, entry_col, row_block, num_vars, tile_cap, entry_cap, stages};
  ys::spmv3_x32_tiled_kernel<<<grid, ys::kTileThreads, smem, (cudaStream_t)stream>>>(
      T, reinterpret_cast<const float4*>(x32), y, beta, stage_status);
  YS_CHECK_LAUNCH();
  return YS_OK;
}


int32_t ys_spmv_stream_words(uint32_t num_entries, uint32_t num_vars, uint64_t* words) {
  YS_REQUIRE(words, YS_ERR_INVALID, "null argument");
  *words = ys::stream_words(num_entries, num_vars);
  return YS_OK;
}

int32_t ys_spmv_stream_plan(const uint32_t* row_ptr, const uint32_t* entry_block, const uint32_t* entry_col,
                            const uint32_t* row_block, uint32_t num_vars, uint64_t capacity_words, uint32_t* desc,
                            uint32_t* rows, uint32_t* words, uint32_t* halo, uint32_t* src, uint32_t num_blocks,
                            uint32_t* slot_of, uint32_t* caps_host, void* stream) {
  YS_REQUIRE(row_ptr && entry_block && entry_col && row_block && desc && rows && words && halo && src && slot_of &&
                 caps_host,
             YS_ERR_INVALID, "null argument");
  YS_REQUIRE((reinterpret_cast<uintptr_t>(words) & 15) == 0 && (reinterpret_cast<uintptr_t>(halo) & 15) == 0 &&
                 (reinterpret_cast<uintptr_t>(rows) & 15) == 0 && (reinterpret_cast<uintptr_t>(desc) & 15) == 0,
             YS_ERR_INVALID, "desc, rows, words and halo must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  caps_host[0] = caps_host[1] = caps_host[2] = 0;
  if (num_vars == 0) return YS_OK;
  uint32_t total = 0;
  YS_CUDA_TRY(cudaMemcpyAsync(&total, row_ptr + num_vars, 4, cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaStreamSynchronize(s));
  YS_REQUIRE(capacity_words >= ys::stream_words(total, num_vars), YS_ERR_CAPACITY, "stream plan arrays too small");
  const uint32_t ntiles = (num_vars + ys::kTileRows - 1) / ys::kTileRows;
  uint32_t* caps = desc + 4ull * ntiles;  // the descriptor array's last uint4
  YS_CUDA_TRY(cudaMemsetAsync(caps, 0, 16, s));
  YS_CUDA_TRY(cudaMemsetAsync(src, 0xff, 4ull * capacity_words, s));
  YS_CUDA_TRY(cudaMemsetAsync(slot_of, 0xff, 8ull * num_blocks, s));
  ys::stream_plan_kernel<<<ntiles, ys::kTileThreads, 0, s>>>(row_ptr, entry_block, entry_col, row_block, num_vars,
                                                            reinterpret_cast<uint4*>(desc), rows, words, halo, src,
                                                            slot_of, caps);
  YS_CHECK_LAUNCH();
  uint32_t h[4] = {0, 0, 0, 0};
  YS_CUDA_TRY(cudaMemcpyAsync(h, caps, sizeof(h), cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaStreamSynchronize(s));
  YS_REQUIRE(!(h[0] & 4u), YS_ERR_INVALID, "blocks are not (row, col)-sorted along the row plan");
  YS_REQUIRE(h[0] == 0, YS_ERR_CAPACITY, "a tile exceeds the streamed SpMV's entry, column or slot limits");
  caps_host[0] = h[1];
  caps_host[1] = h[2];
  caps_host[2] = h[3];
  return YS_OK;
}

int32_t ys_spmv_stream_fill(const float* values32, const uint32_t* src, uint64_t slots, float* blocks32,
                            void* stream) {
  YS_REQUIRE(values32 && src && blocks32, YS_ERR_INVALID, "null argument");
  YS_REQUIRE((reinterpret_cast<uintptr_t>(values32) & 15) == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0 &&
                 (reinterpret_cast<uintptr_t>(blocks32) & 15) == 0 && slots % 4 == 0,
             YS_ERR_INVALID, "values32, src and blocks32 16-byte aligned, slots a multiple of 4");
  if (slots == 0) return YS_OK;
  ys::stream_fill_kernel<<<ys::grid_for(slots / 4, 256), 256, 0, (cudaStream_t)stream>>>(values32, src, slots,
                                                                                      blocks32);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_spmv3_x32_streamed(const ys_spmv_stream* plan, const float* values32, const uint32_t* row_ptr,
                              const uint32_t* entry_block, const uint32_t* entry_col, uint32_t num_vars,
                              const float* x32, double* y, int32_t beta, uint32_t stages, uint32_t max_ctas,
                              uint32_t* stage_status, void* stream) {
  YS_REQUIRE(plan && values32 && x32 && row_ptr && entry_block && entry_col, YS_ERR_INVALID, "null argument");
  YS_REQUIRE((reinterpret_cast<uintptr_t>(x32) & 15) == 0 && (reinterpret_cast<uintptr_t>(values32) & 15) == 0,
             YS_ERR_INVALID, "values32 and x32 must be 16-byte aligned");
  if (num_vars == 0) return YS_OK;
  YS_REQUIRE(plan->blocks32 && plan->desc && plan->rows && plan->words && plan->halo && plan->block_cap % 4 == 0 &&
                 plan->entry_cap % 4 == 0 && plan->halo_cap % 4 == 0 && plan->halo_cap <= ys::kStreamMaxHalo,
             YS_ERR_INVALID, "no stream plan");
  YS_REQUIRE(stages == 0 || stages == 2 || stages == 3, YS_ERR_INVALID, "stages: 0 (auto), 2 or 3");
  int dev = 0, sms = 0, per_sm = 0;
  YS_CUDA_TRY(cudaGetDevice(&dev));
  YS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (stages == 0)
    stages = ys::stream_pick_stages((const void*)ys::spmv3_x32_stream_kernel, plan->block_cap, plan->entry_cap,
                                    plan->halo_cap, &per_sm);
  YS_REQUIRE(stages != 0, YS_ERR_CAPACITY, "a tile's stream exceeds the shared-memory stages");
  const size_t smem = ys::stream_smem_bytes(plan->block_cap, plan->entry_cap, plan->halo_cap, stages);
  YS_REQUIRE(smem <= 220u * 1024u, YS_ERR_CAPACITY, "a tile's stream exceeds the shared-memory stages");
  YS_CUDA_TRY(cudaFuncSetAttribute(ys::spmv3_x32_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  YS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ys::spmv3_x32_stream_kernel, ys::kTileThreads,
                                                            smem));
  YS_REQUIRE(per_sm > 0, YS_ERR_CAPACITY, "streamed SpMV does not fit on an SM");
  const uint32_t ntiles = (num_vars + ys::kTileRows - 1) / ys::kTileRows;
  unsigned grid = std::min<unsigned>(ntiles, (unsigned)(sms * per_sm));
  if (max_ctas) grid = std::min<unsigned>(grid, max_ctas);
  ys::StreamSet T =
      ys::stream_set(*plan, ys::SpmvSet{nullptr, values32, row_ptr, entry_block, entry_col}, num_vars, stages);
  ys::spmv3_x32_stream_kernel<<<grid, ys::kTileThreads, smem, (cudaStream_t)stream>>>(
      T, reinterpret_cast<const float4*>(x32), y, beta, stage_status);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

}  // extern "C"
