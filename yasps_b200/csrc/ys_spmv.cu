// Row plan build and the standalone symmetric 3x3-block SpMV.
#include <cub/cub.cuh>

#include "ys_spmv.cuh"
#include "ys_spmv_tiled.cuh"

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

}  // extern "C"
