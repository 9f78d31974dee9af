// Index slots, local compression and block coordinates.
//
// Integer work, bit-exact with the reference's generated index kernels
// (PKG/kernel/Coordinate/gradientIndicesKernel.pyx).  One thread per instance;
// every thread walks its own K slots, so the launch is HBM/latency bound.
#include <cub/cub.cuh>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>

#include "ys_common.cuh"

namespace {
thread_local std::string g_last_error;
}

void ys_set_last_error(const char* msg, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s (%s:%d)", msg, file, line);
  g_last_error = buf;
}

namespace ys {

struct UnionDesc {
  uint32_t prefix[YS_MAX_UNION + 1];
  int32_t kind[YS_MAX_UNION];
  uint32_t wrt_start[YS_MAX_UNION];
  uint32_t num_children;
};

// gradientIndicesKernel.pyx:759-846 (JOIN loop) and :759-800 (UNION switch).
__global__ void join_union_indices_kernel(const uint32_t* __restrict__ conn, uint32_t n, uint32_t join_dim,
                                          UnionDesc u, uint32_t leaf_size, uint32_t* __restrict__ codes,
                                          uint16_t* __restrict__ sizes) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const bool is_union = u.num_children > 1;
  const uint32_t per_arg = is_union ? 2u : 1u;
  const uint32_t K = join_dim * per_arg;
  for (uint32_t a = 0; a < join_dim; ++a) {
    const uint32_t idx = conn[(uint64_t)t * join_dim + a];
    uint32_t child = 0, total = 0;
    for (uint32_t c = 0; c < u.num_children; ++c) {
      if (total + (u.prefix[c + 1] - u.prefix[c]) > idx) { child = c; break; }
      total += u.prefix[c + 1] - u.prefix[c];
      child = c + 1;
    }
    const uint32_t local = idx - total;
    uint32_t code = 0;
    uint16_t size = 0, pad = 0;
    if (child < u.num_children) {
      const int32_t kind = u.kind[child];
      if (kind == 2) { code = u.wrt_start[child] + local * leaf_size + 2u; size = (uint16_t)leaf_size; }
      else if (kind == 1) { code = 1u; size = (uint16_t)leaf_size; }
      else { code = 0u; size = 0; pad = (uint16_t)leaf_size; }
    }
    const uint64_t base = (uint64_t)t * K + a * per_arg;
    codes[base] = code;
    sizes[base] = is_union ? size : (uint16_t)(size + pad);
    if (is_union) { codes[base + 1] = 0u; sizes[base + 1] = pad; }
  }
}

// computePermutation (gradientIndicesKernel.pyx:62-123).  Writes the triangular
// coordinate count u(u+1)/2 into coord_outer[t + 1]; a scan follows.
__global__ void compress_kernel(const uint32_t* __restrict__ codes, const uint16_t* __restrict__ sizes,
                                uint32_t n, uint32_t K, int16_t* __restrict__ perm,
                                uint16_t* __restrict__ total_sizes, uint32_t* __restrict__ coord_counts) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint64_t base = (uint64_t)t * K;
  int offset = 0;
  uint32_t total = 0, uniq = 0;
  for (uint32_t i = 0; i < K; ++i) {
    const uint32_t ci = codes[base + i];
    perm[base + i] = 0;
    if (ci == 0) continue;
    bool found = false;
    if (ci >= 2) {
      for (uint32_t j = 0; j < i; ++j) {
        if (codes[base + j] == ci) { perm[base + i] = (int16_t)(-perm[base + j]); found = true; break; }
      }
    }
    if (!found) {
      perm[base + i] = (int16_t)(offset + 1);
      offset += sizes[base + i];
      total += sizes[base + i];
      if (ci >= 2) ++uniq;
    }
  }
  if (total_sizes) total_sizes[t] = (uint16_t)total;
  coord_counts[t] = uniq * (uniq + 1) / 2;
}

// computeCoordinatesDeviceFunction (gradientIndicesKernel.pyx:234-274).
__global__ void coordinates_kernel(const uint32_t* __restrict__ codes, const int16_t* __restrict__ perm,
                                   const uint16_t* __restrict__ sizes, const uint32_t* __restrict__ outer,
                                   uint32_t n, uint32_t K, uint32_t* __restrict__ coords,
                                   uint16_t* __restrict__ dims) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint64_t base = (uint64_t)t * K;
  uint64_t out = 2ull * outer[t];
  for (uint32_t i = 0; i < K; ++i) {
    const uint32_t ci = codes[base + i];
    if (!(perm[base + i] > 0 && ci >= 2)) continue;
    for (uint32_t j = i; j < K; ++j) {
      const uint32_t cj = codes[base + j];
      if (!(perm[base + j] > 0 && cj >= 2)) continue;
      if (ci < cj) {
        coords[out] = ci - 2; coords[out + 1] = cj - 2;
        dims[out] = sizes[base + i]; dims[out + 1] = sizes[base + j];
      } else {
        coords[out] = cj - 2; coords[out + 1] = ci - 2;
        dims[out] = sizes[base + j]; dims[out + 1] = sizes[base + i];
      }
      out += 2;
    }
  }
}

__global__ void grad_count_kernel(const uint32_t* __restrict__ codes, uint32_t n, uint32_t K,
                                  uint32_t* __restrict__ counts) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t c = 0;
  for (uint32_t i = 0; i < K; ++i) c += codes[(uint64_t)t * K + i] >= 2 ? 1u : 0u;
  counts[t] = c;
}

__global__ void grad_coords_kernel(const uint32_t* __restrict__ codes, const uint16_t* __restrict__ sizes, uint32_t n,
                                   uint32_t K, const uint32_t* __restrict__ outer, uint32_t* __restrict__ coords,
                                   uint16_t* __restrict__ dims) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint64_t o = outer[t];
  for (uint32_t i = 0; i < K; ++i) {
    const uint32_t c = codes[(uint64_t)t * K + i];
    if (c < 2) continue;
    coords[2 * o] = c - 2;
    coords[2 * o + 1] = c - 2;
    dims[2 * o] = sizes[(uint64_t)t * K + i];
    dims[2 * o + 1] = 1;
    ++o;
  }
}

// ---- allocation-free compression -----------------------------------------
//
// ys_compress_indices_noalloc runs compress_kernel and then scans the counts
// with a three-pass tiled scan (tile sums, one-block scan of the tile sums,
// per-tile scan plus offset) instead of the CUB device scan, whose temporary
// storage comes from cudaMallocAsync.  The tile sums live in a fixed
// file-scope device array: at most kNoAllocMaxTiles tiles of kScanTile counts,
// i.e. n <= 67,108,864 instances, 128 KiB of scratch per device.  Each call
// writes every tile sum it reads before reading it, so nothing has to start
// at zero; all calls on a device share the array, so two calls that overlap in
// time (different streams or threads) race on it.  The scan is modulo 2^32
// like the CUB scan, so the outputs are bit-identical.
constexpr uint32_t kScanThreads = 256;
constexpr uint32_t kScanItems = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;
constexpr uint32_t kNoAllocMaxTiles = 32768;
constexpr uint64_t kNoAllocMaxInstances = (uint64_t)kNoAllocMaxTiles * kScanTile;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) uint32_t g_noalloc_tile_sums[kNoAllocMaxTiles];

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums(const uint32_t* __restrict__ v, uint32_t n,
                                                               uint32_t* __restrict__ tile_sums) {
  using Reduce = cub::BlockReduce<uint32_t, kScanThreads>;
  __shared__ typename Reduce::TempStorage tmp;
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  uint32_t s = 0;
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; ++k) {
    const uint64_t i = base + k * kScanThreads + threadIdx.x;
    if (i < n) s += v[i];
  }
  s = Reduce(tmp).Sum(s);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = s;
}

// Exclusive scan of the tile sums in place, one block of 1024 threads; thread
// t owns a run of ceil(tiles / 1024) consecutive sums.
__global__ void __launch_bounds__(1024) scan_tile_offsets(uint32_t* __restrict__ tile_sums, uint32_t tiles) {
  using Scan = cub::BlockScan<uint32_t, 1024>;
  __shared__ typename Scan::TempStorage tmp;
  const uint32_t per = (tiles + 1023) / 1024;
  const uint32_t b = threadIdx.x * per;
  uint32_t s = 0;
  for (uint32_t k = 0; k < per; ++k)
    if (b + k < tiles) s += tile_sums[b + k];
  uint32_t pre = 0;
  Scan(tmp).ExclusiveSum(s, pre);
  for (uint32_t k = 0; k < per; ++k) {
    if (b + k < tiles) {
      const uint32_t v = tile_sums[b + k];
      tile_sums[b + k] = pre;
      pre += v;
    }
  }
}

// In-place inclusive scan of one tile plus its offset.  The tile is staged in
// shared memory with one pad word per 32 (conflict-free striped and blocked
// access).
__global__ void __launch_bounds__(kScanThreads) scan_tiles(uint32_t* __restrict__ v, uint32_t n,
                                                           const uint32_t* __restrict__ tile_offsets) {
  using Scan = cub::BlockScan<uint32_t, kScanThreads>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ uint32_t tile[kScanTile + kScanTile / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; ++k) {
    const uint32_t x = k * kScanThreads + threadIdx.x;
    tile[x + (x >> 5)] = base + x < n ? v[base + x] : 0u;
  }
  __syncthreads();
  uint32_t run[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; ++k) {
    const uint32_t x = threadIdx.x * kScanItems + k;
    s += tile[x + (x >> 5)];
    run[k] = s;
  }
  uint32_t pre = 0;
  Scan(tmp).ExclusiveSum(s, pre);
  pre += tile_offsets[blockIdx.x];
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; ++k) {
    const uint32_t x = threadIdx.x * kScanItems + k;
    tile[x + (x >> 5)] = run[k] + pre;
  }
  __syncthreads();
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; ++k) {
    const uint32_t x = k * kScanThreads + threadIdx.x;
    if (base + x < n) v[base + x] = tile[x + (x >> 5)];
  }
}

// Device address of the tile-sum array for the current device, resolved once
// per device (the first call on a device does this set-up) and then read
// without a lock.  The address belongs to the device's primary context: after
// a cudaDeviceReset (or anything else that destroys and recreates that
// context) the module is loaded again, possibly elsewhere, and the cached
// address is stale: the entry point must not be called on that device after
// such a reset in the same process.
static std::atomic<void*> g_noalloc_addr[kNoAllocMaxDevices];

static int32_t noalloc_tile_sums(uint32_t** out) {
  int dev = 0;
  YS_CUDA_TRY(cudaGetDevice(&dev));
  YS_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, YS_ERR_INVALID, "device ordinal beyond 63");
  void* p = g_noalloc_addr[dev].load(std::memory_order_acquire);
  if (!p) {
    static std::mutex mu;  // taken only to resolve a device's address
    std::lock_guard<std::mutex> lock(mu);
    p = g_noalloc_addr[dev].load(std::memory_order_relaxed);
    if (!p) {
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tile_sums);
      if (e != cudaSuccess || !p) {
        ys_set_last_error(e != cudaSuccess ? cudaGetErrorString(e) : "null scratch address", __FILE__, __LINE__);
        return YS_ERR_CUDA;
      }
      g_noalloc_addr[dev].store(p, std::memory_order_release);
    }
  }
  *out = static_cast<uint32_t*>(p);
  return YS_OK;
}

}  // namespace ys

extern "C" {

int32_t ys_gradient_coordinates(const uint32_t* codes, const uint16_t* sizes, uint32_t n, uint32_t K,
                                uint32_t* grad_outer, uint32_t* coords, uint16_t* dims, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  YS_CUDA_TRY(cudaMemsetAsync(grad_outer, 0, sizeof(uint32_t), s));
  if (n == 0) return YS_OK;
  ys::grad_count_kernel<<<ys::grid_for(n, 256), 256, 0, s>>>(codes, n, K, grad_outer + 1);
  YS_CHECK_LAUNCH();
  size_t tmp = 0;
  YS_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, tmp, grad_outer + 1, grad_outer + 1, (int)n, s));
  void* d_tmp = nullptr;
  YS_CUDA_TRY(cudaMallocAsync(&d_tmp, tmp, s));
  cudaError_t e = cub::DeviceScan::InclusiveSum(d_tmp, tmp, grad_outer + 1, grad_outer + 1, (int)n, s);
  cudaFreeAsync(d_tmp, s);
  YS_CUDA_TRY(e);
  if (coords) {
    ys::grad_coords_kernel<<<ys::grid_for(n, 256), 256, 0, s>>>(codes, sizes, n, K, grad_outer, coords, dims);
    YS_CHECK_LAUNCH();
  }
  return YS_OK;
}

const char* ys_last_error(void) { return g_last_error.c_str(); }

int32_t ys_version(void) { return 100; }

int32_t ys_join_union_indices(const uint32_t* connectivity, uint32_t n, uint32_t join_dim, uint32_t num_children,
                              const uint32_t* child_prefix, const int32_t* child_kind,
                              const uint32_t* child_wrt_start, uint32_t leaf_size, uint32_t* codes,
                              uint16_t* sizes, void* stream) {
  YS_REQUIRE(num_children >= 1 && num_children <= YS_MAX_UNION, YS_ERR_INVALID, "num_children must be 1..8");
  YS_REQUIRE(join_dim >= 1 && leaf_size >= 1 && leaf_size < 65536, YS_ERR_INVALID, "bad join_dim/leaf_size");
  if (n == 0) return YS_OK;
  ys::UnionDesc u{};
  u.num_children = num_children;
  for (uint32_t c = 0; c <= num_children; ++c) u.prefix[c] = child_prefix[c];
  for (uint32_t c = 0; c < num_children; ++c) { u.kind[c] = child_kind[c]; u.wrt_start[c] = child_wrt_start[c]; }
  ys::join_union_indices_kernel<<<ys::grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
      connectivity, n, join_dim, u, leaf_size, codes, sizes);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_compress_indices(const uint32_t* codes, const uint16_t* sizes, uint32_t n, uint32_t K, int16_t* perm,
                            uint16_t* total_sizes, uint32_t* coord_outer, void* stream) {
  YS_REQUIRE(K >= 1 && K <= 4096, YS_ERR_INVALID, "K must be 1..4096");
  cudaStream_t s = (cudaStream_t)stream;
  YS_CUDA_TRY(cudaMemsetAsync(coord_outer, 0, sizeof(uint32_t), s));
  if (n == 0) return YS_OK;
  ys::compress_kernel<<<ys::grid_for(n, 256), 256, 0, s>>>(codes, sizes, n, K, perm, total_sizes, coord_outer + 1);
  YS_CHECK_LAUNCH();
  // In-place inclusive scan of the counts (the reference's
  // transform_inclusive_scan, gradientIndicesKernel.pyx:203-209).
  size_t tmp = 0;
  YS_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, tmp, coord_outer + 1, coord_outer + 1, (int)n, s));
  void* d_tmp = nullptr;
  YS_CUDA_TRY(cudaMallocAsync(&d_tmp, tmp, s));
  cudaError_t e = cub::DeviceScan::InclusiveSum(d_tmp, tmp, coord_outer + 1, coord_outer + 1, (int)n, s);
  cudaFreeAsync(d_tmp, s);
  YS_CUDA_TRY(e);
  return YS_OK;
}

int32_t ys_compute_coordinates(const uint32_t* codes, const int16_t* perm, const uint16_t* sizes,
                               const uint32_t* coord_outer, uint32_t n, uint32_t K, uint32_t* coords,
                               uint16_t* dims, void* stream) {
  if (n == 0) return YS_OK;
  ys::coordinates_kernel<<<ys::grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(codes, perm, sizes, coord_outer, n,
                                                                                   K, coords, dims);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_compress_indices_noalloc(const uint32_t* codes, const uint16_t* sizes, uint32_t n, uint32_t K,
                                    int16_t* perm, uint16_t* total_sizes, uint32_t* coord_outer, void* stream) {
  YS_REQUIRE(K >= 1 && K <= 4096, YS_ERR_INVALID, "K must be 1..4096");
  YS_REQUIRE(n <= ys::kNoAllocMaxInstances, YS_ERR_CAPACITY,
             "n exceeds the allocation-free scan's fixed scratch (at most 67,108,864 instances)");
  uint32_t* tile_sums = nullptr;
  const int32_t rc = ys::noalloc_tile_sums(&tile_sums);
  if (rc != YS_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  YS_CUDA_TRY(cudaMemsetAsync(coord_outer, 0, sizeof(uint32_t), s));
  if (n == 0) return YS_OK;
  ys::compress_kernel<<<ys::grid_for(n, 256), 256, 0, s>>>(codes, sizes, n, K, perm, total_sizes, coord_outer + 1);
  YS_CHECK_LAUNCH();
  const uint32_t tiles = (uint32_t)((n + ys::kScanTile - 1) / ys::kScanTile);
  ys::scan_tile_sums<<<tiles, ys::kScanThreads, 0, s>>>(coord_outer + 1, n, tile_sums);
  YS_CHECK_LAUNCH();
  ys::scan_tile_offsets<<<1, 1024, 0, s>>>(tile_sums, tiles);
  YS_CHECK_LAUNCH();
  ys::scan_tiles<<<tiles, ys::kScanThreads, 0, s>>>(coord_outer + 1, n, tile_sums);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

}  // extern "C"
