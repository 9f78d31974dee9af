// Global sparsity pattern: unique sort of block occurrences by (h, w, row, col).
//
// Restates get_unique_coords + compress_unique_coords
// (PKG/kernel/Coordinate/coordinateCompressionKernel.pyx:92-144, 350-419) with
// LSD radix sorts (stable), and additionally returns the deterministic
// assembly plan: the sorted position of every occurrence is the slot of its
// element record, so one unique block's records are contiguous and in
// occurrence order.  Setup-time code (once per static structure, every step
// for dynamic terms).
#include <algorithm>
#include <cstring>

#include <cub/cub.cuh>

#include "ys_common.cuh"

namespace ys {

__global__ void pack_keys_kernel(const uint32_t* __restrict__ coords, uint32_t m, uint64_t* __restrict__ keys,
                                 uint32_t* __restrict__ vals) {
  const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= m) return;
  keys[o] = ((uint64_t)coords[2ull * o] << 32) | coords[2ull * o + 1];
  vals[o] = o;
}

__global__ void cat_keys_kernel(const uint16_t* __restrict__ dims, const uint32_t* __restrict__ order, uint32_t m,
                                uint32_t* __restrict__ cat) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const uint32_t o = order[p];
  cat[p] = ((uint32_t)dims[2ull * o] << 16) | dims[2ull * o + 1];
}

__device__ __forceinline__ bool same_key(const uint32_t* coords, const uint16_t* dims, uint32_t a, uint32_t b) {
  return coords[2ull * a] == coords[2ull * b] && coords[2ull * a + 1] == coords[2ull * b + 1] &&
         dims[2ull * a] == dims[2ull * b] && dims[2ull * a + 1] == dims[2ull * b + 1];
}

// head[p] = 1 at the first occurrence of every unique key; hw[p] = h*w.
__global__ void heads_kernel(const uint32_t* __restrict__ coords, const uint16_t* __restrict__ dims,
                             const uint32_t* __restrict__ order, uint32_t m, uint32_t* __restrict__ head,
                             uint32_t* __restrict__ hw) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const uint32_t o = order[p];
  head[p] = (p == 0 || !same_key(coords, dims, o, order[p - 1])) ? 1u : 0u;
  hw[p] = (uint32_t)dims[2ull * o] * dims[2ull * o + 1];
}

// After inclusive scan, ord[p] = 1 + unique ordinal; rec[p] = exclusive scan of hw.
__global__ void unique_kernel(const uint32_t* __restrict__ coords, const uint16_t* __restrict__ dims,
                              const uint32_t* __restrict__ order, const uint32_t* __restrict__ ord,
                              const uint32_t* __restrict__ rec, uint32_t m, uint32_t* __restrict__ positions,
                              uint16_t* __restrict__ bdims, uint32_t* __restrict__ vsize,
                              uint32_t* __restrict__ rec_begin, uint32_t* __restrict__ rec_count) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const uint32_t u = ord[p] - 1;
  const bool is_head = (p == 0) || ord[p - 1] != ord[p];
  if (is_head) {
    const uint32_t o = order[p];
    positions[2ull * u] = coords[2ull * o];
    positions[2ull * u + 1] = coords[2ull * o + 1];
    bdims[2ull * u] = dims[2ull * o];
    bdims[2ull * u + 1] = dims[2ull * o + 1];
    vsize[u] = (uint32_t)dims[2ull * o] * dims[2ull * o + 1];
    rec_begin[u] = rec[p];
  }
}

__global__ void counts_kernel(const uint32_t* __restrict__ ord, uint32_t m, uint32_t* __restrict__ rec_count) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const bool is_head = (p == 0) || ord[p - 1] != ord[p];
  if (!is_head) return;
  uint32_t q = p + 1;
  while (q < m && ord[q] == ord[p]) ++q;
  rec_count[ord[p] - 1] = q - p;
}

__global__ void lookup_kernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ ord,
                              const uint32_t* __restrict__ rec, const uint32_t* __restrict__ value_offset,
                              uint32_t m, uint32_t* __restrict__ lookup, uint32_t* __restrict__ record) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const uint32_t o = order[p];
  lookup[o] = value_offset[ord[p] - 1];
  record[o] = rec[p];
}

struct CatEntry {
  uint32_t first;
  uint32_t hw;
};

__global__ void category_kernel(const uint16_t* __restrict__ bdims, uint32_t nu, CatEntry* __restrict__ cats,
                                uint32_t* __restrict__ ncat) {
  const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nu) return;
  const bool head = u == 0 || bdims[2ull * u] != bdims[2ull * (u - 1)] || bdims[2ull * u + 1] != bdims[2ull * (u - 1) + 1];
  if (!head) return;
  const uint32_t slot = atomicAdd(ncat, 1u);
  if (slot < 16) cats[slot] = CatEntry{u, ((uint32_t)bdims[2ull * u] << 16) | bdims[2ull * u + 1]};
}

struct PatternWorkspace {
  uint64_t* keys[2];
  uint32_t* vals[2];
  uint32_t* cat[2];
  uint32_t* head;
  uint32_t* hw;
  uint32_t* small;   // [64] scratch for category entries and counters
  void* cub_tmp;
  size_t cub_bytes;
};

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

static size_t cub_bytes_for(uint32_t m) {
  size_t a = 0, b = 0, c = 0, d = 0;
  cub::DoubleBuffer<uint64_t> k64(nullptr, nullptr);
  cub::DoubleBuffer<uint32_t> v(nullptr, nullptr), k32(nullptr, nullptr);
  cub::DeviceRadixSort::SortPairs(nullptr, a, k64, v, (int)m);
  cub::DeviceRadixSort::SortPairs(nullptr, b, k32, v, (int)m);
  cub::DeviceScan::InclusiveSum(nullptr, c, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)m);
  cub::DeviceScan::ExclusiveSum(nullptr, d, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)m + 1);
  return std::max(std::max(a, b), std::max(c, d));
}

static size_t workspace_bytes(uint32_t m) {
  size_t total = 0;
  total += 2 * align256(8ull * m);
  total += 4 * align256(4ull * m);
  total += 2 * align256(4ull * (m + 1));
  total += align256(64 * 4);
  total += align256(cub_bytes_for(m));
  return total;
}

static PatternWorkspace carve(void* base, uint32_t m) {
  PatternWorkspace w{};
  char* p = (char*)base;
  auto take = [&](size_t bytes) { void* r = p; p += align256(bytes); return r; };
  w.keys[0] = (uint64_t*)take(8ull * m);
  w.keys[1] = (uint64_t*)take(8ull * m);
  w.vals[0] = (uint32_t*)take(4ull * m);
  w.vals[1] = (uint32_t*)take(4ull * m);
  w.cat[0] = (uint32_t*)take(4ull * (m + 1));
  w.cat[1] = (uint32_t*)take(4ull * (m + 1));
  w.head = (uint32_t*)take(4ull * m);
  w.hw = (uint32_t*)take(4ull * m);
  w.small = (uint32_t*)take(64 * 4);
  w.cub_bytes = cub_bytes_for(m);
  w.cub_tmp = take(w.cub_bytes);
  return w;
}

}  // namespace ys

extern "C" {

int32_t ys_pattern_workspace_bytes(uint32_t n_coords, uint64_t* bytes) {
  *bytes = ys::workspace_bytes(n_coords > 0 ? n_coords : 1);
  return YS_OK;
}

int32_t ys_pattern_build(const uint32_t* coords, const uint16_t* dims, uint32_t m, void* workspace,
                         uint64_t workspace_bytes, ys_pattern_out* out, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  out->num_unique = 0;
  out->num_categories = 0;
  out->total_records = 0;
  out->category_starts[0] = 0;
  if (m == 0) {
    YS_CUDA_TRY(cudaMemsetAsync(out->value_offset, 0, sizeof(uint32_t), s));
    return YS_OK;
  }
  YS_REQUIRE(m < 0x7fffffffu, YS_ERR_INVALID, "too many coordinates");
  YS_REQUIRE(workspace_bytes >= ys::workspace_bytes(m), YS_ERR_CAPACITY, "pattern workspace too small");
  ys::PatternWorkspace w = ys::carve(workspace, m);
  const unsigned g = ys::grid_for(m, 256);
  ys::pack_keys_kernel<<<g, 256, 0, s>>>(coords, m, w.keys[0], w.vals[0]);
  YS_CHECK_LAUNCH();
  // Pass 1: stable sort by (row, col).
  cub::DoubleBuffer<uint64_t> k64(w.keys[0], w.keys[1]);
  cub::DoubleBuffer<uint32_t> v(w.vals[0], w.vals[1]);
  size_t tb = w.cub_bytes;
  YS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(w.cub_tmp, tb, k64, v, (int)m, 0, 64, s));
  // Pass 2: stable sort by (h, w) keeps (row, col) order inside a category.
  ys::cat_keys_kernel<<<g, 256, 0, s>>>(dims, v.Current(), m, w.cat[0]);
  YS_CHECK_LAUNCH();
  cub::DoubleBuffer<uint32_t> k32(w.cat[0], w.cat[1]);
  uint32_t* other = v.Current() == w.vals[0] ? w.vals[1] : w.vals[0];
  cub::DoubleBuffer<uint32_t> v2(v.Current(), other);
  tb = w.cub_bytes;
  YS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(w.cub_tmp, tb, k32, v2, (int)m, 0, 32, s));
  const uint32_t* order = v2.Current();
  uint32_t* ord = w.head;
  uint32_t* rec = w.hw;
  ys::heads_kernel<<<g, 256, 0, s>>>(coords, dims, order, m, ord, rec);
  YS_CHECK_LAUNCH();
  tb = w.cub_bytes;
  YS_CUDA_TRY(cub::DeviceScan::InclusiveSum(w.cub_tmp, tb, ord, ord, (int)m, s));
  // rec: exclusive scan of h*w in sorted order (record offsets).  Reuse the
  // spare value buffer for the scan output.
  uint32_t* rec_off = (uint32_t*)(v2.Current() == w.vals[0] ? w.vals[1] : w.vals[0]);
  tb = w.cub_bytes;
  YS_CUDA_TRY(cub::DeviceScan::ExclusiveSum(w.cub_tmp, tb, rec, rec_off, (int)m, s));
  uint32_t nu = 0, last_rec = 0, last_hw = 0;
  YS_CUDA_TRY(cudaMemcpyAsync(&nu, ord + (m - 1), 4, cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaMemcpyAsync(&last_rec, rec_off + (m - 1), 4, cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaMemcpyAsync(&last_hw, rec + (m - 1), 4, cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaStreamSynchronize(s));
  const uint64_t total_records = (uint64_t)last_rec + last_hw;
  YS_REQUIRE(total_records < 0xffffffffull, YS_ERR_CAPACITY, "record offsets exceed 32 bits");
  ys::unique_kernel<<<g, 256, 0, s>>>(coords, dims, order, ord, rec_off, m, out->positions, out->block_dims,
                                      w.cat[0], out->record_begin, out->record_count);
  YS_CHECK_LAUNCH();
  ys::counts_kernel<<<g, 256, 0, s>>>(ord, m, out->record_count);
  YS_CHECK_LAUNCH();
  // value_offset = exclusive scan of h*w over unique blocks (nu + 1 entries).
  YS_CUDA_TRY(cudaMemsetAsync(w.cat[0] + nu, 0, 4, s));
  tb = w.cub_bytes;
  YS_CUDA_TRY(cub::DeviceScan::ExclusiveSum(w.cub_tmp, tb, w.cat[0], out->value_offset, (int)nu + 1, s));
  ys::lookup_kernel<<<g, 256, 0, s>>>(order, ord, rec_off, out->value_offset, m, out->lookup, out->record);
  YS_CHECK_LAUNCH();
  YS_CUDA_TRY(cudaMemsetAsync(w.small, 0, 64 * 4, s));
  ys::CatEntry* cats = (ys::CatEntry*)(w.small + 1);
  ys::category_kernel<<<ys::grid_for(nu, 256), 256, 0, s>>>(out->block_dims, nu, cats, w.small);
  YS_CHECK_LAUNCH();
  uint32_t host_small[64];
  uint32_t total_values = 0;
  YS_CUDA_TRY(cudaMemcpyAsync(host_small, w.small, sizeof(host_small), cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaMemcpyAsync(&total_values, out->value_offset + nu, 4, cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaStreamSynchronize(s));
  const uint32_t ncat = host_small[0];
  YS_REQUIRE(ncat >= 1 && ncat <= 16, YS_ERR_CAPACITY, "more than 16 block categories");
  ys::CatEntry entries[16];
  memcpy(entries, host_small + 1, sizeof(ys::CatEntry) * ncat);
  std::sort(entries, entries + ncat, [](const ys::CatEntry& a, const ys::CatEntry& b) { return a.first < b.first; });
  out->num_unique = nu;
  out->num_categories = ncat;
  out->total_records = total_records;
  uint32_t vstart = 0;
  for (uint32_t c = 0; c < ncat; ++c) {
    const uint32_t first = entries[c].first;
    const uint32_t next = c + 1 < ncat ? entries[c + 1].first : nu;
    const uint32_t h = entries[c].hw >> 16, wd = entries[c].hw & 0xffffu;
    out->category_dims[2 * c] = (uint16_t)h;
    out->category_dims[2 * c + 1] = (uint16_t)wd;
    out->category_counts[c] = next - first;
    out->category_starts[c] = vstart;
    vstart += (next - first) * h * wd;
  }
  out->category_starts[ncat] = vstart;
  YS_REQUIRE(vstart == total_values, YS_ERR_INVALID, "category metadata mismatch");
  return YS_OK;
}

}  // extern "C"
