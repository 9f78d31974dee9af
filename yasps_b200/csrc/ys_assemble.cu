// Deterministic assembly of element records, diagonal blocks and their
// pseudo-inverse.
//
// The pattern build places every occurrence's record at its sorted position,
// so the records of one unique block are contiguous and ordered by
// occurrence index.  Assembly is a segmented sum over contiguous memory in
// that order: no float atomics, bit-reproducible, HBM bound (read records
// once, write the assembled values once).
#include <algorithm>

#include "ys_common.cuh"
#include "ys_eigen.cuh"

namespace ys {

// One warp per unique entry: lanes own output elements e < hw (hw <= 32 per
// pass) and walk the contiguous records in order.
template <typename Out32>
__global__ void __launch_bounds__(256) assemble_kernel(const double* __restrict__ rec,
                                                       const uint32_t* __restrict__ begin,
                                                       const uint32_t* __restrict__ count,
                                                       const uint32_t* __restrict__ offset, uint32_t offset_stride,
                                                       const uint16_t* __restrict__ dims, uint32_t nu,
                                                       double* __restrict__ out, Out32* __restrict__ out32) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (warp >= nu) return;
  const uint32_t hw = (uint32_t)dims[2ull * warp] * dims[2ull * warp + 1];
  const uint32_t b = begin[warp], c = count[warp];
  const uint64_t o = offset[(uint64_t)warp * offset_stride];
  for (uint32_t e = lane; e < hw; e += 32) {
    double acc = 0.0;
    for (uint32_t k = 0; k < c; ++k) acc += rec[(uint64_t)b + (uint64_t)k * hw + e];
    out[o + e] = acc;
    if (out32) out32[o + e] = (Out32)acc;
  }
}

// Small entries (gradient segments, hw = 3 for 3-DoF vertices): 3 lanes per
// unique entry, 10 entries per warp; a group walks elements sub, sub+3, ...
// of its entry, each summed over the records in order (the same order as
// assemble_kernel).
__global__ void __launch_bounds__(256) assemble_small_kernel(const double* __restrict__ rec,
                                                             const uint32_t* __restrict__ begin,
                                                             const uint32_t* __restrict__ count,
                                                             const uint32_t* __restrict__ offset,
                                                             uint32_t offset_stride,
                                                             const uint16_t* __restrict__ dims, uint32_t nu,
                                                             double* __restrict__ out) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (lane >= 30) return;
  const uint32_t u = warp * 10 + lane / 3, sub = lane % 3;
  if (u >= nu) return;
  const uint32_t hw = (uint32_t)dims[2ull * u] * dims[2ull * u + 1];
  const uint32_t b = begin[u], c = count[u];
  const uint64_t o = offset[(uint64_t)u * offset_stride];
  for (uint32_t e = sub; e < hw; e += 3) {
    double acc = 0.0;
    for (uint32_t k = 0; k < c; ++k) acc += rec[(uint64_t)b + (uint64_t)k * hw + e];
    out[o + e] = acc;
  }
}

// 3x3 fast path: 9 lanes per unique block (3 blocks per warp, 5 lanes idle).
__global__ void __launch_bounds__(256) assemble3_kernel(const double* __restrict__ rec,
                                                        const uint32_t* __restrict__ begin,
                                                        const uint32_t* __restrict__ count,
                                                        const uint32_t* __restrict__ offset, uint32_t nu,
                                                        double* __restrict__ out, float* __restrict__ out32,
                                                        const uint2* __restrict__ slot_of,
                                                        float* __restrict__ blocks32) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t u = warp * 3 + lane / 9;
  const uint32_t e = lane % 9;
  if (lane >= 27 || u >= nu) return;
  const uint32_t b = begin[u], c = count[u];
  double acc = 0.0;
  for (uint32_t k = 0; k < c; ++k) acc += rec[(uint64_t)b + 9ull * k + e];
  const uint64_t o = offset[u];
  out[o + e] = acc;
  if (out32) out32[12ull * u + e] = (float)acc;  // 12-float FP32 block slots
  if (blocks32) {
    // the streamed SpMV's packed copies: the block's slot in its row's tile
    // and, for a block used transposed by a later tile, its slot there
    const uint2 sl = slot_of[u];
    blocks32[9ull * sl.x + e] = (float)acc;
    if (sl.y != 0xffffffffu) blocks32[9ull * sl.y + e] = (float)acc;
  }
}

struct DiagLayout {
  uint32_t n;
  uint32_t seg[9];
  uint32_t size[8];
  uint32_t dstart[8];
};

__global__ void extract_diag_kernel(const double* __restrict__ values, const uint32_t* __restrict__ positions,
                                    const uint16_t* __restrict__ bdims, const uint32_t* __restrict__ voff,
                                    uint32_t nu, DiagLayout L, double* __restrict__ dblocks,
                                    double* __restrict__ diagonal, int accumulate) {
  const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nu) return;
  const uint32_t r = positions[2ull * u], c = positions[2ull * u + 1];
  int a = 0;
  while (a + 1 < (int)L.n && r >= L.seg[a + 1]) ++a;
  const uint32_t s = L.size[a];
  const uint32_t h = bdims[2ull * u], w = bdims[2ull * u + 1];
  if (c < L.seg[a] || c >= L.seg[a + 1]) return;
  const uint32_t inst = (r - L.seg[a]) / s;
  if ((c - L.seg[a]) / s != inst) return;
  const double* v = values + voff[u];
  double* d = dblocks ? dblocks + L.dstart[a] + (uint64_t)inst * s * s : nullptr;
  if (r == c && h == s) {
    for (uint32_t k = 0; k < s * s; ++k) {
      if (d) d[k] = accumulate ? d[k] + v[k] : v[k];
    }
    if (diagonal)
      for (uint32_t k = 0; k < s; ++k) diagonal[r + k] = accumulate ? diagonal[r + k] + v[k * s + k] : v[k * s + k];
    return;
  }
  // A block inside one instance of a larger attribute (the rows of an affine
  // matrix are stored as 3x3 blocks): placed at its offset, mirrored when it
  // lies off the diagonal.
  const uint32_t base = L.seg[a] + inst * s, ro = r - base, co = c - base;
  if (ro + h > s || co + w > s) return;
  if (d)
    for (uint32_t k = 0; k < h; ++k)
      for (uint32_t l = 0; l < w; ++l) {
        const double x = v[k * w + l];
        double& e0 = d[(ro + k) * s + co + l];
        e0 = accumulate ? e0 + x : x;
        if (r != c) {
          double& e1 = d[(co + l) * s + ro + k];
          e1 = accumulate ? e1 + x : x;
        }
      }
  if (diagonal && r == c)
    for (uint32_t k = 0; k < h && k < w; ++k)
      diagonal[r + k] = accumulate ? diagonal[r + k] + v[k * w + k] : v[k * w + k];
}

// |lambda| -> |1/lambda| (|lambda| < 1e-6 -> |lambda|), diagonalBlockInverseKernel.pyx:69,91.
template <int S>
__global__ void invert_blocks_kernel(const double* __restrict__ in, double* __restrict__ out, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a[S][S], v[S][S];
  const double* src = in + (uint64_t)i * S * S;
#pragma unroll
  for (int r = 0; r < S; ++r)
#pragma unroll
    for (int c = 0; c < S; ++c) a[r][c] = 0.5 * (src[r * S + c] + src[c * S + r]);
  jacobi_eigen<S>(a, v);
  double w[S];
#pragma unroll
  for (int k = 0; k < S; ++k) {
    const double l = a[k][k];
    w[k] = fabs(l) < 1e-6 ? fabs(l) : fabs(1.0 / l);
  }
  double* dst = out + (uint64_t)i * S * S;
  for (int r = 0; r < S; ++r)
    for (int c = 0; c < S; ++c) {
      double acc = 0.0;
      for (int k = 0; k < S; ++k) acc += v[r][k] * w[k] * v[c][k];
      dst[r * S + c] = acc;
    }
}

// Deterministic sum: block sums of a fixed grid, then the last block adds
// them in index order.
constexpr int kSumThreads = 256;
constexpr unsigned kSumBlocks = 1024;

__global__ void __launch_bounds__(kSumThreads) sum_kernel(const double* __restrict__ x, uint32_t n,
                                                          double* __restrict__ partials, unsigned* __restrict__ ticket,
                                                          double* __restrict__ out) {
  __shared__ double red[kSumThreads / 32];
  __shared__ bool last;
  double v = 0.0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v += x[i];
  const double sb = block_sum<kSumThreads>(v, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = sb;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  double acc = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) acc += __ldcg(partials + b);
  acc = block_sum<kSumThreads>(acc, red);
  if (threadIdx.x == 0) {
    *out = acc;
    *ticket = 0u;
  }
}

}  // namespace ys

extern "C" {

int32_t ys_assemble(const double* records, const uint32_t* begin, const uint32_t* count, const uint32_t* offset,
                    const uint16_t* dims, uint32_t nu, double* out, float* out32, void* stream) {
  if (nu == 0) return YS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const uint64_t threads = (uint64_t)nu * 32;
  ys::assemble_kernel<float><<<ys::grid_for(threads, 256), 256, 0, s>>>(records, begin, count, offset, 1, dims, nu,
                                                                         out, out32);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_assemble3(const double* records, const uint32_t* begin, const uint32_t* count, const uint32_t* offset,
                     uint32_t nu, double* out, float* out32, void* stream) {
  if (nu == 0) return YS_OK;
  const uint64_t warps = (nu + 2) / 3;
  ys::assemble3_kernel<<<ys::grid_for(warps * 32, 256), 256, 0, (cudaStream_t)stream>>>(records, begin, count, offset,
                                                                                        nu, out, out32, nullptr,
                                                                                        nullptr);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_assemble3_streamed(const double* records, const uint32_t* begin, const uint32_t* count,
                              const uint32_t* offset, uint32_t nu, double* out, float* out32, const uint32_t* slot_of,
                              float* blocks32, void* stream) {
  YS_REQUIRE(slot_of && blocks32, YS_ERR_INVALID, "null argument");
  YS_REQUIRE((reinterpret_cast<uintptr_t>(slot_of) & 7) == 0, YS_ERR_INVALID, "slot_of must be 8-byte aligned");
  if (nu == 0) return YS_OK;
  const uint64_t warps = (nu + 2) / 3;
  ys::assemble3_kernel<<<ys::grid_for(warps * 32, 256), 256, 0, (cudaStream_t)stream>>>(
      records, begin, count, offset, nu, out, out32, reinterpret_cast<const uint2*>(slot_of), blocks32);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_assemble_strided(const double* records, const uint32_t* begin, const uint32_t* count,
                            const uint32_t* offset, uint32_t offset_stride, const uint16_t* dims, uint32_t nu,
                            double* out, void* stream) {
  if (nu == 0) return YS_OK;
  const uint64_t threads = ((uint64_t)nu + 9) / 10 * 32;
  ys::assemble_small_kernel<<<ys::grid_for(threads, 256), 256, 0, (cudaStream_t)stream>>>(
      records, begin, count, offset, offset_stride, dims, nu, out);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_extract_diagonal(const double* values, const uint32_t* positions, const uint16_t* block_dims,
                            const uint32_t* value_offset, uint32_t nu, uint32_t num_attributes,
                            const uint32_t* seg_start, const uint32_t* attr_size, const uint32_t* diag_start,
                            double* diag_blocks, double* diagonal, int32_t accumulate, void* stream) {
  YS_REQUIRE(num_attributes >= 1 && num_attributes <= 8, YS_ERR_INVALID, "1..8 attributes");
  if (nu == 0) return YS_OK;
  ys::DiagLayout L{};
  L.n = num_attributes;
  for (uint32_t a = 0; a <= num_attributes; ++a) L.seg[a] = seg_start[a];
  for (uint32_t a = 0; a < num_attributes; ++a) { L.size[a] = attr_size[a]; L.dstart[a] = diag_start[a]; }
  ys::extract_diag_kernel<<<ys::grid_for(nu, 256), 256, 0, (cudaStream_t)stream>>>(
      values, positions, block_dims, value_offset, nu, L, diag_blocks, diagonal, accumulate);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_invert_diagonal_blocks(const double* diag_blocks, double* inverse, uint32_t num_attributes,
                                  const uint32_t* diag_start, const uint32_t* count, const uint32_t* attr_size,
                                  void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  for (uint32_t a = 0; a < num_attributes; ++a) {
    const uint32_t n = count[a];
    if (n == 0) continue;
    const double* in = diag_blocks + diag_start[a];
    double* out = inverse + diag_start[a];
    const unsigned g = ys::grid_for(n, 128);
    switch (attr_size[a]) {
      case 1: ys::invert_blocks_kernel<1><<<g, 128, 0, s>>>(in, out, n); break;
      case 2: ys::invert_blocks_kernel<2><<<g, 128, 0, s>>>(in, out, n); break;
      case 3: ys::invert_blocks_kernel<3><<<g, 128, 0, s>>>(in, out, n); break;
      case 4: ys::invert_blocks_kernel<4><<<g, 128, 0, s>>>(in, out, n); break;
      case 6: ys::invert_blocks_kernel<6><<<g, 128, 0, s>>>(in, out, n); break;
      case 9: ys::invert_blocks_kernel<9><<<g, 128, 0, s>>>(in, out, n); break;
      case 12: ys::invert_blocks_kernel<12><<<g, 128, 0, s>>>(in, out, n); break;
      default: YS_REQUIRE(false, YS_ERR_INVALID, "unsupported attribute size for the block inverse");
    }
    YS_CHECK_LAUNCH();
  }
  return YS_OK;
}

uint64_t ys_sum_workspace_doubles(void) { return ys::kSumBlocks + 1; }

int32_t ys_sum(const double* values, uint32_t n, double* out, double* workspace, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  unsigned* ticket = reinterpret_cast<unsigned*>(workspace + ys::kSumBlocks);
  YS_CUDA_TRY(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
  if (n == 0) {
    YS_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double), s));
    return YS_OK;
  }
  const unsigned grid = std::min<unsigned>(ys::grid_for(n, ys::kSumThreads), ys::kSumBlocks);
  ys::sum_kernel<<<grid, ys::kSumThreads, 0, s>>>(values, n, workspace, ticket, out);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

}  // extern "C"
