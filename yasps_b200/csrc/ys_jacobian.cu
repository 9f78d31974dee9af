// Rectangular second-order Jacobians d2E / (d rows d cols).
//
// The reference differentiates a scalar energy once with respect to the row
// targets and the result with respect to the column targets
// (PKG/differentiator/differentiator.pyx:367-489), builds the coordinates of
// every (row slot, column slot) pair of an instance
// (PKG/kernel/Coordinate/secondOrderJacobianIndicesKernel.pyx:16-84: a pair
// counts when both slots carry a target code >= 2, row-major over the
// instance's row slots) and compresses them into unique blocks like a
// Hessian, without the upper-triangle fold
// (PKG/matrixAndVector/matrix/secondOrderJacobian.pyx:296-335).  Here the
// instance's values come from its unprojected local Hessian over the
// energy's arguments (an argument may carry a row code, a column code, or
// both), repeated target codes of one instance are merged (first occurrence
// order), and the blocks are summed in a fixed order by the assembly plan of
// ys_pattern_build.  The product y = J x or y = J^T x gathers per output
// block row in block order: deterministic.
#include <algorithm>

#include <cub/cub.cuh>

#include "ys_common.cuh"

namespace ys {

constexpr int kRectMaxArgs = 8;

__device__ __forceinline__ int rect_groups(const uint32_t* __restrict__ codes, uint32_t t, uint32_t K,
                                           uint32_t stride, int args, int (&group)[kRectMaxArgs],
                                           int (&first)[kRectMaxArgs]) {
  int nfirst = 0;
  for (int a = 0; a < args; ++a) {
    const uint32_t c = codes[(uint64_t)t * K + (uint64_t)a * stride];
    group[a] = -1;
    if (c < 2) continue;
    int g = -1;
    for (int q = 0; q < nfirst; ++q)
      if (codes[(uint64_t)t * K + (uint64_t)first[q] * stride] == c) g = q;
    if (g < 0) {
      first[nfirst] = a;
      g = nfirst++;
    }
    group[a] = g;
  }
  return nfirst;
}

__global__ void rect_count_kernel(const uint32_t* __restrict__ row_codes, const uint32_t* __restrict__ col_codes,
                                  uint32_t n, uint32_t K, uint32_t stride, int args, uint32_t* __restrict__ count) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int group[kRectMaxArgs], first[kRectMaxArgs];
  const int nr = rect_groups(row_codes, t, K, stride, args, group, first);
  const int nc = rect_groups(col_codes, t, K, stride, args, group, first);
  count[t] = (uint32_t)(nr * nc);
}

__global__ void rect_coords_kernel(const uint32_t* __restrict__ row_codes, const uint32_t* __restrict__ col_codes,
                                   uint32_t n, uint32_t K, uint32_t stride, int args,
                                   const uint32_t* __restrict__ outer, uint32_t* __restrict__ coords,
                                   uint16_t* __restrict__ dims) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int rg[kRectMaxArgs], rf[kRectMaxArgs], cg[kRectMaxArgs], cf[kRectMaxArgs];
  const int nr = rect_groups(row_codes, t, K, stride, args, rg, rf);
  const int nc = rect_groups(col_codes, t, K, stride, args, cg, cf);
  uint32_t o = outer[t];
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j, ++o) {
      coords[2ull * o] = row_codes[(uint64_t)t * K + (uint64_t)rf[i] * stride] - 2u;
      coords[2ull * o + 1] = col_codes[(uint64_t)t * K + (uint64_t)cf[j] * stride] - 2u;
      dims[2ull * o] = 3;
      dims[2ull * o + 1] = 3;
    }
}

// Records of one instance: for every (row group, column group) the sum of
// its argument blocks of the packed upper local Hessian.  With `diff` > 0
// the local Hessian covers the first `diff` arguments only and arguments
// diff .. 2 diff - 1 are the step-start positions of an energy of x - x_old:
// their blocks are the first ones negated once per step-start side.
__global__ void rect_records_kernel(const double* __restrict__ local_h, int args, int diff,
                                    const uint32_t* __restrict__ row_codes, const uint32_t* __restrict__ col_codes,
                                    uint32_t n, uint32_t K, uint32_t stride, const uint32_t* __restrict__ outer,
                                    const uint32_t* __restrict__ record, double* __restrict__ out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int hargs = diff > 0 ? diff : args;
  const int N = 3 * hargs;
  const double* h = local_h + (uint64_t)t * (N * (N + 1) / 2);
  int rg[kRectMaxArgs], rf[kRectMaxArgs], cg[kRectMaxArgs], cf[kRectMaxArgs];
  const int nr = rect_groups(row_codes, t, K, stride, args, rg, rf);
  const int nc = rect_groups(col_codes, t, K, stride, args, cg, cf);
  // packed upper index of (r, c) for any order, arguments folded onto the
  // local Hessian's with their sign
  auto at = [&](int r, int c) {
    double sign = 1.0;
    if (diff > 0) {
      if (r >= N) { r -= N; sign = -sign; }
      if (c >= N) { c -= N; sign = -sign; }
    }
    const int lo = r < c ? r : c, hi = r < c ? c : r;
    return sign * h[lo * N - lo * (lo - 1) / 2 + (hi - lo)];
  };
  uint32_t o = outer[t];
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j, ++o) {
      double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int a = 0; a < args; ++a) {
        if (rg[a] != i) continue;
        for (int b = 0; b < args; ++b) {
          if (cg[b] != j) continue;
#pragma unroll
          for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int l = 0; l < 3; ++l) acc[k][l] += at(3 * a + k, 3 * b + l);
        }
      }
      double* dst = out + record[o];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) dst[3 * k + l] = acc[k][l];
    }
}

// Columns of a per-element scalar parameter (element t's column is
// param_start + t): one (3 x 1) pair per row group of the element.
__global__ void rect_param_count_kernel(const uint32_t* __restrict__ row_codes, uint32_t n, uint32_t K,
                                        uint32_t stride, int args, uint32_t* __restrict__ count) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int group[kRectMaxArgs], first[kRectMaxArgs];
  count[t] = (uint32_t)rect_groups(row_codes, t, K, stride, args, group, first);
}

__global__ void rect_param_coords_kernel(const uint32_t* __restrict__ row_codes, uint32_t n, uint32_t K,
                                         uint32_t stride, int args, uint32_t param_start,
                                         const uint32_t* __restrict__ outer, uint32_t* __restrict__ coords,
                                         uint16_t* __restrict__ dims) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int group[kRectMaxArgs], first[kRectMaxArgs];
  const int nr = rect_groups(row_codes, t, K, stride, args, group, first);
  uint32_t o = outer[t];
  for (int i = 0; i < nr; ++i, ++o) {
    coords[2ull * o] = row_codes[(uint64_t)t * K + (uint64_t)first[i] * stride] - 2u;
    coords[2ull * o + 1] = param_start + t;
    dims[2ull * o] = 3;
    dims[2ull * o + 1] = 1;
  }
}

// Records (3 doubles) of the parameter pairs: per row group, the sum of its
// arguments' derivatives d[t][3 a .. 3 a + 2].
__global__ void rect_param_records_kernel(const double* __restrict__ d, int args,
                                          const uint32_t* __restrict__ row_codes, uint32_t n, uint32_t K,
                                          uint32_t stride, const uint32_t* __restrict__ outer,
                                          const uint32_t* __restrict__ record, double* __restrict__ out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int group[kRectMaxArgs], first[kRectMaxArgs];
  const int nr = rect_groups(row_codes, t, K, stride, args, group, first);
  const double* src = d + 3ull * args * t;
  uint32_t o = outer[t];
  for (int i = 0; i < nr; ++i, ++o) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < args; ++a) {
      if (group[a] != i) continue;
#pragma unroll
      for (int k = 0; k < 3; ++k) acc[k] += src[3 * a + k];
    }
    double* dst = out + record[o];
#pragma unroll
    for (int k = 0; k < 3; ++k) dst[k] = acc[k];
  }
}

// First-order Jacobian of the affine-body vertex positions x_i = A_b xbar_i
// + t_b (b the body of vertex i): rows 3 i; the (3 x 9) block of A (row r
// holds xbar_i at columns 3 r .. 3 r + 2) and the (3 x 3) identity of t,
// in this order per vertex.
__global__ void affine_jacobian_coords_kernel(const uint32_t* __restrict__ vertex_body, uint32_t n, int64_t a_col,
                                              int64_t t_col, uint32_t* __restrict__ coords,
                                              uint16_t* __restrict__ dims) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t b = vertex_body[i];
  uint64_t o = (uint64_t)i * ((a_col >= 0) + (t_col >= 0));
  if (a_col >= 0) {
    coords[2 * o] = 3u * i;
    coords[2 * o + 1] = (uint32_t)(a_col + 9ll * b);
    dims[2 * o] = 3;
    dims[2 * o + 1] = 9;
    ++o;
  }
  if (t_col >= 0) {
    coords[2 * o] = 3u * i;
    coords[2 * o + 1] = (uint32_t)(t_col + 3ll * b);
    dims[2 * o] = 3;
    dims[2 * o + 1] = 3;
  }
}

__global__ void affine_jacobian_records_kernel(const double* __restrict__ xbar, uint32_t n, int with_a, int with_t,
                                               const uint32_t* __restrict__ record, double* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t o = (uint64_t)i * (with_a + with_t);
  if (with_a) {
    double* dst = out + record[o++];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 9; ++c) dst[9 * r + c] = (c / 3 == r) ? xbar[3ull * i + c % 3] : 0.0;
  }
  if (with_t) {
    double* dst = out + record[o];
    for (int k = 0; k < 9; ++k) dst[k] = (k % 4 == 0) ? 1.0 : 0.0;
  }
}

// First block of every block row (rows sorted): row_ptr[r] = lower bound.
__global__ void rect_row_ptr_kernel(const uint32_t* __restrict__ positions, uint32_t nb, uint32_t block_rows,
                                    uint32_t* __restrict__ row_ptr) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > block_rows) return;
  uint32_t lo = 0, hi = nb;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (positions[2ull * mid] / 3u < r) lo = mid + 1;
    else hi = mid;
  }
  row_ptr[r] = lo;
}

__global__ void rect_col_ptr_kernel(const uint32_t* __restrict__ keys, uint32_t nb, uint32_t block_cols,
                                    uint32_t* __restrict__ col_ptr) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > block_cols) return;
  uint32_t lo = 0, hi = nb;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (keys[mid] < c) lo = mid + 1;
    else hi = mid;
  }
  col_ptr[c] = lo;
}

__global__ void rect_col_keys_kernel(const uint32_t* __restrict__ positions, uint32_t nb, uint32_t width,
                                     uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nb) return;
  keys[u] = positions[2ull * u + 1] / width;
  vals[u] = u;
}

// Blocks of 3 rows and `width` (1, 3 or 9) columns, values row-major and
// contiguous (3 width a block).  J x: one thread an output block row, its
// blocks in order; J^T x: one thread an output column unit, its blocks in the
// stable column order.  accumulate: y += instead of y =.
__global__ void rect_spmv_kernel(const double* __restrict__ values, const uint32_t* __restrict__ positions,
                                 const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ order,
                                 uint32_t out_rows, int width, int transpose, int accumulate,
                                 const double* __restrict__ x, double* __restrict__ y) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= out_rows) return;
  const uint32_t e0 = ptr[r], e1 = ptr[r + 1];
  if (transpose && e0 == e1) return;
  // output rows are block rows of 3; output columns sit at their blocks'
  // scalar column (a column target need not start at a multiple of 3)
  const uint64_t base = transpose ? positions[2ull * (order ? order[e0] : e0) + 1] : 3ull * r;
  double s[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (uint32_t e = e0; e < e1; ++e) {
    const uint32_t u = order ? order[e] : e;
    const double* b = values + 3ull * width * u;
    if (!transpose) {
      const double* xv = x + positions[2ull * u + 1];
      for (int k = 0; k < 3; ++k)
        for (int c = 0; c < width; ++c) s[k] += b[k * width + c] * xv[c];
    } else {
      const double* xv = x + positions[2ull * u];
      for (int c = 0; c < width; ++c) s[c] += b[c] * xv[0] + b[width + c] * xv[1] + b[2 * width + c] * xv[2];
    }
  }
  const int m = transpose ? width : 3;
  double* yv = y + base;
  for (int k = 0; k < m; ++k) yv[k] = accumulate ? yv[k] + s[k] : s[k];
}

}  // namespace ys

extern "C" {

int32_t ys_rect_coordinates(const uint32_t* row_codes, const uint32_t* col_codes, uint32_t n, uint32_t K,
                            uint32_t slot_stride, uint32_t args, uint32_t* coord_outer, uint32_t* coords,
                            uint16_t* dims, void* stream) {
  YS_REQUIRE(row_codes && col_codes && coord_outer, YS_ERR_INVALID, "null argument");
  YS_REQUIRE(args >= 1 && args <= (uint32_t)ys::kRectMaxArgs, YS_ERR_INVALID, "1..8 arguments an instance");
  YS_REQUIRE((uint64_t)(args - 1) * slot_stride < K, YS_ERR_INVALID, "slot stride beyond the code row");
  cudaStream_t s = (cudaStream_t)stream;
  if (coords == nullptr) {
    // counts into coord_outer[1..n], then an inclusive scan in place
    YS_CUDA_TRY(cudaMemsetAsync(coord_outer, 0, sizeof(uint32_t), s));
    if (n == 0) return YS_OK;
    ys::rect_count_kernel<<<ys::grid_for(n, 256), 256, 0, s>>>(row_codes, col_codes, n, K, slot_stride, (int)args,
                                                              coord_outer + 1);
    YS_CHECK_LAUNCH();
    size_t tmp = 0;
    YS_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, tmp, coord_outer + 1, coord_outer + 1, (int)n, s));
    void* d_tmp = nullptr;
    YS_CUDA_TRY(cudaMallocAsync(&d_tmp, tmp, s));
    const cudaError_t e = cub::DeviceScan::InclusiveSum(d_tmp, tmp, coord_outer + 1, coord_outer + 1, (int)n, s);
    cudaFreeAsync(d_tmp, s);
    YS_CUDA_TRY(e);
    return YS_OK;
  }
  YS_REQUIRE(dims != nullptr, YS_ERR_INVALID, "null dims");
  if (n == 0) return YS_OK;
  ys::rect_coords_kernel<<<ys::grid_for(n, 256), 256, 0, s>>>(row_codes, col_codes, n, K, slot_stride, (int)args,
                                                             coord_outer, coords, dims);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_rect_records(const double* local_hessians, uint32_t args, uint32_t difference_args,
                        const uint32_t* row_codes, const uint32_t* col_codes, uint32_t n, uint32_t K,
                        uint32_t slot_stride, const uint32_t* coord_outer, const uint32_t* record, double* records,
                        void* stream) {
  YS_REQUIRE(local_hessians && row_codes && col_codes && coord_outer && record && records, YS_ERR_INVALID,
             "null argument");
  YS_REQUIRE(args >= 1 && args <= (uint32_t)ys::kRectMaxArgs, YS_ERR_INVALID, "1..8 arguments an instance");
  YS_REQUIRE(difference_args == 0 || 2 * difference_args == args, YS_ERR_INVALID,
             "difference form: args must be twice difference_args");
  if (n == 0) return YS_OK;
  ys::rect_records_kernel<<<ys::grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
      local_hessians, (int)args, (int)difference_args, row_codes, col_codes, n, K, slot_stride, coord_outer, record,
      records);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_rect_param_coordinates(const uint32_t* row_codes, uint32_t n, uint32_t K, uint32_t slot_stride,
                                  uint32_t args, uint32_t param_start, uint32_t* coord_outer, uint32_t* coords,
                                  uint16_t* dims, void* stream) {
  YS_REQUIRE(row_codes && coord_outer, YS_ERR_INVALID, "null argument");
  YS_REQUIRE(args >= 1 && args <= (uint32_t)ys::kRectMaxArgs, YS_ERR_INVALID, "1..8 arguments an instance");
  YS_REQUIRE((uint64_t)(args - 1) * slot_stride < K, YS_ERR_INVALID, "slot stride beyond the code row");
  cudaStream_t s = (cudaStream_t)stream;
  if (coords == nullptr) {
    YS_CUDA_TRY(cudaMemsetAsync(coord_outer, 0, sizeof(uint32_t), s));
    if (n == 0) return YS_OK;
    ys::rect_param_count_kernel<<<ys::grid_for(n, 256), 256, 0, s>>>(row_codes, n, K, slot_stride, (int)args,
                                                                    coord_outer + 1);
    YS_CHECK_LAUNCH();
    size_t tmp = 0;
    YS_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, tmp, coord_outer + 1, coord_outer + 1, (int)n, s));
    void* d_tmp = nullptr;
    YS_CUDA_TRY(cudaMallocAsync(&d_tmp, tmp, s));
    const cudaError_t e = cub::DeviceScan::InclusiveSum(d_tmp, tmp, coord_outer + 1, coord_outer + 1, (int)n, s);
    cudaFreeAsync(d_tmp, s);
    YS_CUDA_TRY(e);
    return YS_OK;
  }
  YS_REQUIRE(dims != nullptr, YS_ERR_INVALID, "null dims");
  if (n == 0) return YS_OK;
  ys::rect_param_coords_kernel<<<ys::grid_for(n, 256), 256, 0, s>>>(row_codes, n, K, slot_stride, (int)args,
                                                                   param_start, coord_outer, coords, dims);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_rect_param_records(const double* derivatives, uint32_t args, const uint32_t* row_codes, uint32_t n,
                              uint32_t K, uint32_t slot_stride, const uint32_t* coord_outer, const uint32_t* record,
                              double* records, void* stream) {
  YS_REQUIRE(derivatives && row_codes && coord_outer && record && records, YS_ERR_INVALID, "null argument");
  YS_REQUIRE(args >= 1 && args <= (uint32_t)ys::kRectMaxArgs, YS_ERR_INVALID, "1..8 arguments an instance");
  if (n == 0) return YS_OK;
  ys::rect_param_records_kernel<<<ys::grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
      derivatives, (int)args, row_codes, n, K, slot_stride, coord_outer, record, records);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_affine_position_jacobian(const uint32_t* vertex_body, const double* xbar, uint32_t n,
                                    int64_t a_column_start, int64_t t_column_start, uint32_t* coords,
                                    uint16_t* dims, const uint32_t* record, double* records, void* stream) {
  YS_REQUIRE(a_column_start >= 0 || t_column_start >= 0, YS_ERR_INVALID, "no column target");
  if (n == 0) return YS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (record == nullptr) {
    YS_REQUIRE(vertex_body && coords && dims, YS_ERR_INVALID, "null argument");
    ys::affine_jacobian_coords_kernel<<<ys::grid_for(n, 256), 256, 0, s>>>(vertex_body, n, a_column_start,
                                                                         t_column_start, coords, dims);
  } else {
    YS_REQUIRE(xbar && records, YS_ERR_INVALID, "null argument");
    ys::affine_jacobian_records_kernel<<<ys::grid_for(n, 256), 256, 0, s>>>(
        xbar, n, a_column_start >= 0 ? 1 : 0, t_column_start >= 0 ? 1 : 0, record, records);
  }
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_rect_plan_workspace_bytes(uint32_t num_blocks, uint64_t* bytes) {
  YS_REQUIRE(bytes != nullptr, YS_ERR_INVALID, "null output");
  size_t tmp = 0;
  const int m = (int)std::max<uint32_t>(num_blocks, 1);
  YS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                              (const uint32_t*)nullptr, (uint32_t*)nullptr, m));
  const uint64_t keys = 4ull * m;
  *bytes = 4 * ((keys + 255) / 256 * 256) + (tmp + 255) / 256 * 256;
  return YS_OK;
}

int32_t ys_rect_plan(const uint32_t* positions, uint32_t num_blocks, uint32_t block_rows, uint32_t block_cols,
                     uint32_t col_width, uint32_t* row_ptr, uint32_t* col_ptr, uint32_t* col_order, void* workspace,
                     uint64_t workspace_bytes, void* stream) {
  YS_REQUIRE(row_ptr && col_ptr && col_order, YS_ERR_INVALID, "null output");
  YS_REQUIRE(col_width == 1 || col_width == 3 || col_width == 9, YS_ERR_INVALID, "blocks 1, 3 or 9 columns wide");
  YS_REQUIRE(num_blocks == 0 || positions, YS_ERR_INVALID, "null positions");
  uint64_t need = 0;
  const int32_t rc = ys_rect_plan_workspace_bytes(num_blocks, &need);
  if (rc != YS_OK) return rc;
  YS_REQUIRE(workspace && workspace_bytes >= need, YS_ERR_INVALID, "workspace too small");
  cudaStream_t s = (cudaStream_t)stream;
  ys::rect_row_ptr_kernel<<<ys::grid_for(block_rows + 1, 256), 256, 0, s>>>(positions, num_blocks, block_rows,
                                                                            row_ptr);
  YS_CHECK_LAUNCH();
  const int m = (int)std::max<uint32_t>(num_blocks, 1);
  const uint64_t keys = (4ull * m + 255) / 256 * 256;
  uint8_t* w = static_cast<uint8_t*>(workspace);
  uint32_t* k_in = reinterpret_cast<uint32_t*>(w);
  uint32_t* v_in = reinterpret_cast<uint32_t*>(w + keys);
  uint32_t* k_out = reinterpret_cast<uint32_t*>(w + 2 * keys);
  void* tmp = w + 4 * keys;
  size_t tmp_bytes = workspace_bytes - 4 * keys;
  if (num_blocks) {
    ys::rect_col_keys_kernel<<<ys::grid_for(num_blocks, 256), 256, 0, s>>>(positions, num_blocks, col_width, k_in,
                                                                           v_in);
    YS_CHECK_LAUNCH();
    // stable: the blocks of one column stay in block order
    YS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k_in, k_out, v_in, col_order, (int)num_blocks, 0,
                                                32, s));
  }
  ys::rect_col_ptr_kernel<<<ys::grid_for(block_cols + 1, 256), 256, 0, s>>>(k_out, num_blocks, block_cols, col_ptr);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_rect_spmv(const double* values, const uint32_t* positions, const uint32_t* row_ptr,
                     const uint32_t* col_ptr, const uint32_t* col_order, uint32_t block_rows, uint32_t block_cols,
                     uint32_t col_width, const double* x, double* y, uint32_t transpose, uint32_t accumulate,
                     void* stream) {
  YS_REQUIRE(row_ptr && col_ptr && x && y, YS_ERR_INVALID, "null argument");
  YS_REQUIRE(col_width == 1 || col_width == 3 || col_width == 9, YS_ERR_INVALID, "blocks 1, 3 or 9 columns wide");
  const uint32_t out_rows = transpose ? block_cols : block_rows;
  if (out_rows == 0) return YS_OK;
  ys::rect_spmv_kernel<<<ys::grid_for(out_rows, 128), 128, 0, (cudaStream_t)stream>>>(
      values, positions, transpose ? col_ptr : row_ptr, transpose ? col_order : nullptr, out_rows, (int)col_width,
      (int)transpose, (int)accumulate, x, y);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

}  // extern "C"
