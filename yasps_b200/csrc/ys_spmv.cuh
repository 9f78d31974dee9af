// Symmetric 3x3-block SpMV row gather (shared by ys_spmv.cu and the PCG/MAS kernels).
//
// Storage: the reference's upper-triangle, duplicate-free block COO
// (PKG/matrixAndVector/matrix/matrix.pyx:101-113); a block (r, c) with r < c
// implies its transpose.  The row plan lists, for variable i, the stored
// blocks with row i (direct) and col i (transposed, flag bit 31), so every
// output row is a gather with a fixed summation order: deterministic and
// free of atomics.  The second read of an off-diagonal block (from the other
// row) is an L2 hit when rows are processed in (Morton) order.
#pragma once

#include "ys_common.cuh"

namespace ys {

struct SpmvSet {
  const double* values;
  const float* values32;
  const uint32_t* row_ptr;
  const uint32_t* entry_block;
  const uint32_t* entry_col;
};

// Block values: FP64 blocks are the reference's 9 doubles per block; the FP32
// copy keeps every block in a 16-byte aligned slot of 12 floats (3 float4
// loads per block instead of 9 scalar ones: a third of the L1/L2 requests;
// a run of slots is also one 16-byte aligned stream for bulk copies).
constexpr uint32_t kFp32BlockStride = 12;

__device__ __forceinline__ void load_block(const double* __restrict__ vals, uint32_t eb, double (&b)[9]) {
  const double* p = vals + 9ull * eb;
#pragma unroll
  for (int k = 0; k < 9; ++k) b[k] = __ldg(p + k);
}

__device__ __forceinline__ void load_block(const float* __restrict__ vals, uint32_t eb, float (&b)[9]) {
  const float4* p = reinterpret_cast<const float4*>(vals + (uint64_t)kFp32BlockStride * eb);
  const float4 v0 = __ldg(p), v1 = __ldg(p + 1), v2 = __ldg(p + 2);
  b[0] = v0.x; b[1] = v0.y; b[2] = v0.z; b[3] = v0.w;
  b[4] = v1.x; b[5] = v1.y; b[6] = v1.z; b[7] = v1.w;
  b[8] = v2.x;
}

// Neighbour vector gather: FP64 x (three scalar loads, rounded to T), or the
// FP32 copy in 16-byte slots (x, y, z, 0) per variable (one float4 load; the
// copy holds the same roundings, so both give the same products).
template <typename T>
__device__ __forceinline__ void load_x(const double* __restrict__ x, uint32_t j, T (&v)[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = (T)__ldg(x + 3ull * j + k);
}

__device__ __forceinline__ void load_x(const float4* __restrict__ x, uint32_t j, float (&v)[3]) {
  const float4 t = __ldg(x + j);
  v[0] = t.x; v[1] = t.y; v[2] = t.z;
}

__device__ __forceinline__ float mac(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double mac(double a, double b, double c) { return __fma_rn(a, b, c); }

// a += B x (or B^T x for a transposed entry) as explicit fused multiply-add
// chains: the rounding is fixed by the source, not by how the compiler
// contracts, so every kernel that gathers a row gets the same bits.
template <typename T>
__device__ __forceinline__ void block_mac(const T (&b)[9], const T (&x)[3], bool transposed, T& a0, T& a1, T& a2) {
  if (transposed) {
    a0 = mac(b[6], x[2], mac(b[3], x[1], mac(b[0], x[0], a0)));
    a1 = mac(b[7], x[2], mac(b[4], x[1], mac(b[1], x[0], a1)));
    a2 = mac(b[8], x[2], mac(b[5], x[1], mac(b[2], x[0], a2)));
  } else {
    a0 = mac(b[2], x[2], mac(b[1], x[1], mac(b[0], x[0], a0)));
    a1 = mac(b[5], x[2], mac(b[4], x[1], mac(b[3], x[0], a1)));
    a2 = mac(b[8], x[2], mac(b[7], x[1], mac(b[6], x[0], a2)));
  }
}

template <typename T>
__device__ __forceinline__ void spmv3_row_accumulate(const T* __restrict__ vals, const uint32_t* __restrict__ row_ptr,
                                                     const uint32_t* __restrict__ eblock,
                                                     const uint32_t* __restrict__ ecol, uint32_t i,
                                                     const double* __restrict__ x, double& y0, double& y1,
                                                     double& y2) {
  const uint32_t e0 = row_ptr[i], e1 = row_ptr[i + 1];
  T a0 = 0, a1 = 0, a2 = 0;
  for (uint32_t e = e0; e < e1; ++e) {
    const uint32_t eb = __ldg(eblock + e);
    const uint32_t j = __ldg(ecol + e);
    T bv[9], xv[3];
    load_block(vals, eb & 0x7fffffffu, bv);
    load_x(x, j, xv);
    block_mac(bv, xv, (eb & 0x80000000u) != 0, a0, a1, a2);
  }
  y0 += (double)a0;
  y1 += (double)a1;
  y2 += (double)a2;
}

// Row gather by a group of kRowLanes lanes: lane l handles entries l, l+8, ...
// of the row; the partial sums are combined by a fixed shuffle tree, so the
// result is deterministic.  Every lane of the warp executes the same
// shuffles: a row beyond the matrix passes an empty entry range.
constexpr int kRowLanes = 8;

template <typename T, typename X>
__device__ __forceinline__ void spmv3_group_accumulate(const T* __restrict__ vals, uint32_t e0, uint32_t e1,
                                                       const uint32_t* __restrict__ eblock,
                                                       const uint32_t* __restrict__ ecol, int lane,
                                                       const X* __restrict__ x, double& y0, double& y1,
                                                       double& y2) {
  T a0 = 0, a1 = 0, a2 = 0;
  // Two entries per iteration (e and e + kRowLanes): both index loads, then
  // both value/vector gathers are in flight before any use.
  for (uint32_t e = e0 + lane; e < e1; e += 2 * kRowLanes) {
    const uint32_t f = e + kRowLanes;
    const bool two = f < e1;
    const uint32_t ebA = __ldg(eblock + e), jA = __ldg(ecol + e);
    const uint32_t ebB = two ? __ldg(eblock + f) : ebA, jB = two ? __ldg(ecol + f) : jA;
    T xa[3], xb[3], ba[9], bb[9];
    load_x(x, jA, xa);
    load_x(x, jB, xb);
    load_block(vals, ebA & 0x7fffffffu, ba);
    load_block(vals, ebB & 0x7fffffffu, bb);
    const T wB = two ? (T)1 : (T)0;
#pragma unroll
    for (int k = 0; k < 3; ++k) xb[k] *= wB;
    block_mac(ba, xa, (ebA & 0x80000000u) != 0, a0, a1, a2);
    block_mac(bb, xb, (ebB & 0x80000000u) != 0, a0, a1, a2);
  }
#pragma unroll
  for (int o = kRowLanes / 2; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o, kRowLanes);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o, kRowLanes);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o, kRowLanes);
  }
  y0 += (double)a0;
  y1 += (double)a1;
  y2 += (double)a2;
}

// Group version over the (up to two) block sets; every lane of the warp must
// call it, rows beyond the matrix with valid == false.
__device__ __forceinline__ void spmv3_group(const SpmvSet* sets, int nsets, bool fp32, uint32_t i, bool valid,
                                            int lane, const double* __restrict__ x, double& y0, double& y1,
                                            double& y2) {
  y0 = y1 = y2 = 0.0;
  for (int s = 0; s < nsets; ++s) {
    const uint32_t e0 = valid ? sets[s].row_ptr[i] : 0u;
    const uint32_t e1 = valid ? sets[s].row_ptr[i + 1] : 0u;
    if (fp32)
      spmv3_group_accumulate<float>(sets[s].values32, e0, e1, sets[s].entry_block, sets[s].entry_col, lane, x, y0,
                                    y1, y2);
    else
      spmv3_group_accumulate<double>(sets[s].values, e0, e1, sets[s].entry_block, sets[s].entry_col, lane, x, y0,
                                     y1, y2);
  }
}

// FP32 group version reading the float4 copy of x.
__device__ __forceinline__ void spmv3_group_x32(const SpmvSet* sets, int nsets, uint32_t i, bool valid, int lane,
                                                const float4* __restrict__ x32, double& y0, double& y1, double& y2) {
  y0 = y1 = y2 = 0.0;
  for (int s = 0; s < nsets; ++s) {
    const uint32_t e0 = valid ? sets[s].row_ptr[i] : 0u;
    const uint32_t e1 = valid ? sets[s].row_ptr[i + 1] : 0u;
    spmv3_group_accumulate<float>(sets[s].values32, e0, e1, sets[s].entry_block, sets[s].entry_col, lane, x32, y0, y1,
                                  y2);
  }
}

// y_i = sum over the (up to two) block sets.
__device__ __forceinline__ void spmv3_row(const SpmvSet* sets, int nsets, bool fp32, uint32_t i,
                                          const double* __restrict__ x, double& y0, double& y1, double& y2) {
  y0 = y1 = y2 = 0.0;
  for (int s = 0; s < nsets; ++s) {
    if (fp32)
      spmv3_row_accumulate<float>(sets[s].values32, sets[s].row_ptr, sets[s].entry_block, sets[s].entry_col, i, x, y0,
                                  y1, y2);
    else
      spmv3_row_accumulate<double>(sets[s].values, sets[s].row_ptr, sets[s].entry_block, sets[s].entry_col, i, x, y0,
                                   y1, y2);
  }
}

}  // namespace ys
