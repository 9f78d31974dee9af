// Multilevel additive Schwarz (MAS) preconditioner on the device.
//
// Follows the reference's MAS (PKG/solver/mas): levels of aggregated nodes,
// dense explicit inverses of every domain (computed in FP64, stored FP32;
// mas/cuda/local_inverse.cu:190-545, mas/local_inverse.py:40-78) and the
// weighted additive application z = sum_l w_l P_l A_l^-1 R_l r
// (mas/preconditioner.py:128-154, mas/cuda/preconditioner_apply.cu).
//
// Numeric update (once per Newton step):
//   mas_level_blocks : Galerkin block sums of level l from level l-1 blocks
//                      (fixed source order -> deterministic);
//   mas_domain_inverse: one CTA per domain assembles its dense FP64 matrix in
//                      shared memory and inverts it in place (Gauss-Jordan,
//                      the reference's default backend), writes FP32.
// Application (every PCG iteration, HBM bound on the FP32 inverses):
//   mas_restrict : packed FP32 level residuals (fixed-order child sums);
//   mas_gemv     : one CTA per domain, z_d = A_d^-1 r_d from the packed upper
//                  triangle staged in shared memory;
//   mas_collect  : z = sum_l w_l z_l(map_l(i)) fused with r^T z, r^T r and the
//                  PCG stop test (deterministic last-block reduction).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "ys_mas.cuh"
#include "ys_mas_dev.cuh"

namespace ys {

constexpr int kInvThreads = 256;

// One warp per coarse block: lane l sums sources l, l+32, ... (mode 0: B,
// 1: B^T, 2: B + B^T), then a fixed xor-shuffle tree combines the lanes, so
// the sum order is fixed (deterministic) and long source lists (the coarse
// levels) are summed 32-wide instead of serially.
__global__ void __launch_bounds__(256) mas_level_blocks(MasDev M, uint32_t begin, uint32_t end) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t cb = begin + warp;
  if (cb >= end) return;  // warp-uniform
  double acc[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) acc[e] = 0.0;
  for (uint32_t s = M.cb_src_ptr[cb] + lane; s < M.cb_src_ptr[cb + 1]; s += 32) {
    const uint32_t src = M.cb_src[s];
    const uint32_t mode = src >> 30, idx = src & 0x3fffffffu;
    const double* b = level_block(M, idx);
    double v[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) v[e] = b[e];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        const double d = v[3 * k + l], t = v[3 * l + k];
        acc[3 * k + l] += mode == 0 ? d : (mode == 1 ? t : d + t);
      }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int e = 0; e < 9; ++e) acc[e] += __shfl_xor_sync(0xffffffffu, acc[e], o);
  if (lane == 0) {
#pragma unroll
    for (int e = 0; e < 9; ++e) M.coarse_values[9ull * cb + e] = acc[e];
  }
}

// Union of two 3x3 block sets (the static set and the dynamic contact set)
// on their union pattern: block u = A[a_index[u]] + B[b_index[u]], a
// negative index standing for no block (one order, deterministic).
__global__ void union_values_kernel(const double* __restrict__ a, const int32_t* __restrict__ ai,
                                    const double* __restrict__ b, const int32_t* __restrict__ bi, uint32_t nu,
                                    double* __restrict__ out) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 9ull * nu) return;
  const uint32_t u = (uint32_t)(t / 9), e = (uint32_t)(t % 9);
  const int32_t ia = ai[u], ib = bi[u];
  double v = 0.0;
  if (ia >= 0) v = a[9ull * ia + e];
  if (ib >= 0) v += b[9ull * ib + e];
  out[t] = v;
}

// f(integral_constant<int, I>) for I = B .. E-1 (a loop whose index is a
// compile-time constant in its body).
template <int B, int E, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

// Dense assembly + in-place Gauss-Jordan inverse of one domain per CTA.
// T: register tile edge (domain size <= 16 T).
// PB pivots per blocked step (2: fits 128 registers, two CTAs per SM for the
// 96-DoF domains; 4: the 128-DoF tile, one CTA per SM).
template <int T, int PB>
__global__ void __launch_bounds__(kInvThreads, PB == 2 ? 2 : 1) mas_domain_inverse(MasDev M) {
  extern __shared__ double A[];  // n*n
  __shared__ double colb[2][128 * 4];
  __shared__ double rowb[2][4 * 128];
  __shared__ double dinv[128];
  __shared__ int bad;
  const uint32_t d = blockIdx.x;
  const uint32_t n = 3 * (M.dom_node_ptr[d + 1] - M.dom_node_ptr[d]);
  for (uint32_t i = threadIdx.x; i < n * n; i += blockDim.x) A[i] = 0.0;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  const uint32_t e0 = M.dom_entry_ptr[d], e1 = M.dom_entry_ptr[d + 1];
  for (uint64_t t = (uint64_t)e0 * 9 + threadIdx.x; t < (uint64_t)e1 * 9; t += blockDim.x) {
    const uint64_t e = t / 9;
    const int el = (int)(t % 9), k = el / 3, m = el % 3;
    const uint32_t li = M.dom_entry[3 * e], lj = M.dom_entry[3 * e + 1], bi = M.dom_entry[3 * e + 2];
    const double v = level_block(M, bi)[el];
    A[(3 * li + k) * n + 3 * lj + m] = v;
    if (li != lj) A[(3 * lj + m) * n + 3 * li + k] = v;
  }
  __syncthreads();
  // Gauss-Jordan without pivoting (SPD domains): after a step, A holds the
  // inverse in the eliminated columns.  Relative pivot tolerance 1e-12 of
  // the largest diagonal entry (mas/local_inverse.py:43-65).
  // Thread (ty, tx) of a 16 x 16 grid owns rows ty + 16a and columns tx + 16b
  // (a, b < T) in registers.  The matrix is first scaled to unit diagonal,
  // S = D^-1/2 A D^-1/2 (pivots in (0, 1]); the inverse is D^-1/2 S^-1 D^-1/2;
  // a scalar pivot below 1e-12 (or a non-positive diagonal) marks the domain
  // singular.  The order is padded to a multiple of PB with identity rows.
  // Blocked steps of PB pivots K: with P = S[K,K], C = S[:,K] except
  // C[K,:] = P - I and R = S[K,:] except R[:,K] = P + I, the one update
  //   S -= (C P^-1) R
  // gives the scaled rows P^-1 S[K,:], the columns -S[:,K] P^-1 and P^-1 in
  // place, so the update is pure FMAs; the owners of the next block's rows and
  // columns publish them to double-buffered shared memory, one barrier a step.
  const uint32_t np = (n + PB - 1) / PB * PB;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double dii = A[i * n + i];
    if (!(dii > 0.0)) bad = 1;
    dinv[i] = dii > 0.0 ? rsqrt(dii) : 1.0;
  }
  __syncthreads();
  const double tol = 1.0e-12;
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  double R[T][T];
#pragma unroll
  for (int a = 0; a < T; ++a)
#pragma unroll
    for (int b = 0; b < T; ++b) {
      const uint32_t i = ty + 16 * a, j = tx + 16 * b;
      R[a][b] = (i < n && j < n) ? A[i * n + j] * dinv[i] * dinv[j] : (i == j && i < np ? 1.0 : 0.0);
    }
  // PB == 2 runs the symmetric form (the sweep operator): with v = S[:,K]
  // except v[K,:] = P - I, the update S -= (v P^-1) v^T and then S[k,k] -= 2
  // on the pivots sweeps K; after every pivot S holds -S_0^-1.  The update is
  // symmetric, so only the upper register tiles (a <= b) are kept: v is read
  // from the published column K for rows in tiles up to the pivot's and from
  // the published row K beyond it, never from a lower tile.
  constexpr bool kSweep = PB == 2;
  // publish block k: colb[buf][i][m] = C[i][m], rowb[buf][m][j] = R[m][j].
  // Block k lies in register column/row KB = PB k / 16 of its owners; KB is a
  // compile-time constant (the step loop is unrolled over it), so the owners
  // read their tile entries directly.
  auto publish = [&](auto kb_c, uint32_t k) {
    constexpr int KB = decltype(kb_c)::value;
    const int base = (int)((PB * k) & 15), buf = (int)(k & 1);
    if (tx >= base && tx < base + PB) {
      const int m = tx - base;
#pragma unroll
      for (int a = 0; a < T; ++a) {
        if (kSweep && a > KB) continue;  // lower tile: not kept (consumers read row K there)
        const double v = R[a][KB];
        const bool diag = (ty + 16 * a) == (int)(PB * k) + m;
        colb[buf][(ty + 16 * a) * PB + m] = diag ? v - 1.0 : v;
      }
    }
    if (ty >= base && ty < base + PB) {
      const int m = ty - base;
#pragma unroll
      for (int b = 0; b < T; ++b) {
        if (kSweep && b < KB) continue;  // lower tile: not kept (consumers read column K there)
        const double v = R[KB][b];
        const bool diag = (tx + 16 * b) == (int)(PB * k) + m;
        rowb[buf][m * 128 + tx + 16 * b] = diag ? (kSweep ? v - 1.0 : v + 1.0) : v;
      }
    }
  };
  constexpr int kSteps = 16 / PB;  // blocked steps per register column
  publish(std::integral_constant<int, 0>{}, 0u);
  __syncthreads();
  const uint32_t nblk = np / PB;
  static_for<0, T>([&](auto kb_c) {
  constexpr int KB = decltype(kb_c)::value;
  for (int sub = 0; sub < kSteps; ++sub) {
    const uint32_t k = (uint32_t)(KB * kSteps + sub);
    if (k >= nblk) break;
    const int buf = (int)(k & 1);
    double P[PB][PB];
    if constexpr (PB == 2) {
      const double q00 = colb[buf][(2 * k) * 2] + 1.0, q01 = colb[buf][(2 * k) * 2 + 1];
      const double q10 = colb[buf][(2 * k + 1) * 2], q11 = colb[buf][(2 * k + 1) * 2 + 1] + 1.0;
      const double da = q00 * q11 - q01 * q10;
      const double ida = 1.0 / da;
      P[0][0] = q11 * ida; P[0][1] = -q01 * ida; P[1][0] = -q10 * ida; P[1][1] = q00 * ida;
      if (!(q00 > tol && da > tol * q00) && threadIdx.x == 0) bad = 1;
    } else {
    // P^-1 of the 4x4 pivot block (every thread alike) by 2x2 blocks:
    // P = [A B; B' D], S = D - B' A^-1 B, P^-1 = [A^-1 + E S^-1 E', -E S^-1;
    // -S^-1 E', S^-1] with E = A^-1 B (P is symmetric up to rounding; the
    // blocks are read as stored).  The leading pivot and the Schur
    // determinant carry the singularity test.
      double q[4][4];
#pragma unroll
      for (int l = 0; l < 4; ++l)
#pragma unroll
        for (int m = 0; m < 4; ++m) q[l][m] = colb[buf][(4 * k + l) * 4 + m] + (l == m ? 1.0 : 0.0);
      const double da = q[0][0] * q[1][1] - q[0][1] * q[1][0];
      const double ida = 1.0 / da;
      const double ai00 = q[1][1] * ida, ai01 = -q[0][1] * ida, ai10 = -q[1][0] * ida, ai11 = q[0][0] * ida;
      // E = A^-1 B (2x2), F = C A^-1 (2x2), S = D - C A^-1 B
      const double e00 = ai00 * q[0][2] + ai01 * q[1][2], e01 = ai00 * q[0][3] + ai01 * q[1][3];
      const double e10 = ai10 * q[0][2] + ai11 * q[1][2], e11 = ai10 * q[0][3] + ai11 * q[1][3];
      const double f00 = q[2][0] * ai00 + q[2][1] * ai10, f01 = q[2][0] * ai01 + q[2][1] * ai11;
      const double f10 = q[3][0] * ai00 + q[3][1] * ai10, f11 = q[3][0] * ai01 + q[3][1] * ai11;
      const double s00 = q[2][2] - (q[2][0] * e00 + q[2][1] * e10), s01 = q[2][3] - (q[2][0] * e01 + q[2][1] * e11);
      const double s10 = q[3][2] - (q[3][0] * e00 + q[3][1] * e10), s11 = q[3][3] - (q[3][0] * e01 + q[3][1] * e11);
      const double ds = s00 * s11 - s01 * s10;
      const double ids = 1.0 / ds;
      const double si00 = s11 * ids, si01 = -s01 * ids, si10 = -s10 * ids, si11 = s00 * ids;
      // bottom right S^-1, top right -E S^-1, bottom left -S^-1 F, top left A^-1 + E S^-1 F
      P[2][2] = si00; P[2][3] = si01; P[3][2] = si10; P[3][3] = si11;
      P[0][2] = -(e00 * si00 + e01 * si10); P[0][3] = -(e00 * si01 + e01 * si11);
      P[1][2] = -(e10 * si00 + e11 * si10); P[1][3] = -(e10 * si01 + e11 * si11);
      P[2][0] = -(si00 * f00 + si01 * f10); P[2][1] = -(si00 * f01 + si01 * f11);
      P[3][0] = -(si10 * f00 + si11 * f10); P[3][1] = -(si10 * f01 + si11 * f11);
      P[0][0] = ai00 - (P[0][2] * f00 + P[0][3] * f10); P[0][1] = ai01 - (P[0][2] * f01 + P[0][3] * f11);
      P[1][0] = ai10 - (P[1][2] * f00 + P[1][3] * f10); P[1][1] = ai11 - (P[1][2] * f01 + P[1][3] * f11);
      // scalar pivots of the same elimination: q00, da / q00, and the two of S
      const bool ok = q[0][0] > tol && da > tol * q[0][0] && s00 > tol && ds > tol * s00;
      if (!ok && threadIdx.x == 0) bad = 1;
    }
    double rj[PB][T];
#pragma unroll
    for (int m = 0; m < PB; ++m)
#pragma unroll
      for (int b = 0; b < T; ++b)
        rj[m][b] = (!kSweep || b >= KB) ? rowb[buf][m * 128 + tx + 16 * b] : colb[buf][(tx + 16 * b) * PB + m];
#pragma unroll
    for (int a = 0; a < T; ++a) {
      double c[PB];
#pragma unroll
      for (int l = 0; l < PB; ++l)
        c[l] = (!kSweep || a <= KB) ? colb[buf][(ty + 16 * a) * PB + l] : rowb[buf][l * 128 + ty + 16 * a];
      double w[PB];
#pragma unroll
      for (int m = 0; m < PB; ++m) {
        double acc = 0.0;
#pragma unroll
        for (int l = 0; l < PB; ++l) acc += c[l] * P[l][m];
        w[m] = acc;
      }
#pragma unroll
      for (int b = 0; b < T; ++b) {
        if (kSweep && a > b) continue;  // lower tile: never read
        double v = R[a][b];
#pragma unroll
        for (int m = 0; m < PB; ++m) v = fma(-w[m], rj[m][b], v);
        R[a][b] = v;
      }
    }
    if constexpr (kSweep) {
      // the swept pivots' diagonal: 2 I - P^-1 -> -P^-1
      const int base = (int)((PB * k) & 15);
      if (ty == tx && ty >= base && ty < base + PB) R[KB][KB] -= 2.0;
    }
    if (k + 1 < nblk) {
      if (sub + 1 < kSteps) {
        publish(kb_c, k + 1);
      } else {
        if constexpr (KB + 1 < T) publish(std::integral_constant<int, KB + 1>{}, k + 1);
      }
    }
    __syncthreads();
  }
  });
  if (threadIdx.x == 0 && bad) atomicAdd(M.status, 1);
  // FP32 upper 4x4 tiles (inv_tile_slot order), straight from the register
  // tiles; the padding rows and columns up to 4 * inv_tiles(n) are zero.
  float* out = M.inverse + M.inv_offset[d];
  const uint32_t nt = inv_tiles(n);
#pragma unroll
  for (int a = 0; a < T; ++a) {
    const uint32_t i = ty + 16 * a;
    const uint32_t rb = inv_tile_rowbase(nt, i >> 2);
#pragma unroll
    for (int b = 0; b < T; ++b) {
      if (kSweep && a > b) continue;  // strictly lower: no upper 4x4 tile there
      const uint32_t j = tx + 16 * b;
      if (i < 4 * nt && j < 4 * nt && (i >> 2) <= (j >> 2)) {
        const double r = kSweep ? -R[a][b] : R[a][b];  // the sweep leaves -S^-1
        const float v = (i < n && j < n) ? (float)(r * dinv[i] * dinv[j]) : 0.0f;
        out[16u * (rb + (j >> 2)) + 4 * (i & 3) + (j & 3)] = v;
      }
    }
  }
}

// Level 0: a thread per node; levels >= 1: a warp per node.
__global__ void mas_restrict(MasDev M, const double* __restrict__ r, uint32_t level) {
  const uint32_t begin = M.level_node_offset[level], end = M.level_node_offset[level + 1];
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (level == 0) {
    const uint32_t p = begin + t;
    if (p >= end) return;
    M.rl[3ull * p] = (float)r[3ull * p];
    M.rl[3ull * p + 1] = (float)r[3ull * p + 1];
    M.rl[3ull * p + 2] = (float)r[3ull * p + 2];
    return;
  }
  const uint32_t p = begin + (t >> 5);
  if (p >= end) return;  // warp-uniform
  restrict_node_warp(M, r, level, p, (int)(t & 31));
}

__host__ inline unsigned restrict_grid(uint32_t level, uint32_t cnt) {
  return grid_for(level == 0 ? (uint64_t)cnt : 32ull * cnt, 256);
}

// All levels from `first` to the coarsest in one CTA (small levels: the
// launch would cost more than the work), level by level.
__global__ void __launch_bounds__(1024) mas_restrict_tail(MasDev M, const double* __restrict__ r, uint32_t first) {
  restrict_tail_levels(M, r, first);
}

// Domains d0 .. d0 + gridDim.x - 1.
__global__ void __launch_bounds__(kGemvThreads) mas_gemv(MasDev M, uint32_t d0) {
  extern __shared__ float4 gemv_smem[];
  gemv_domain(M, d0 + blockIdx.x, gemv_smem);
}

struct MasPcg {
  MasDev M;
  SpmvSet sets[2];
  int nsets;
  int fp32;
  uint32_t nv;
  const double* rhs;
  double* x;
  double* r;
  double* p;
  float4* p32;  // FP32 copy of p for the FP32 SpMV, else null
  double* q;
  double* z;
  double* st;
  double* partials;
  unsigned* tickets;
  int stop_rule;
  int zero_guess;
  double tolerance;
  uint32_t max_it;
  cudaGraphConditionalHandle cond;
};

__global__ void __launch_bounds__(kPcgBlock) mas_init_residual(MasPcg P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.nv) return;
  double r0 = P.rhs[3ull * i], r1 = P.rhs[3ull * i + 1], r2 = P.rhs[3ull * i + 2];
  if (P.zero_guess) {
    P.x[3ull * i] = 0.0; P.x[3ull * i + 1] = 0.0; P.x[3ull * i + 2] = 0.0;
  } else {
    double h0, h1, h2;
    spmv3_row(P.sets, P.nsets, P.fp32, i, P.x, h0, h1, h2);
    r0 -= h0; r1 -= h1; r2 -= h2;
  }
  P.r[3ull * i] = r0; P.r[3ull * i + 1] = r1; P.r[3ull * i + 2] = r2;
  P.M.rl[3ull * i] = (float)r0; P.M.rl[3ull * i + 1] = (float)r1; P.M.rl[3ull * i + 2] = (float)r2;
}

__device__ __forceinline__ void collect_node(const MasPcg& P, uint32_t i, double (&z)[3]) {
  collect_levels(P.M, P.nv, i, z);
}

// z = M^-1 r; p = z; r^T z, r^T r, g^T g; stop threshold; loop flag.
__global__ void __launch_bounds__(kPcgBlock) mas_init_collect(MasPcg P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[3] = {0.0, 0.0, 0.0};
  if (i < P.nv) {
    double z[3];
    collect_node(P, i, z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double r = P.r[3ull * i + k], g = P.rhs[3ull * i + k];
      P.z[3ull * i + k] = z[k];
      P.p[3ull * i + k] = z[k];
      v[0] += r * z[k];
      v[1] += r * r;
      v[2] += g * g;
    }
    if (P.p32) P.p32[i] = make_float4((float)z[0], (float)z[1], (float)z[2], 0.0f);
  }
  if (!grid_reduce_last<3>(v, P.partials, P.tickets)) return;
  if (threadIdx.x != 0) return;
  double* st = P.st;
  const double delta = v[0];
  st[kDeltaNew] = delta;
  st[kDelta0] = delta;
  st[kRR] = v[1];
  st[kRR0] = v[1];
  st[kGG] = v[2];
  st[kIter] = 0.0;
  st[kAlpha] = 0.0;
  st[kBeta] = 0.0;
  st[kBarrierFail] = 0.0;
  st[kRestart] = 0.0;
  int status = kContinue;
  double tol;
  if (P.stop_rule == YS_STOP_RESIDUAL) {
    tol = P.st[kTolParam] * P.st[kTolParam] * v[2];
    if (!(isfinite(v[1]) && isfinite(v[2]))) status = kInvalidInit;
    else if (v[1] <= tol) status = kConverged;
    else if (!(isfinite(delta) && delta > 0.0)) status = kInvalidInit;
  } else {
    // mas/pcg.py:44-66: converged when r^T z <= tol * reference.
    tol = P.st[kTolParam] * delta;
    if (!(isfinite(delta) && delta >= 0.0)) status = kInvalidInit;
    else if (delta <= tol) status = kConverged;
    else if (!(delta > 0.0)) status = kInvalidInit;
  }
  if (status == kContinue && P.st[kMaxItParam] < 1.0) status = kMaxIter;
  st[kTolAbs] = tol;
  st[kStatus] = (double)status;
  cudaGraphSetConditional(P.cond, status == kContinue ? 1u : 0u);
}

__global__ void __launch_bounds__(kPcgBlock) mas_update(MasPcg P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.nv || P.st[kStatus] != (double)kContinue) return;
  const double alpha = P.st[kAlpha];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    P.x[3ull * i + k] = P.x[3ull * i + k] + P.p[3ull * i + k] * alpha;
    const double r = P.r[3ull * i + k] - P.q[3ull * i + k] * alpha;
    P.r[3ull * i + k] = r;
    P.M.rl[3ull * i + k] = (float)r;  // level-0 restriction fused
  }
}

// mas_update fused with the level-1 restriction: a warp per level-1 node
// updates the node's children (lanes stride them as restrict_node_warp does)
// and sums their new residuals in the same order, so the level-1 values are
// bit-identical to a separate restriction pass.  Every fine variable is the
// child of exactly one level-1 node.
__global__ void __launch_bounds__(kPcgBlock) mas_update_restrict(MasPcg P) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t p = P.M.level_node_offset[1] + (t >> 5);
  if (p >= P.M.level_node_offset[2] || P.st[kStatus] != (double)kContinue) return;  // warp-uniform
  const int lane = (int)(t & 31);
  const double alpha = P.st[kAlpha];
  const uint32_t c = p - P.M.nv;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (uint32_t q = P.M.child_ptr[c] + lane; q < P.M.child_ptr[c + 1]; q += 32) {
    const uint32_t i = P.M.child_fine[q];
    double r[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      P.x[3ull * i + k] = P.x[3ull * i + k] + P.p[3ull * i + k] * alpha;
      r[k] = P.r[3ull * i + k] - P.q[3ull * i + k] * alpha;
      P.r[3ull * i + k] = r[k];
      P.M.rl[3ull * i + k] = (float)r[k];
    }
    s0 += r[0]; s1 += r[1]; s2 += r[2];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    P.M.rl64[3ull * p] = s0;
    P.M.rl64[3ull * p + 1] = s1;
    P.M.rl64[3ull * p + 2] = s2;
    P.M.rl[3ull * p] = (float)s0;
    P.M.rl[3ull * p + 1] = (float)s1;
    P.M.rl[3ull * p + 2] = (float)s2;
  }
}

__global__ void __launch_bounds__(kPcgBlock) mas_iter_collect(MasPcg P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = P.st[kStatus] == (double)kContinue;
  double v[2] = {0.0, 0.0};
  if (i < P.nv && live) {
    double z[3];
    collect_node(P, i, z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double r = P.r[3ull * i + k];
      P.z[3ull * i + k] = z[k];
      v[0] += r * z[k];
      v[1] += r * r;
    }
  }
  if (!grid_reduce_last<2>(v, P.partials, P.tickets + 2)) return;
  if (threadIdx.x != 0 || !live) return;
  double* st = P.st;
  const double next = v[0], prev = st[kDeltaOld];
  const double it = st[kIter] + 1.0;
  st[kIter] = it;
  st[kDeltaNew] = next;
  st[kRR] = v[1];
  int status = kContinue;
  // mas/pcg.py:80-98
  if (!isfinite(next) || next < 0.0 || !isfinite(prev) || prev <= 0.0) {
    st[kBeta] = 0.0;
    status = kNonSpd;
  } else {
    // after a zero step (non-positive curvature) the direction restarts
    // from z = M^-1 r (mas/cuda/pcg.cu:240)
    st[kBeta] = st[kRestart] != 0.0 ? 0.0 : next / prev;
    st[kRestart] = 0.0;
    const bool done = P.stop_rule == YS_STOP_RESIDUAL ? v[1] <= st[kTolAbs] : next <= st[kTolAbs];
    if (done) status = kConverged;
    else if (next == 0.0) status = kNonSpd;
    else if (it >= P.st[kMaxItParam]) status = kMaxIter;
  }
  st[kStatus] = (double)status;
  cudaGraphSetConditional(P.cond, status == kContinue ? 1u : 0u);
}

// mas_iter_collect and pcg_direction in one cooperative (co-resident) grid:
// each thread collects z for its nodes (the first two kept in registers,
// further ones through P.z), the blocks meet at a grid barrier whose last
// arriving block finishes the reductions and the iteration bookkeeping (the
// code of mas_iter_collect, same order), then every thread sets p = z +
// beta p for its nodes.  The barrier wait is bounded: a block that gives up
// marks the solve void (kBarrierFail) and skips the direction.
__global__ void __launch_bounds__(kPcgBlock) mas_iter_collect_direction(MasPcg P) {
  __shared__ double red[kPcgBlock / 32];
  __shared__ int last;
  __shared__ int ok;
  double* st = P.st;
  const bool live = st[kStatus] == (double)kContinue;
  if (!live) return;  // grid-uniform: nobody writes the status before the barrier
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  double z0[3] = {0.0, 0.0, 0.0}, z1[3] = {0.0, 0.0, 0.0};
  double v[2] = {0.0, 0.0};
  uint32_t kk = 0;
  for (uint32_t i = i0; i < P.nv; i += stride, ++kk) {
    double z[3];
    collect_node(P, i, z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double r = P.r[3ull * i + k];
      v[0] += r * z[k];
      v[1] += r * r;
    }
    if (kk == 0) {
#pragma unroll
      for (int k = 0; k < 3; ++k) z0[k] = z[k];
    } else if (kk == 1) {
#pragma unroll
      for (int k = 0; k < 3; ++k) z1[k] = z[k];
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k) P.z[3ull * i + k] = z[k];
    }
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double sk = block_sum<kPcgBlock>(v[k], red);
    if (threadIdx.x == 0) P.partials[(uint64_t)k * gridDim.x + blockIdx.x] = sk;
  }
  unsigned* count = P.tickets + 4;
  unsigned* gen = P.tickets + 5;
  __syncthreads();
  unsigned g0 = 0;
  if (threadIdx.x == 0) {
    g0 = atomicAdd(gen, 0u);
    __threadfence();
    last = atomicAdd(count, 1u) == gridDim.x - 1;
    ok = 1;
  }
  __syncthreads();
  if (last) {
    __threadfence();
#pragma unroll
    for (int k = 0; k < 2; ++k)
      v[k] = block_sum<kPcgBlock>(thread_partial_sum(P.partials + (uint64_t)k * gridDim.x, gridDim.x), red);
    if (threadIdx.x == 0) {
      const double next = v[0], prev = st[kDeltaOld];
      const double it = st[kIter] + 1.0;
      st[kIter] = it;
      st[kDeltaNew] = next;
      st[kRR] = v[1];
      int status = kContinue;
      // mas/pcg.py:80-98
      if (!isfinite(next) || next < 0.0 || !isfinite(prev) || prev <= 0.0) {
        st[kBeta] = 0.0;
        status = kNonSpd;
      } else {
        st[kBeta] = st[kRestart] != 0.0 ? 0.0 : next / prev;  // restart: see mas_iter_collect
        st[kRestart] = 0.0;
        const bool done = P.stop_rule == YS_STOP_RESIDUAL ? v[1] <= st[kTolAbs] : next <= st[kTolAbs];
        if (done) status = kConverged;
        else if (next == 0.0) status = kNonSpd;
        else if (it >= st[kMaxItParam]) status = kMaxIter;
      }
      st[kStatus] = (double)status;
      cudaGraphSetConditional(P.cond, status == kContinue ? 1u : 0u);
      *count = 0u;
      __threadfence();
      atomicAdd(gen, 1u);  // release
    }
  } else if (threadIdx.x == 0) {
    // bounded wait for the release (the grid is co-resident, so the last
    // block always arrives; the bound, kPollLimitParam polls, only keeps a
    // failure from hanging: a block that gives up voids the solve)
    const double limit = *(volatile double*)&st[kPollLimitParam];
    uint32_t spins = 0;
    while (atomicAdd(gen, 0u) == g0) {
      if ((double)spins >= limit) {
        ok = 0;
        st[kBarrierFail] = 1.0;
        break;
      }
      ++spins;
      __nanosleep(64);
    }
    __threadfence();
  }
  __syncthreads();
  if (!ok) return;
  const double st_status = *(volatile double*)&st[kStatus];
  if (st_status == (double)kNonSpd) return;
  const double beta = *(volatile double*)&st[kBeta];
  kk = 0;
  for (uint32_t i = i0; i < P.nv; i += stride, ++kk) {
    double z[3];
    if (kk == 0) {
#pragma unroll
      for (int k = 0; k < 3; ++k) z[k] = z0[k];
    } else if (kk == 1) {
#pragma unroll
      for (int k = 0; k < 3; ++k) z[k] = z1[k];
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k) z[k] = P.z[3ull * i + k];
    }
    double p[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      p[k] = z[k] + P.p[3ull * i + k] * beta;
      P.p[3ull * i + k] = p[k];
    }
    if (P.p32) P.p32[i] = make_float4((float)p[0], (float)p[1], (float)p[2], 0.0f);
  }
}

__global__ void __launch_bounds__(kPcgBlock) mas_collect_only(MasPcg P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.nv) return;
  double z[3];
  collect_node(P, i, z);
#pragma unroll
  for (int k = 0; k < 3; ++k) P.z[3ull * i + k] = z[k];
}

struct MasHandle {
  MasDev M;
  std::vector<uint32_t> cb_level_begin;
  std::vector<MasPcg*> pcgs;
  int* status_host = nullptr;
  int64_t fine_domains = -1;  // level-0 domains (the first ones), looked up once
};

// Number of level-0 domains: domains are numbered level by level, so they
// are the first ones and cover exactly the level-0 nodes.
static cudaError_t fine_domain_count(MasHandle* h, uint32_t* out) {
  if (h->fine_domains < 0) {
    const MasDev& M = h->M;
    std::vector<uint32_t> ptr(M.num_domains + 1);
    const cudaError_t e =
        cudaMemcpy(ptr.data(), M.dom_node_ptr, sizeof(uint32_t) * ptr.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    const uint32_t end = M.levels > 1 ? M.level_node_offset[1] : ptr.back();
    h->fine_domains = std::lower_bound(ptr.begin(), ptr.end(), end) - ptr.begin();
  }
  *out = (uint32_t)h->fine_domains;
  return cudaSuccess;
}

const MasDev* mas_device_state(void* handle) { return handle ? &static_cast<MasHandle*>(handle)->M : nullptr; }

static cudaError_t add_kernel(cudaGraph_t g, cudaGraphNode_t* node, const cudaGraphNode_t* deps, size_t ndeps,
                              const void* fn, unsigned grid, unsigned block, size_t smem, void** args) {
  cudaKernelNodeParams kp{};
  kp.func = const_cast<void*>(fn);
  kp.gridDim = dim3(grid);
  kp.blockDim = dim3(block);
  kp.sharedMemBytes = (unsigned)smem;
  kp.kernelParams = args;
  return cudaGraphAddKernelNode(node, g, deps, ndeps, &kp);
}

// z_l = A_l^-1 r_l for every domain, as two branches joined by an empty
// node: the level-0 domains need only the level-0 residual (written by the
// kernel that produces r), so their GEMV runs beside the restriction chain
// of the coarse levels (grid restrictions, the one-CTA tail) and the GEMV of
// the coarse domains that follows it.
static cudaError_t add_apply_nodes(MasHandle* h, const MasDev& M, cudaGraph_t g, const cudaGraphNode_t* deps,
                                   size_t ndeps, cudaGraphNode_t* last, const double* r, uint32_t restricted) {
  MasDev m = M;
  const double* rr = r;
  uint32_t fine = 0;
  cudaError_t e = fine_domain_count(h, &fine);
  if (e != cudaSuccess) return e;
  const unsigned smem = (unsigned)gemv_smem_bytes(M.max_dofs);
  cudaGraphNode_t fine_gemv = nullptr;
  uint32_t d0 = 0;
  void* af[] = {&m, &d0};
  e = add_kernel(g, &fine_gemv, deps, ndeps, (const void*)mas_gemv, fine, kGemvThreads, smem, af);
  if (e != cudaSuccess || fine == M.num_domains) {
    *last = fine_gemv;
    return e;
  }
  // The coarse chain is a string of small launches: at the greatest
  // priority its CTAs are dispatched ahead of the waiting level-0 GEMV CTAs,
  // so it finishes under the GEMV instead of after it.
  int least = 0, greatest = 0;
  e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (e != cudaSuccess) return e;
  cudaKernelNodeAttrValue prio{};
  prio.priority = greatest;
  const uint32_t first = restrict_tail_first(M);
  const cudaGraphNode_t* dp = deps;
  size_t nd = ndeps;
  cudaGraphNode_t prev = nullptr;
  // levels up to `restricted` are written by the kernel that produces r
  for (uint32_t l = restricted + 1; l < first && e == cudaSuccess; ++l) {
    uint32_t level = l;
    void* a1[] = {&m, &rr, &level};
    const uint32_t cnt = M.level_node_offset[l + 1] - M.level_node_offset[l];
    cudaGraphNode_t n = nullptr;
    e = add_kernel(g, &n, dp, nd, (const void*)mas_restrict, restrict_grid(l, cnt), 256, 0, a1);
    if (e == cudaSuccess) e = cudaGraphKernelNodeSetAttribute(n, cudaKernelNodeAttributePriority, &prio);
    prev = n;
    dp = &prev;
    nd = 1;
  }
  uint32_t f = first > restricted ? first : restricted + 1;
  if (e == cudaSuccess && f < M.levels) {
    void* a1[] = {&m, &rr, &f};
    cudaGraphNode_t n = nullptr;
    e = add_kernel(g, &n, dp, nd, (const void*)mas_restrict_tail, 1, 1024, 0, a1);
    if (e == cudaSuccess) e = cudaGraphKernelNodeSetAttribute(n, cudaKernelNodeAttributePriority, &prio);
    prev = n;
    dp = &prev;
    nd = 1;
  }
  if (e != cudaSuccess) return e;
  cudaGraphNode_t coarse_gemv = nullptr;
  uint32_t d1 = fine;
  void* ac[] = {&m, &d1};
  e = add_kernel(g, &coarse_gemv, dp, nd, (const void*)mas_gemv, M.num_domains - fine, kGemvThreads, smem, ac);
  if (e == cudaSuccess) e = cudaGraphKernelNodeSetAttribute(coarse_gemv, cudaKernelNodeAttributePriority, &prio);
  if (e != cudaSuccess) return e;
  const cudaGraphNode_t both[2] = {fine_gemv, coarse_gemv};
  return cudaGraphAddEmptyNode(last, g, both, 2);
}

cudaError_t mas_add_init_nodes(void* mas, cudaGraph_t g, const cudaGraphNode_t* deps, size_t ndeps,
                               cudaGraphNode_t* last, uint32_t nv, const double* rhs, double* x, double* r, double* p,
                               float4* p32, double* q, double* z, double* st, double* partials, unsigned* tickets, const SpmvSet* sets,
                               int nsets, int fp32, int stop_rule, int zero_guess, double tolerance, uint32_t max_it,
                               cudaGraphConditionalHandle cond, MasPcgHooks* hooks) {
  auto* h = static_cast<MasHandle*>(mas);
  if (h->M.nv != nv) return cudaErrorInvalidValue;
  if (!zero_guess) return cudaErrorNotSupported;
  auto* P = new MasPcg{};
  P->M = h->M;
  for (int s = 0; s < nsets; ++s) P->sets[s] = sets[s];
  P->nsets = nsets;
  P->fp32 = fp32;
  P->nv = nv;
  P->rhs = rhs;
  P->x = x;
  P->r = r;
  P->p = p;
  P->p32 = p32;
  P->q = q;
  P->z = z;
  P->st = st;
  P->partials = partials;
  P->tickets = tickets;
  P->stop_rule = stop_rule;
  P->zero_guess = zero_guess;
  P->tolerance = tolerance;
  P->max_it = max_it;
  P->cond = cond;
  h->pcgs.push_back(P);
  hooks->params = P;
  const unsigned grid = grid_for(nv, kPcgBlock);
  cudaGraphNode_t n0 = nullptr, n1 = nullptr, n2 = nullptr;
  void* a0[] = {P};
  cudaError_t e = add_kernel(g, &n0, deps, ndeps, (const void*)mas_init_residual, grid, kPcgBlock, 0, a0);
  if (e == cudaSuccess) e = add_apply_nodes(h, P->M, g, &n0, 1, &n1, r, 0u);
  if (e == cudaSuccess) e = add_kernel(g, &n2, &n1, 1, (const void*)mas_init_collect, grid, kPcgBlock, 0, a0);
  *last = n2;
  return e;
}

cudaError_t mas_add_update_nodes(void* mas, cudaGraph_t body, const cudaGraphNode_t* deps, size_t ndeps,
                                 cudaGraphNode_t* last, MasPcgHooks* hooks) {
  auto* h = static_cast<MasHandle*>(mas);
  auto* P = static_cast<MasPcg*>(hooks->params);
  const unsigned grid = grid_for(P->nv, kPcgBlock);
  cudaGraphNode_t n0 = nullptr, n1 = nullptr, n2 = nullptr;
  void* a0[] = {P};
  // with a level 1, the update writes the level-1 residuals too
  const bool fused = P->M.levels > 1;
  const unsigned grid1 = fused ? grid_for(32ull * (P->M.level_node_offset[2] - P->M.level_node_offset[1]), kPcgBlock) : grid;
  cudaError_t e = add_kernel(body, &n0, deps, ndeps, fused ? (const void*)mas_update_restrict : (const void*)mas_update,
                             grid1, kPcgBlock, 0, a0);
  if (e == cudaSuccess) e = add_apply_nodes(h, P->M, body, &n0, 1, &n1, P->r, fused ? 1u : 0u);
  // collect + direction as one cooperative kernel when the device takes it
  // (co-resident grid); otherwise mas_iter_collect and pcg_direction
  if (e == cudaSuccess) {
    int dev = 0, sms = 0, per_sm = 0, coop = 0;
    const void* fn = (const void*)mas_iter_collect_direction;
    bool fused = cudaGetDevice(&dev) == cudaSuccess &&
                 cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && coop &&
                 cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
                 cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPcgBlock, 0) == cudaSuccess && per_sm > 0;
    if (fused) {
      const unsigned cgrid = std::min<unsigned>(grid, (unsigned)(sms * per_sm));
      e = add_kernel(body, &n2, &n1, 1, fn, cgrid, kPcgBlock, 0, a0);
      cudaKernelNodeAttrValue cv{};
      cv.cooperative = 1;
      if (e == cudaSuccess) e = cudaGraphKernelNodeSetAttribute(n2, cudaKernelNodeAttributeCooperative, &cv);
      if (e == cudaSuccess) hooks->fused_direction = true;
    } else {
      e = add_kernel(body, &n2, &n1, 1, (const void*)mas_iter_collect, grid, kPcgBlock, 0, a0);
    }
  }
  *last = n2;
  return e;
}

}  // namespace ys

extern "C" {

int32_t ys_mas_create(const ys_mas_desc* d, void** handle) {
  YS_REQUIRE(d && handle, YS_ERR_INVALID, "null argument");
  YS_REQUIRE(d->num_levels >= 1 && d->num_levels <= ys::kMaxLevels, YS_ERR_INVALID, "1..8 levels");
  YS_REQUIRE(d->max_domain_dofs >= 3 && d->max_domain_dofs <= 128, YS_ERR_INVALID, "domain DoF must be <= 128");
  auto* h = new ys::MasHandle();
  ys::MasDev& M = h->M;
  M.nv = d->num_fine_vars;
  M.levels = d->num_levels;
  for (uint32_t l = 0; l <= d->num_levels; ++l) M.level_node_offset[l] = d->level_node_offset[l];
  for (uint32_t l = 0; l < d->num_levels; ++l) M.weight[l] = (float)d->level_weights[l];
  M.packed_nodes = d->level_node_offset[d->num_levels];
  M.cmap = d->cmap;
  M.child_ptr = d->child_ptr;
  M.child_fine = d->child_fine;
  M.num_domains = d->num_domains;
  M.dom_node_ptr = d->dom_node_ptr;
  M.dom_nodes = d->dom_nodes;
  M.inv_offset = d->inv_offset;
  M.dom_entry_ptr = d->dom_entry_ptr;
  M.dom_entry = d->dom_entry;
  M.fine_blocks = d->fine_blocks;
  M.coarse_blocks = d->coarse_blocks;
  M.cb_src_ptr = d->cb_src_ptr;
  M.cb_src = d->cb_src;
  for (uint32_t l = 0; l <= d->num_levels; ++l) M.cb_level_begin[l] = d->cb_level_begin[l];
  M.coarse_values = d->coarse_values;
  M.inverse = d->inverse;
  M.rl = d->level_residual;
  M.rl64 = d->level_residual64;
  M.zl = d->level_correction;
  M.status = d->status;
  M.max_dofs = d->max_domain_dofs;
  M.fine_values = nullptr;
  cudaError_t e = cudaSuccess;
  {
    const size_t smem = sizeof(double) * d->max_domain_dofs * d->max_domain_dofs;
    e = cudaFuncSetAttribute(ys::mas_domain_inverse<6, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(ys::mas_domain_inverse<8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // prefer the largest shared-memory carveout so two 96-DoF domains fit per SM
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(ys::mas_domain_inverse<6, 2>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(ys::mas_domain_inverse<8, 4>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  }
  if (e != cudaSuccess) {
    ys_set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    if (h->status_host) cudaFreeHost(h->status_host);
    delete h;
    return YS_ERR_CUDA;
  }
  *handle = h;
  return YS_OK;
}

int32_t ys_mas_union_values(const double* a, const int32_t* a_index, const double* b, const int32_t* b_index,
                            uint32_t num_blocks, double* out, void* stream) {
  YS_REQUIRE(out && a_index && b_index, YS_ERR_INVALID, "null argument");
  if (num_blocks == 0) return YS_OK;
  ys::union_values_kernel<<<ys::grid_for(9ull * num_blocks, 256), 256, 0, (cudaStream_t)stream>>>(
      a, a_index, b, b_index, num_blocks, out);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_mas_numeric_update(void* handle, const double* fine_values, void* stream, int32_t* failed_domains) {
  YS_REQUIRE(handle, YS_ERR_INVALID, "null handle");
  auto* h = static_cast<ys::MasHandle*>(handle);
  cudaStream_t s = (cudaStream_t)stream;
  ys::MasDev& M = h->M;
  M.fine_values = fine_values;
  for (auto* p : h->pcgs) p->M.fine_values = fine_values;
  YS_CUDA_TRY(cudaMemsetAsync(M.status, 0, sizeof(int), s));
  for (uint32_t l = 1; l < M.levels; ++l) {
    const uint32_t b = M.cb_level_begin[l], e = M.cb_level_begin[l + 1];
    if (e > b) {
      ys::mas_level_blocks<<<ys::grid_for(32ull * (e - b), 256), 256, 0, s>>>(M, b, e);
      YS_CHECK_LAUNCH();
    }
  }
  const size_t smem = sizeof(double) * M.max_dofs * M.max_dofs;
  if (M.max_dofs <= 96)
    ys::mas_domain_inverse<6, 2><<<M.num_domains, ys::kInvThreads, smem, s>>>(M);
  else
    ys::mas_domain_inverse<8, 4><<<M.num_domains, ys::kInvThreads, smem, s>>>(M);
  YS_CHECK_LAUNCH();
  if (failed_domains) {
    // pinned status word, allocated on first use (callers that never ask,
    // such as the serving loop, never synchronise on a host allocation)
    if (!h->status_host) YS_CUDA_TRY(cudaMallocHost(&h->status_host, sizeof(int)));
    YS_CUDA_TRY(cudaMemcpyAsync(h->status_host, M.status, sizeof(int), cudaMemcpyDeviceToHost, s));
    YS_CUDA_TRY(cudaStreamSynchronize(s));
    *failed_domains = *h->status_host;
    if (*failed_domains) return YS_ERR_SINGULAR_DOMAIN;
  }
  return YS_OK;
}

int32_t ys_mas_failed_domains(void* handle, void* stream, int32_t* failed_domains) {
  YS_REQUIRE(handle && failed_domains, YS_ERR_INVALID, "null argument");
  auto* h = static_cast<ys::MasHandle*>(handle);
  cudaStream_t s = (cudaStream_t)stream;
  if (!h->status_host) YS_CUDA_TRY(cudaMallocHost(&h->status_host, sizeof(int)));
  YS_CUDA_TRY(cudaMemcpyAsync(h->status_host, h->M.status, sizeof(int), cudaMemcpyDeviceToHost, s));
  YS_CUDA_TRY(cudaStreamSynchronize(s));
  *failed_domains = *h->status_host;
  return *failed_domains ? YS_ERR_SINGULAR_DOMAIN : YS_OK;
}

int32_t ys_mas_apply(void* handle, const double* r, double* z, void* stream) {
  YS_REQUIRE(handle, YS_ERR_INVALID, "null handle");
  auto* h = static_cast<ys::MasHandle*>(handle);
  cudaStream_t s = (cudaStream_t)stream;
  ys::MasDev& M = h->M;
  for (uint32_t l = 0; l < M.levels; ++l) {
    const uint32_t cnt = M.level_node_offset[l + 1] - M.level_node_offset[l];
    ys::mas_restrict<<<ys::restrict_grid(l, cnt), 256, 0, s>>>(M, r, l);
    YS_CHECK_LAUNCH();
  }
  ys::mas_gemv<<<M.num_domains, ys::kGemvThreads, ys::gemv_smem_bytes(M.max_dofs), s>>>(M, 0u);
  YS_CHECK_LAUNCH();
  ys::MasPcg P{};
  P.M = M;
  P.nv = M.nv;
  P.z = z;
  ys::mas_collect_only<<<ys::grid_for(M.nv, ys::kPcgBlock), ys::kPcgBlock, 0, s>>>(P);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

uint64_t ys_mas_inverse_floats(uint32_t dofs) { return ys::inv_floats(dofs); }

int32_t ys_mas_gemv(void* handle, void* stream, uint64_t* algorithmic_bytes) {
  YS_REQUIRE(handle, YS_ERR_INVALID, "null handle");
  auto* h = static_cast<ys::MasHandle*>(handle);
  ys::MasDev& M = h->M;
  if (algorithmic_bytes) {
    // the distinct entries of every FP32 inverse (its upper triangle, read
    // once) + the gathered residual, the node ids and the correction; the
    // tile layout reads ~3 % more (padding, full diagonal tiles)
    std::vector<uint32_t> ptr(M.num_domains + 1);
    cudaMemcpy(ptr.data(), M.dom_node_ptr, sizeof(uint32_t) * (M.num_domains + 1), cudaMemcpyDeviceToHost);
    uint64_t bytes = 0;
    for (uint32_t d = 0; d < M.num_domains; ++d) {
      const uint64_t n = 3ull * (ptr[d + 1] - ptr[d]);
      bytes += 4 * (n * (n + 1) / 2) + 4 * n + 4 * n + 4 * (n / 3);
    }
    *algorithmic_bytes = bytes;
  }
  ys::mas_gemv<<<M.num_domains, ys::kGemvThreads, ys::gemv_smem_bytes(M.max_dofs), (cudaStream_t)stream>>>(M, 0u);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_mas_destroy(void* handle) {
  if (!handle) return YS_OK;
  auto* h = static_cast<ys::MasHandle*>(handle);
  for (auto* p : h->pcgs) delete p;
  if (h->status_host) cudaFreeHost(h->status_host);
  delete h;
  return YS_OK;
}

}  // extern "C"
