// Element evaluation: Stable Neo-Hookean tetrahedra and implicit-Euler inertia.
//
// SNH (examples/dropping_in_container_mixed/helpers.py:102-127):
//   F = Ds Dm^-1, IC = |F|^2, J = det F,
//   E = vol * (mu/2 (IC-3) - mu/2 log(IC+1) + lam/2 (J - 1 - 3mu/(4lam))^2) * dt^2.
// With G = D Dm^-1 (4x3, D the edge-difference matrix) the 12x12 local
// Hessian is A = B^T M B, B = G^T (x) I3, M = vol dt^2 d2psi/dF2, and its
// 3x3 block (a, b) is
//   s [c1 (G_a.G_b) I + c2 (F G_a)(F G_b)^T + lam (cof G_a)(cof G_b)^T + c3 X(F (G_a x G_b))]
// with c1 = mu (1 - 1/(IC+1)), c2 = 2 mu/(IC+1)^2, c3 = lam (J - alpha) and
// X(w)[k][l] = eps_klp w_p.
//
// Projection (the reference projects this full 12x12 matrix,
// PKG/differentiator/differentiator.pyx:794-799, hessianKernelHeader.pyx:224-252):
// the exact LDL^T PSD test runs on A; for the others, W = G^T G = L L^T gives
// A = U^T K U with U = (L^-1 G^T) (x) I3 having orthonormal rows, so the
// nonzero spectrum of A is that of the 9x9 K = (I (x) L)^T M (I (x) L) and
// proj(A) = U^T proj(K) U exactly (the 3 translation modes of A are zero).  K
// has the same block form as A with G_a replaced by the columns of L.
//
// Two passes: `snh_eval_kernel` (one thread per tet) computes the gradient and
// A, runs the PSD test and writes records for the PSD tets; tets that need the
// eigen-solve are compacted into a work list and finished by
// `snh_project_kernel`, so the expensive path runs without divergence.
#include "ys_ad.cuh"
#include "ys_common.cuh"
#include "ys_eigen.cuh"

namespace ys {

struct V3 {
  double x, y, z;
};
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// 3x3 matrix stored by columns c0, c1, c2.
struct M3 {
  V3 c[3];
};
__device__ __forceinline__ V3 mul(const M3& m, V3 v) { return v.x * m.c[0] + v.y * m.c[1] + v.z * m.c[2]; }

__device__ __forceinline__ V3 load3(const ys_union3& u, uint32_t idx) {
  uint32_t c = 0;
#pragma unroll
  for (int k = 1; k < YS_MAX_UNION; ++k)
    if (k < (int)u.num_children && idx >= u.prefix[k]) c = k;
  const double* p = u.child[c] + 3ull * (idx - u.prefix[c]);
  return {__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}

// Per-tet kinematics shared by both passes.
struct SnhState {
  V3 g[4];        // rows of G (one per vertex)
  M3 f;           // deformation gradient (columns)
  M3 cof;         // cofactor matrix (columns)
  double s;       // vol * dt^2
  double c1, c2, c3, lam;
  double energy;
  V3 grad[4];
};

__device__ __forceinline__ void snh_state(const ys_snh_args& a, uint32_t t, SnhState& st) {
  const uint4 tv = reinterpret_cast<const uint4*>(a.tets)[t];
  const uint32_t id[4] = {tv.x, tv.y, tv.z, tv.w};
  V3 x[4], r[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    x[k] = load3(a.position, id[k]);
    r[k] = load3(a.rest, id[k]);
  }
  const V3 e0 = r[1] - r[0], e1 = r[2] - r[0], e2 = r[3] - r[0];
  // Dm = [e0 e1 e2] (columns); Dm^-1 rows are (e1 x e2, e2 x e0, e0 x e1) / det.
  const V3 k0 = cross(e1, e2), k1 = cross(e2, e0), k2 = cross(e0, e1);
  const double det = dot(e0, k0);
  const double inv = 1.0 / det;
  // IB row i = k_i / det; G_{a} = IB row (a-1), G_0 = -(sum of IB rows).
  st.g[1] = inv * k0;
  st.g[2] = inv * k1;
  st.g[3] = inv * k2;
  st.g[0] = -1.0 * (st.g[1] + st.g[2] + st.g[3]);
  // F columns f_j = sum_a x_a G[a][j].
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    V3 col = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 4; ++k) col = col + comp(st.g[k], j) * x[k];
    st.f.c[j] = col;
  }
  st.cof.c[0] = cross(st.f.c[1], st.f.c[2]);
  st.cof.c[1] = cross(st.f.c[2], st.f.c[0]);
  st.cof.c[2] = cross(st.f.c[0], st.f.c[1]);
  const double mu = a.mu ? a.mu[t] : a.mu_value;
  const double lam = a.lam ? a.lam[t] : a.lam_value;
  const double ic = dot(st.f.c[0], st.f.c[0]) + dot(st.f.c[1], st.f.c[1]) + dot(st.f.c[2], st.f.c[2]);
  const double J = dot(st.f.c[0], st.cof.c[0]);
  const double alpha = 1.0 + 0.75 * mu / lam;
  const double vol = det / 6.0;
  st.s = vol * a.dt * a.dt;
  st.lam = lam;
  st.c1 = mu * (1.0 - 1.0 / (ic + 1.0));
  st.c2 = 2.0 * mu / ((ic + 1.0) * (ic + 1.0));
  st.c3 = lam * (J - alpha);
  st.energy = st.s * (0.5 * mu * (ic - 3.0) - 0.5 * mu * log(ic + 1.0) + 0.5 * lam * (J - alpha) * (J - alpha));
  // P = c1 F + c3 cof; grad_a = s P G_a^T.
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const V3 pf = mul(st.f, st.g[k]);
    const V3 pc = mul(st.cof, st.g[k]);
    st.grad[k] = st.s * (st.c1 * pf + st.c3 * pc);
  }
}

// 3x3 block of the form s [c1 (ga.gb) I + c2 u_a u_b^T + lam v_a v_b^T + c3 X(F (ga x gb))].
__device__ __forceinline__ void hess_block(const SnhState& st, V3 ga, V3 gb, V3 ua, V3 ub, V3 va, V3 vb,
                                           double (&blk)[3][3]) {
  const double d = st.c1 * dot(ga, gb);
  const V3 w = mul(st.f, cross(ga, gb));
  const double ua_[3] = {ua.x, ua.y, ua.z}, ub_[3] = {ub.x, ub.y, ub.z};
  const double va_[3] = {va.x, va.y, va.z}, vb_[3] = {vb.x, vb.y, vb.z};
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int l = 0; l < 3; ++l) blk[k][l] = st.c2 * ua_[k] * ub_[l] + st.lam * va_[k] * vb_[l] + (k == l ? d : 0.0);
  // X(w) = [[0, w2, -w1], [-w2, 0, w0], [w1, -w0, 0]]
  blk[0][1] += st.c3 * w.z;
  blk[0][2] -= st.c3 * w.y;
  blk[1][0] -= st.c3 * w.z;
  blk[1][2] += st.c3 * w.x;
  blk[2][0] += st.c3 * w.y;
  blk[2][1] -= st.c3 * w.x;
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int l = 0; l < 3; ++l) blk[k][l] *= st.s;
}

// Scatter of one instance's projected local Hessian (4 arguments of size 3)
// into pattern records, merging repeated target arguments and transposing
// blocks whose row DoF exceeds the column DoF (hessianKernelNoProject.pyx:94-264).
template <typename BlockFn>
__device__ __forceinline__ void write_hessian_records(const uint32_t (&code)[4], uint32_t occ0,
                                                      const uint32_t* __restrict__ record, double* __restrict__ out,
                                                      BlockFn&& block) {
  bool dup = false;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = a + 1; b < 4; ++b) dup |= (code[a] >= 2 && code[a] == code[b]);
  if (!dup) {
    // Common case: every target argument is its own group (compile-time indices).
    uint32_t occ = occ0;
#pragma unroll
    for (int ai = 0; ai < 4; ++ai) {
      if (code[ai] < 2) continue;
#pragma unroll
      for (int bi = ai; bi < 4; ++bi) {
        if (code[bi] < 2) continue;
        double blk[3][3];
        block(ai, bi, blk);
        double* dst = out + record[occ++];
        const bool upper = code[ai] < code[bi];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int l = 0; l < 3; ++l) dst[3 * k + l] = upper ? blk[k][l] : blk[l][k];
      }
    }
    return;
  }
  int first[4];
  int nfirst = 0;
  int group[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    group[a] = -1;
    if (code[a] < 2) continue;
    int gsel = -1;
    for (int q = 0; q < nfirst; ++q)
      if (code[first[q]] == code[a]) gsel = q;
    if (gsel < 0) { first[nfirst] = a; gsel = nfirst++; }
    group[a] = gsel;
  }
  uint32_t occ = occ0;
  for (int gi = 0; gi < nfirst; ++gi) {
    for (int gj = gi; gj < nfirst; ++gj) {
      double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int a = 0; a < 4; ++a) {
        if (group[a] != gi) continue;
        for (int b = 0; b < 4; ++b) {
          if (group[b] != gj) continue;
          double blk[3][3];
          block(a, b, blk);
#pragma unroll
          for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int l = 0; l < 3; ++l) acc[k][l] += blk[k][l];
        }
      }
      double* dst = out + record[occ];
      const bool upper = code[first[gi]] < code[first[gj]];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) dst[3 * k + l] = upper ? acc[k][l] : acc[l][k];
      ++occ;
    }
  }
}

__device__ __forceinline__ void write_gradient_records(const uint32_t (&code)[4], uint32_t q0,
                                                       const uint32_t* __restrict__ grec, double* __restrict__ out,
                                                       const V3 (&grad)[4]) {
  uint32_t q = q0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    if (code[a] < 2) continue;
    double* dst = out + grec[q++];
    dst[0] = grad[a].x;
    dst[1] = grad[a].y;
    dst[2] = grad[a].z;
  }
}

__device__ __forceinline__ void load_codes(const ys_term_plan& p, uint32_t t, uint32_t (&code)[4]) {
#pragma unroll
  for (int a = 0; a < 4; ++a) code[a] = p.codes[(uint64_t)t * p.K + (uint64_t)a * p.slot_stride];
}

__global__ void __launch_bounds__(128) snh_eval_kernel(const ys_snh_args a) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.num_elements) return;
  SnhState st;
  snh_state(a, t, st);
  uint32_t code[4];
  load_codes(a.plan, t, code);
  if (a.energy) a.energy[t] = st.energy;
  write_gradient_records(code, a.plan.grad_outer[t], a.plan.grad_record, a.grad_records, st.grad);
  V3 u[4], v[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    u[k] = mul(st.f, st.g[k]);
    v[k] = mul(st.cof, st.g[k]);
  }
  auto block = [&](int ai, int bi, double (&blk)[3][3]) {
    hess_block(st, st.g[ai], st.g[bi], u[ai], u[bi], v[ai], v[bi], blk);
  };
  if (a.projection_method >= 1) {
    double s[78];
#pragma unroll
    for (int ai = 0; ai < 4; ++ai) {
#pragma unroll
      for (int bi = 0; bi <= ai; ++bi) {
        double blk[3][3];
        hess_block(st, st.g[ai], st.g[bi], u[ai], u[bi], v[ai], v[bi], blk);
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int l = 0; l < 3; ++l) {
            const int r = 3 * ai + k, c = 3 * bi + l;
            if (c <= r) s[tri(r, c)] = blk[k][l];
          }
      }
    }
    if (!psd_test_packed<12>(s)) {
      const uint32_t slot = atomicAdd(a.work_count, 1u);
      a.work_list[slot] = t;
      return;
    }
  }
  write_hessian_records(code, a.plan.coord_outer[t], a.plan.record, a.block_records, block);
}

// Lower Cholesky of a 3x3 SPD matrix W given by its entries.
__device__ __forceinline__ bool chol3(double w00, double w01, double w02, double w11, double w12, double w22,
                                      double (&l)[3][3]) {
  if (!(w00 > 0.0)) return false;
  const double l00 = sqrt(w00);
  const double l10 = w01 / l00, l20 = w02 / l00;
  const double d1 = w11 - l10 * l10;
  if (!(d1 > 0.0)) return false;
  const double l11 = sqrt(d1);
  const double l21 = (w12 - l20 * l10) / l11;
  const double d2 = w22 - l20 * l20 - l21 * l21;
  if (!(d2 > 0.0)) return false;
  const double l22 = sqrt(d2);
  l[0][0] = l00; l[0][1] = 0.0; l[0][2] = 0.0;
  l[1][0] = l10; l[1][1] = l11; l[1][2] = 0.0;
  l[2][0] = l20; l[2][1] = l21; l[2][2] = l22;
  return true;
}

__device__ __forceinline__ void snh_project_one(const ys_snh_args& a, uint32_t t, double* __restrict__ stash,
                                                int stride) {
  SnhState st;
  snh_state(a, t, st);
  uint32_t code[4];
  load_codes(a.plan, t, code);
  // W = G^T G (3x3 over the column index j).
  double w[3][3];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < 4; ++k) acc += comp(st.g[k], j) * comp(st.g[k], m);
      w[j][m] = acc;
    }
  double l[3][3];
  const bool ok = chol3(w[0][0], w[0][1], w[0][2], w[1][1], w[1][2], w[2][2], l);
  if (!ok) {
    // Degenerate rest tetrahedron: no finite projection exists; keep A as is.
    V3 u[4], v[4];
    for (int k = 0; k < 4; ++k) { u[k] = mul(st.f, st.g[k]); v[k] = mul(st.cof, st.g[k]); }
    auto raw = [&](int ai, int bi, double (&blk)[3][3]) {
      hess_block(st, st.g[ai], st.g[bi], u[ai], u[bi], v[ai], v[bi], blk);
    };
    write_hessian_records(code, a.plan.coord_outer[t], a.plan.record, a.block_records, raw);
    return;
  }
  // Columns of L play the role of G in K.
  V3 lc[3], lu[3], lv[3];
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    lc[p] = {l[0][p], l[1][p], l[2][p]};
    lu[p] = mul(st.f, lc[p]);
    lv[p] = mul(st.cof, lc[p]);
  }
  // Q = G L^-T: Q[a][p] = sum_j G[a][j] (L^-1)[p][j]; solve L y = G_a per vertex.
  constexpr int QS = project_stash_doubles<9>();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double g0 = st.g[k].x, g1 = st.g[k].y, g2 = st.g[k].z;
    const double y0 = g0 / l[0][0];
    const double y1 = (g1 - l[1][0] * y0) / l[1][1];
    const double y2 = (g2 - l[2][0] * y0 - l[2][1] * y1) / l[2][2];
    stash[(QS + 3 * k) * stride] = y0;
    stash[(QS + 3 * k + 1) * stride] = y1;
    stash[(QS + 3 * k + 2) * stride] = y2;
  }
  // K (9x9, packed upper triangle in registers), projected in place.
  double kmat[45];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = p; q < 3; ++q) {
      double blk[3][3];
      hess_block(st, lc[p], lc[q], lu[p], lu[q], lv[p], lv[q], blk);
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int m = 0; m < 3; ++m)
          if (3 * p + k <= 3 * q + m) kmat[utri<9>(3 * p + k, 3 * q + m)] = blk[k][m];
    }
  project_negative_modes<9>(kmat, a.projection_method, stash, stride);
  double qm[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int p = 0; p < 3; ++p) qm[k][p] = stash[(QS + 3 * k + p) * stride];
  auto block = [&](int ai, int bi, double (&blk)[3][3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        double acc = 0.0;
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
          for (int q = 0; q < 3; ++q) acc += qm[ai][p] * qm[bi][q] * kmat[utri<9>(3 * p + k, 3 * q + m)];
        blk[k][m] = acc;
      }
  };
  write_hessian_records(code, a.plan.coord_outer[t], a.plan.record, a.block_records, block);
}

constexpr int kProjThreads = 64;

// Per-thread shared-memory stash of the projection (original K, reflectors,
// Q), thread-interleaved.
constexpr int kProjStash = project_stash_doubles<9>() + 12;

__global__ void __launch_bounds__(kProjThreads) snh_project_kernel(const ys_snh_args a) {
  extern __shared__ double proj_stash[];
  double* stash = proj_stash + threadIdx.x;
  const uint32_t count = *a.work_count;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    snh_project_one(a, a.work_list[i], stash, blockDim.x);
}

// Unprojected 12x12 local Hessian A of every tet (packed upper, 78 doubles),
// from the same blocks as the records of snh_eval_kernel.
__global__ void __launch_bounds__(128) snh_local_hessian_kernel(const ys_snh_args a, double* out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.num_elements) return;
  SnhState st;
  snh_state(a, t, st);
  V3 u[4], v[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    u[k] = mul(st.f, st.g[k]);
    v[k] = mul(st.cof, st.g[k]);
  }
  double* dst = out + (uint64_t)t * 78;
#pragma unroll
  for (int ai = 0; ai < 4; ++ai)
#pragma unroll
    for (int bi = ai; bi < 4; ++bi) {
      double blk[3][3];
      hess_block(st, st.g[ai], st.g[bi], u[ai], u[bi], v[ai], v[bi], blk);
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l)
          if (3 * ai + k <= 3 * bi + l) dst[utri<12>(3 * ai + k, 3 * bi + l)] = blk[k][l];
    }
}

// ---- SNH with respect to the rest positions too ----------------------------
// The position gradient s (c1 F G_k + c3 cof G_k) of the same SNH formulas,
// differentiated in the rest positions of one vertex at a time by a
// first-order dual number over its 3 coordinates (the current positions held
// constant): the position-rest block d(dE/dx)/dX of the tet's Hessian.
struct D3 {
  double v, d[3];
};
__device__ __forceinline__ D3 d3c(double c) { return D3{c, {0.0, 0.0, 0.0}}; }
__device__ __forceinline__ D3 operator+(const D3& a, const D3& b) {
  return D3{a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}};
}
__device__ __forceinline__ D3 operator-(const D3& a, const D3& b) {
  return D3{a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]}};
}
__device__ __forceinline__ D3 operator*(const D3& a, const D3& b) {
  return D3{a.v * b.v, {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2]}};
}
__device__ __forceinline__ D3 operator*(double s, const D3& a) { return D3{s * a.v, {s * a.d[0], s * a.d[1], s * a.d[2]}}; }
__device__ __forceinline__ D3 d3_recip(const D3& a) {
  const double i = 1.0 / a.v, di = -i * i;
  return D3{i, {di * a.d[0], di * a.d[1], di * a.d[2]}};
}

// x-X block (12 x 3) of rest vertex `va`: out[3k + c][m] = d(dE/dx_kc)/dX_va,m.
__device__ void snh_rest_column(const double (&x)[4][3], const double (&X)[4][3], int va, double mu, double lam,
                                double dt, double (&out)[12][3]) {
  D3 P[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      P[k][c] = d3c(X[k][c]);
      if (k == va) P[k][c].d[c] = 1.0;
    }
  D3 e[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) e[k][c] = P[k + 1][c] - P[0][c];
  auto crossc = [&](const D3 (&a)[3], const D3 (&b)[3], D3 (&o)[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  D3 k0[3], k1[3], k2[3];
  crossc(e[1], e[2], k0);
  crossc(e[2], e[0], k1);
  crossc(e[0], e[1], k2);
  const D3 det = e[0][0] * k0[0] + e[0][1] * k0[1] + e[0][2] * k0[2];
  const D3 inv = d3_recip(det);
  D3 G[4][3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    G[1][j] = k0[j] * inv;
    G[2][j] = k1[j] * inv;
    G[3][j] = k2[j] * inv;
    G[0][j] = -1.0 * (G[1][j] + G[2][j] + G[3][j]);
  }
  D3 F[3][3];  // columns f_j
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      D3 acc = x[0][c] * G[0][j];
#pragma unroll
      for (int k = 1; k < 4; ++k) acc = acc + x[k][c] * G[k][j];
      F[j][c] = acc;
    }
  D3 C[3][3];
  crossc(F[1], F[2], C[0]);
  crossc(F[2], F[0], C[1]);
  crossc(F[0], F[1], C[2]);
  D3 ic = d3c(0.0);
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int c = 0; c < 3; ++c) ic = ic + F[j][c] * F[j][c];
  const D3 J = F[0][0] * C[0][0] + F[0][1] * C[0][1] + F[0][2] * C[0][2];
  const double alpha = 1.0 + 0.75 * mu / lam;
  const D3 s = (dt * dt / 6.0) * det;
  const D3 c1 = mu * (d3c(1.0) - d3_recip(ic + d3c(1.0)));
  const D3 c3 = lam * (J - d3c(alpha));
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      D3 pf = G[k][0] * F[0][c], pc = G[k][0] * C[0][c];
#pragma unroll
      for (int j = 1; j < 3; ++j) {
        pf = pf + G[k][j] * F[j][c];
        pc = pc + G[k][j] * C[j][c];
      }
      const D3 gx = s * (c1 * pf + c3 * pc);
#pragma unroll
      for (int m = 0; m < 3; ++m) out[3 * k + c][m] = gx.d[m];
    }
}

// Rest-rest block (3 x 3) of rest vertices va, vb: out[i][j] =
// d2E/(dX_va,i dX_vb,j), the SNH energy of the tet (the formula of
// snh_state) evaluated in hyper-dual numbers over the rest positions, the
// current positions held constant.
__device__ __noinline__ void snh_rest_rest_block(const double (&x)[4][3], const double (&X)[4][3], int va, int vb,
                                                 double mu, double lam, double dt, double (&out)[3][3]) {
  H33 P[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      P[k][c] = h33c(X[k][c]);
      if (k == va) P[k][c].a[c] = 1.0;
      if (k == vb) P[k][c].b[c] = 1.0;
    }
  H33 e[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) e[k][c] = P[k + 1][c] - P[0][c];
  auto crossc = [&](const H33 (&a)[3], const H33 (&b)[3], H33 (&o)[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  H33 k0[3], k1[3], k2[3];
  crossc(e[1], e[2], k0);
  crossc(e[2], e[0], k1);
  crossc(e[0], e[1], k2);
  const H33 det = e[0][0] * k0[0] + e[0][1] * k0[1] + e[0][2] * k0[2];
  const H33 inv = h33_recip(det);
  H33 G[4][3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    G[1][j] = k0[j] * inv;
    G[2][j] = k1[j] * inv;
    G[3][j] = k2[j] * inv;
    G[0][j] = (-1.0) * (G[1][j] + G[2][j] + G[3][j]);
  }
  H33 F[3][3];  // columns f_j
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      H33 acc = x[0][c] * G[0][j];
#pragma unroll
      for (int k = 1; k < 4; ++k) acc = acc + x[k][c] * G[k][j];
      F[j][c] = acc;
    }
  H33 c0[3];
  crossc(F[1], F[2], c0);
  H33 ic = h33c(0.0);
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int c = 0; c < 3; ++c) ic = ic + F[j][c] * F[j][c];
  const H33 J = F[0][0] * c0[0] + F[0][1] * c0[1] + F[0][2] * c0[2];
  const double alpha = 1.0 + 0.75 * mu / lam;
  const H33 jm = J - h33c(alpha);
  const H33 psi = (0.5 * mu) * (ic - h33c(3.0)) - (0.5 * mu) * h33_log(ic + h33c(1.0)) + (0.5 * lam) * (jm * jm);
  const H33 E = ((dt * dt / 6.0) * det) * psi;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) out[i][j] = E.ab[i][j];
}

// Packed upper 24x24 Hessian over (x, X) of one tet: the x-x block from the
// SNH blocks, the x-X block by differentiation of the position gradient in
// X, the X-X block by hyper-dual evaluation of the energy.
__global__ void __launch_bounds__(64) snh_rest_local_hessian_kernel(const ys_snh_args a, double* out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.num_elements) return;
  double* dst = out + (uint64_t)t * 300;
  {
    SnhState st;
    snh_state(a, t, st);
    V3 u[4], v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      u[k] = mul(st.f, st.g[k]);
      v[k] = mul(st.cof, st.g[k]);
    }
#pragma unroll
    for (int ai = 0; ai < 4; ++ai)
#pragma unroll
      for (int bi = ai; bi < 4; ++bi) {
        double blk[3][3];
        hess_block(st, st.g[ai], st.g[bi], u[ai], u[bi], v[ai], v[bi], blk);
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int l = 0; l < 3; ++l)
            if (3 * ai + k <= 3 * bi + l) dst[utri<24>(3 * ai + k, 3 * bi + l)] = blk[k][l];
      }
  }
  const uint4 tv = reinterpret_cast<const uint4*>(a.tets)[t];
  const uint32_t id[4] = {tv.x, tv.y, tv.z, tv.w};
  double x[4][3], X[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const V3 p = load3(a.position, id[k]), r = load3(a.rest, id[k]);
    x[k][0] = p.x; x[k][1] = p.y; x[k][2] = p.z;
    X[k][0] = r.x; X[k][1] = r.y; X[k][2] = r.z;
  }
  const double mu = a.mu ? a.mu[t] : a.mu_value;
  const double lam = a.lam ? a.lam[t] : a.lam_value;
#pragma unroll 1
  for (int va = 0; va < 4; ++va) {
    double col[12][3];
    snh_rest_column(x, X, va, mu, lam, a.dt, col);
    for (int i = 0; i < 12; ++i)
#pragma unroll
      for (int m = 0; m < 3; ++m) dst[utri<24>(i, 12 + 3 * va + m)] = col[i][m];
  }
#pragma unroll 1
  for (int va = 0; va < 4; ++va)
#pragma unroll 1
    for (int vb = va; vb < 4; ++vb) {
      double blk[3][3];
      snh_rest_rest_block(x, X, va, vb, mu, lam, a.dt, blk);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          if (3 * va + i <= 3 * vb + j) dst[utri<24>(12 + 3 * va + i, 12 + 3 * vb + j)] = blk[i][j];
    }
}

// Derivative of the SNH position gradient s (c1 F G_k + c3 cof G_k) in a
// per-tet material parameter (which 0: mu, with dc1/dmu = 1 - 1/(IC+1) and
// dc3/dmu = -3/4 through alpha; 1: lambda, with dc3/dlam = J - 1):
// out[12 t + 3 k + c].
__global__ void snh_param_jacobian_kernel(const ys_snh_args a, int which, double* out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.num_elements) return;
  SnhState st;
  snh_state(a, t, st);
  const double ic = dot(st.f.c[0], st.f.c[0]) + dot(st.f.c[1], st.f.c[1]) + dot(st.f.c[2], st.f.c[2]);
  const double J = dot(st.f.c[0], st.cof.c[0]);
  const double d1 = which == 0 ? 1.0 - 1.0 / (ic + 1.0) : 0.0;
  const double d3 = which == 0 ? -0.75 : J - 1.0;
  double* dst = out + 12ull * t;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const V3 gk = st.s * (d1 * mul(st.f, st.g[k]) + d3 * mul(st.cof, st.g[k]));
    dst[3 * k] = gk.x;
    dst[3 * k + 1] = gk.y;
    dst[3 * k + 2] = gk.z;
  }
}

// Derivative of the inertia gradient in the vertex's mass, per argument
// (x, x_before[, v]): x - x~, -(x - x~), -dt (x - x~)  (out[3 args i + 3 a + k]).
__global__ void inertia_mass_jacobian_kernel(const ys_inertia_args a, int args, double* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.num_vertices) return;
  const double* x = a.position + 3ull * i;
  const double* xb = a.x_before + 3ull * i;
  const double h2 = a.dt * a.dt;
  const double scale[3] = {1.0, -1.0, -a.dt};
  double* dst = out + 3ull * args * i;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double d = x[k] - (xb[k] + (a.velocity ? a.velocity[3ull * i + k] * a.dt : 0.0) + a.gravity[k] * h2);
    for (int q = 0; q < args; ++q) dst[3 * q + k] = scale[q] * d;
  }
}

// Local Hessian of the inertia term 1/2 m |x - x_before - dt v - dt^2 g|^2
// over its arguments (x, x_before[, v]), packed upper: m [[I, -I, -dt I],
// [-I, I, dt I], [-dt I, dt I, dt^2 I]] (helpers.py:138-141).
__global__ void inertia_local_hessian_kernel(const double* __restrict__ mass, double mass_value, double dt,
                                             uint32_t n, int args, double* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double m = mass ? mass[i] : mass_value;
  const double c[3] = {1.0, -1.0, -dt};
  const int N = 3 * args;
  const int H = N * (N + 1) / 2;
  double* dst = out + (uint64_t)i * H;
  int q = 0;
  for (int r = 0; r < N; ++r)
    for (int col = r; col < N; ++col) dst[q++] = (r % 3 == col % 3) ? m * c[r / 3] * c[col / 3] : 0.0;
}

__global__ void inertia_kernel(const ys_inertia_args a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.num_vertices) return;
  const double m = a.mass[i];
  const double* x = a.position + 3ull * i;
  const double* xb = a.x_before + 3ull * i;
  const double h2 = a.dt * a.dt;
  double xt[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) xt[k] = xb[k] + (a.velocity ? a.velocity[3ull * i + k] * a.dt : 0.0) + a.gravity[k] * h2;
  const double d0 = x[0] - xt[0], d1 = x[1] - xt[1], d2 = x[2] - xt[2];
  if (a.energy) a.energy[i] = 0.5 * m * (d0 * d0 + d1 * d1 + d2 * d2);
  if (!a.block_records) return;  // energy only
  const uint32_t code = a.plan.codes[(uint64_t)i * a.plan.K];
  if (code < 2) return;
  double* g = a.grad_records + a.plan.grad_record[a.plan.grad_outer[i]];
  g[0] = m * d0;
  g[1] = m * d1;
  g[2] = m * d2;
  double* h = a.block_records + a.plan.record[a.plan.coord_outer[i]];
#pragma unroll
  for (int k = 0; k < 9; ++k) h[k] = (k % 4 == 0) ? m : 0.0;
}

// Per-tet energy only (line search).
__global__ void __launch_bounds__(128) snh_energy_kernel(const ys_snh_args a) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.num_elements) return;
  SnhState st;
  snh_state(a, t, st);
  a.energy[t] = st.energy;
}

}  // namespace ys

extern "C" {

int32_t ys_snh_eval(const ys_snh_args* args, void* stream) {
  YS_REQUIRE(args != nullptr, YS_ERR_INVALID, "null args");
  const ys_snh_args& a = *args;
  YS_REQUIRE(a.position.num_children >= 1 && a.position.num_children <= YS_MAX_UNION, YS_ERR_INVALID,
             "bad position union");
  YS_REQUIRE(a.rest.num_children >= 1 && a.rest.num_children <= YS_MAX_UNION, YS_ERR_INVALID, "bad rest union");
  YS_REQUIRE(((uintptr_t)a.tets & 15u) == 0, YS_ERR_INVALID, "tets must be 16-byte aligned");
  if (a.num_elements == 0) return YS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (a.block_records == nullptr && a.grad_records == nullptr) {
    YS_REQUIRE(a.energy, YS_ERR_INVALID, "energy-only evaluation needs the energy output");
    ys::snh_energy_kernel<<<ys::grid_for(a.num_elements, 128), 128, 0, s>>>(a);
    YS_CHECK_LAUNCH();
    return YS_OK;
  }
  YS_REQUIRE(a.plan.slot_stride >= 1 && a.plan.K == 4 * a.plan.slot_stride, YS_ERR_INVALID,
             "SNH needs 4 arguments (K = 4 * slot_stride)");
  if (a.projection_method >= 1) {
    YS_REQUIRE(a.work_list && a.work_count, YS_ERR_INVALID, "projection needs work_list/work_count");
    YS_CUDA_TRY(cudaMemsetAsync(a.work_count, 0, sizeof(uint32_t), s));
  }
  const unsigned grid = ys::grid_for(a.num_elements, 128);
  ys::snh_eval_kernel<<<grid, 128, 0, s>>>(a);
  YS_CHECK_LAUNCH();
  if (a.projection_method >= 1) {
    // The work count stays on the device: a grid-stride launch sized to the
    // SMs covers any count without a host round trip.
    const unsigned pgrid = std::min<unsigned>(ys::grid_for(a.num_elements, ys::kProjThreads), ys::kSMs * 16);
    const size_t smem = sizeof(double) * ys::kProjStash * ys::kProjThreads;  // above the 48 KB default
    YS_CUDA_TRY(cudaFuncSetAttribute(ys::snh_project_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ys::snh_project_kernel<<<pgrid, ys::kProjThreads, smem, s>>>(a);
    YS_CHECK_LAUNCH();
  }
  return YS_OK;
}

int32_t ys_inertia_eval(const ys_inertia_args* args, void* stream) {
  YS_REQUIRE(args != nullptr, YS_ERR_INVALID, "null args");
  if (args->num_vertices == 0) return YS_OK;
  ys::inertia_kernel<<<ys::grid_for(args->num_vertices, 256), 256, 0, (cudaStream_t)stream>>>(*args);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

}  // extern "C"

extern "C" int32_t ys_snh_local_hessians(const ys_snh_args* args, double* out, void* stream) {
  YS_REQUIRE(args != nullptr && out != nullptr, YS_ERR_INVALID, "null argument");
  const ys_snh_args& a = *args;
  if (a.num_elements == 0) return YS_OK;
  ys::snh_local_hessian_kernel<<<ys::grid_for(a.num_elements, 128), 128, 0, (cudaStream_t)stream>>>(a, out);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

extern "C" int32_t ys_inertia_local_hessians(const double* mass, double mass_value, double dt, uint32_t n,
                                             uint32_t args, double* out, void* stream) {
  YS_REQUIRE(out != nullptr, YS_ERR_INVALID, "null output");
  YS_REQUIRE(args == 2 || args == 3, YS_ERR_INVALID, "inertia has 2 or 3 arguments");
  if (n == 0) return YS_OK;
  ys::inertia_local_hessian_kernel<<<ys::grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(mass, mass_value, dt, n,
                                                                                           (int)args, out);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

extern "C" int32_t ys_snh_rest_local_hessians(const ys_snh_args* args, double* out, void* stream) {
  YS_REQUIRE(args != nullptr && out != nullptr, YS_ERR_INVALID, "null argument");
  const ys_snh_args& a = *args;
  if (a.num_elements == 0) return YS_OK;
  ys::snh_rest_local_hessian_kernel<<<ys::grid_for(a.num_elements, 64), 64, 0, (cudaStream_t)stream>>>(a, out);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

extern "C" int32_t ys_snh_param_jacobian(const ys_snh_args* args, uint32_t which, double* out, void* stream) {
  YS_REQUIRE(args != nullptr && out != nullptr, YS_ERR_INVALID, "null argument");
  YS_REQUIRE(which <= 1, YS_ERR_INVALID, "which: 0 mu, 1 lambda");
  const ys_snh_args& a = *args;
  if (a.num_elements == 0) return YS_OK;
  ys::snh_param_jacobian_kernel<<<ys::grid_for(a.num_elements, 128), 128, 0, (cudaStream_t)stream>>>(a, (int)which,
                                                                                                   out);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

extern "C" int32_t ys_inertia_mass_jacobian(const ys_inertia_args* args, uint32_t arguments, double* out,
                                            void* stream) {
  YS_REQUIRE(args != nullptr && out != nullptr, YS_ERR_INVALID, "null argument");
  YS_REQUIRE(arguments == 2 || arguments == 3, YS_ERR_INVALID, "inertia has 2 or 3 arguments");
  const ys_inertia_args& a = *args;
  if (a.num_vertices == 0) return YS_OK;
  ys::inertia_mass_jacobian_kernel<<<ys::grid_for(a.num_vertices, 256), 256, 0, (cudaStream_t)stream>>>(
      a, (int)arguments, out);
  YS_CHECK_LAUNCH();
  return YS_OK;
}
