// Vertex-tuple energies of the mixed (cloth + contact) scenes.
//
// Energy formulas follow the reference example helpers
// (examples/dropping_in_container_mixed/helpers.py):
//   point_point / point_edge / point_triangle / edge_edge (:143-199): IPC
//     log-barrier kappa (d - dHat)^2 log^2(d / dHat) on the SQUARED
//     distance d of the pair type;
//   bending (:213-234): kb (theta - theta0)^2 |x1_0 - x0_0| dt^2, theta the
//     dihedral angle 2 atan2(((n0 x n1).axis)/|axis|, n0.n1 + |n0||n1|);
//   baraff_witkin (:272-292): stretch / shear of the rest-frame deformation
//     gradient (compute_rest_shape, :240-270), area-weighted, dt^2;
// the lagged friction of examples/dropping_in_container/friction_helpers.py
// (:12-66 smoothing; point-triangle, point-edge, edge-edge and point-point),
// and a StVK membrane on the same
// rest frame (the reference ships no StVK).  Gradients and Hessians come from
// second-order forward-mode differentiation (ys_ad.cuh); the local Hessian
// is projected like the SNH one (LDL^T PSD test, then the negative modes) and
// scattered with the NoProject merge rules into pattern records.
#include <type_traits>

#include "ys_ad.cuh"
#include "ys_common.cuh"

namespace ys {

template <int A>
struct Pts {
  double p[A][3];
};

__device__ __forceinline__ void load_point(const ys_union3& u, uint32_t idx, double (&p)[3]) {
  uint32_t c = 0;
#pragma unroll
  for (int k = 1; k < YS_MAX_UNION; ++k)
    if (k < (int)u.num_children && idx >= u.prefix[k]) c = k;
  const double* s = u.child[c] + 3ull * (idx - u.prefix[c]);
  p[0] = __ldg(s);
  p[1] = __ldg(s + 1);
  p[2] = __ldg(s + 2);
}

// kappa u^2 L^2 with u = d - dHat, L = log(d / dHat), as f(d), f', f''.
template <int N>
__device__ __forceinline__ HD<N> barrier_of(const HD<N>& d, double dhat, double kappa) {
  const double x = d.v, u = x - dhat, L = log(x / dhat), ix = 1.0 / x;
  const double f = kappa * u * u * L * L;
  const double df = kappa * (2.0 * u * L * L + 2.0 * u * u * L * ix);
  const double d2f = kappa * (2.0 * L * L + 8.0 * u * L * ix + 2.0 * u * u * ix * ix - 2.0 * u * u * L * ix * ix);
  return hd_apply(d, f, df, d2f);
}

struct PointPoint {
  static constexpr int A = 2;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t, const Pts<A>& x, const Pts<A>&) {
    const HV<N> p0 = hv_var<N>(x.p[0], 0), p1 = hv_var<N>(x.p[1], 3);
    const HV<N> e = p1 - p0;
    return barrier_of(dot(e, e), a.values[0], a.values[1]);
  }
};

struct PointEdge {
  static constexpr int A = 3;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t, const Pts<A>& x, const Pts<A>&) {
    const HV<N> p0 = hv_var<N>(x.p[0], 0), p1 = hv_var<N>(x.p[1], 3), p2 = hv_var<N>(x.p[2], 6);
    const HV<N> c = cross(p1 - p0, p2 - p0);
    const HV<N> e = p2 - p1;
    return barrier_of(dot(c, c) / dot(e, e), a.values[0], a.values[1]);
  }
};

struct PointTriangle {
  static constexpr int A = 4;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t, const Pts<A>& x, const Pts<A>&) {
    const HV<N> p0 = hv_var<N>(x.p[0], 0), p1 = hv_var<N>(x.p[1], 3), p2 = hv_var<N>(x.p[2], 6),
                p3 = hv_var<N>(x.p[3], 9);
    const HV<N> b = cross(p2 - p1, p3 - p1);
    const HD<N> atb = dot(p0 - p1, b);
    return barrier_of(sq(atb) / dot(b, b), a.values[0], a.values[1]);
  }
};

struct EdgeEdge {
  static constexpr int A = 4;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t, const Pts<A>& x, const Pts<A>&) {
    const HV<N> p0 = hv_var<N>(x.p[0], 0), p1 = hv_var<N>(x.p[1], 3), p2 = hv_var<N>(x.p[2], 6),
                p3 = hv_var<N>(x.p[3], 9);
    const HV<N> b = cross(p1 - p0, p3 - p2);
    const HD<N> atb = dot(p2 - p0, b);
    return barrier_of(sq(atb) / dot(b, b), a.values[0], a.values[1]);
  }
};

// Plain-double dihedral angle of the same formula (rest state).
__device__ __forceinline__ double dihedral(const double (&q0)[3], const double (&q1)[3], const double (&q2)[3],
                                          const double (&q3)[3]) {
  auto sub = [](const double (&u)[3], const double (&v)[3], double (&o)[3]) {
    o[0] = u[0] - v[0]; o[1] = u[1] - v[1]; o[2] = u[2] - v[2];
  };
  auto crs = [](const double (&u)[3], const double (&v)[3], double (&o)[3]) {
    o[0] = u[1] * v[2] - u[2] * v[1]; o[1] = u[2] * v[0] - u[0] * v[2]; o[2] = u[0] * v[1] - u[1] * v[0];
  };
  auto dt = [](const double (&u)[3], const double (&v)[3]) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
  double a[3], b[3], n0[3], n1[3], axis[3], c[3];
  sub(q0, q2, a); sub(q1, q2, b); crs(a, b, n0);
  sub(q1, q3, a); sub(q0, q3, b); crs(a, b, n1);
  sub(q1, q0, axis);
  crs(n0, n1, c);
  const double num = dt(c, axis) / sqrt(dt(axis, axis));
  const double den = dt(n0, n1) + sqrt(dt(n0, n0)) * sqrt(dt(n1, n1));
  return 2.0 * atan2(num, den);
}

struct Bending {
  static constexpr int A = 4;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t, const Pts<A>& x, const Pts<A>& r) {
    const HV<N> q0 = hv_var<N>(x.p[0], 0), q1 = hv_var<N>(x.p[1], 3), q2 = hv_var<N>(x.p[2], 6),
                q3 = hv_var<N>(x.p[3], 9);
    const HV<N> n0 = cross(q0 - q2, q1 - q2);
    const HV<N> n1 = cross(q1 - q3, q0 - q3);
    const HV<N> axis = q1 - q0;
    const HD<N> num = dot(cross(n0, n1), axis) / norm(axis);
    const HD<N> den = dot(n0, n1) + norm(n0) * norm(n1);
    const HD<N> theta = 2.0 * hd_atan2(num, den);
    const double theta0 = dihedral(r.p[0], r.p[1], r.p[2], r.p[3]);
    const double e0 = r.p[1][0] - r.p[0][0], e1 = r.p[1][1] - r.p[0][1], e2 = r.p[1][2] - r.p[0][2];
    const double len = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
    const double dt = a.values[1];
    return (a.values[0] * len * dt * dt) * sq(theta - theta0);
  }
};

// Rest-frame inverse shape matrix of a triangle (compute_rest_shape,
// helpers.py:240-270: rotate the normal onto +y, keep (x, z)) and the rest
// area |v01 x v02| / 2.
__device__ __forceinline__ void rest_frame(const Pts<3>& r, double (&minv)[2][2], double& area) {
  double v01[3], v02[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) { v01[k] = r.p[1][k] - r.p[0][k]; v02[k] = r.p[2][k] - r.p[0][k]; }
  double n[3] = {v01[1] * v02[2] - v01[2] * v02[1], v01[2] * v02[0] - v01[0] * v02[2],
                 v01[0] * v02[1] - v01[1] * v02[0]};
  const double nl = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  area = 0.5 * nl;
  n[0] /= nl; n[1] /= nl; n[2] /= nl;
  // vec = n x (0, 1, 0), cos = n.(0, 1, 0)
  const double v[3] = {-n[2], 0.0, n[0]};
  const double c = n[1];
  const double vx[3][3] = {{0.0, -v[2], v[1]}, {v[2], 0.0, -v[0]}, {-v[1], v[0], 0.0}};
  double rot[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) s += vx[i][k] * vx[k][j];
      rot[i][j] = (i == j ? 1.0 : 0.0) + vx[i][j] + s / (1.0 + c);
    }
  double uv[3][2];
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    uv[p][0] = rot[0][0] * r.p[p][0] + rot[0][1] * r.p[p][1] + rot[0][2] * r.p[p][2];
    uv[p][1] = rot[2][0] * r.p[p][0] + rot[2][1] * r.p[p][1] + rot[2][2] * r.p[p][2];
  }
  const double m00 = uv[1][0] - uv[0][0], m01 = uv[2][0] - uv[0][0];
  const double m10 = uv[1][1] - uv[0][1], m11 = uv[2][1] - uv[0][1];
  const double idet = 1.0 / (m00 * m11 - m01 * m10);
  minv[0][0] = m11 * idet;
  minv[0][1] = -m01 * idet;
  minv[1][0] = -m10 * idet;
  minv[1][1] = m00 * idet;
}

// Columns of F = [x1 - x0, x2 - x0] M^-1 (3x2).
template <int N>
__device__ __forceinline__ void membrane_f(const Pts<3>& x, const double (&minv)[2][2], HV<N>& f0, HV<N>& f1) {
  const HV<N> p0 = hv_var<N>(x.p[0], 0), p1 = hv_var<N>(x.p[1], 3), p2 = hv_var<N>(x.p[2], 6);
  const HV<N> x10 = p1 - p0, x20 = p2 - p0;
  f0 = minv[0][0] * x10 + minv[1][0] * x20;
  f1 = minv[0][1] * x10 + minv[1][1] * x20;
}

struct BaraffWitkin {
  static constexpr int A = 3;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t, const Pts<A>& x, const Pts<A>& r) {
    double minv[2][2], area;
    rest_frame(r, minv, area);
    HV<N> f0, f1;
    membrane_f<N>(x, minv, f0, f1);
    const HD<N> shear = sq(dot(f0, f1));
    const HD<N> i5u = norm(f0), i5v = norm(f1);
    const double uc = i5u.v < 1.0 ? 0.01 : 1.0, vc = i5v.v < 1.0 ? 0.01 : 1.0;
    const HD<N> stretch = uc * sq(i5u - 1.0) + vc * sq(i5v - 1.0);
    const double dt = a.values[3];
    const double w = a.values[2] * area * dt * dt;  // thickness * area * dt^2
    return w * (a.values[0] * stretch + a.values[1] * shear);
  }
};

// psi = mu tr(E^2) + lam/2 tr(E)^2, E = (F^T F - I) / 2, on the same rest frame.
struct StvkMembrane {
  static constexpr int A = 3;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t, const Pts<A>& x, const Pts<A>& r) {
    double minv[2][2], area;
    rest_frame(r, minv, area);
    HV<N> f0, f1;
    membrane_f<N>(x, minv, f0, f1);
    const HD<N> e00 = 0.5 * (dot(f0, f0) - 1.0), e11 = 0.5 * (dot(f1, f1) - 1.0), e01 = 0.5 * dot(f0, f1);
    const HD<N> tr = e00 + e11;
    const HD<N> psi = a.values[0] * (sq(e00) + sq(e11) + 2.0 * sq(e01)) + (0.5 * a.values[1]) * sq(tr);
    const double dt = a.values[3];
    return (a.values[2] * area * dt * dt) * psi;
  }
};

// ---- the cloth energies over positions and rest positions ------------------
// The same formulas as Bending, BaraffWitkin and StvkMembrane (and their rest
// quantities rest_frame and dihedral), written over H33 numbers so that both
// the positions and the rest positions are inputs: one evaluation gives the
// 3x3 block of d2E between two of the element's 2A vertices (positions 0 ..
// A-1, rest positions A .. 2A-1).
struct HV33 {
  H33 x, y, z;
};
__device__ __forceinline__ HV33 operator-(const HV33& u, const HV33& v) { return {u.x - v.x, u.y - v.y, u.z - v.z}; }
__device__ __forceinline__ HV33 operator+(const HV33& u, const HV33& v) { return {u.x + v.x, u.y + v.y, u.z + v.z}; }
__device__ __forceinline__ HV33 scale(const H33& s, const HV33& v) { return {s * v.x, s * v.y, s * v.z}; }
__device__ __forceinline__ H33 dot(const HV33& u, const HV33& v) { return u.x * v.x + u.y * v.y + u.z * v.z; }
__device__ __forceinline__ HV33 cross(const HV33& u, const HV33& v) {
  return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
__device__ __forceinline__ H33 norm(const HV33& u) { return h33_sqrt(dot(u, u)); }

__device__ __noinline__ H33 dihedral33(const HV33& q0, const HV33& q1, const HV33& q2, const HV33& q3) {
  const HV33 n0 = cross(q0 - q2, q1 - q2);
  const HV33 n1 = cross(q1 - q3, q0 - q3);
  const HV33 axis = q1 - q0;
  const H33 num = dot(cross(n0, n1), axis) / norm(axis);
  const H33 den = dot(n0, n1) + norm(n0) * norm(n1);
  return 2.0 * h33_atan2(num, den);
}

// rest_frame: rotate the rest normal onto +y, keep (x, z); M^-1 and the area
__device__ __noinline__ void rest_frame33(const HV33 (&r)[3], H33 (&minv)[2][2], H33& area) {
  const HV33 nn = cross(r[1] - r[0], r[2] - r[0]);
  const H33 nl = norm(nn);
  area = 0.5 * nl;
  const HV33 n = scale(h33_recip(nl), nn);
  // vec = (-n_z, 0, n_x), cos = n_y: rows 0 and 2 of I + [vec]x + [vec]x^2 / (1 + cos)
  const H33 ic = h33_recip(n.y + 1.0);
  const H33 nx2 = n.x * n.x, nz2 = n.z * n.z, nxz = n.x * n.z;
  // [vec]x = [[0, -n_x, 0], [n_x, 0, n_z], [0, -n_z, 0]];
  // [vec]x^2 = [[-n_x^2, 0, -n_x n_z], [0, -n_x^2 - n_z^2, 0], [-n_x n_z, 0, -n_z^2]]
  const H33 r00 = (-1.0 * nx2) * ic + 1.0, r01 = -1.0 * n.x, r02 = (-1.0 * nxz) * ic;
  const H33 r20 = (-1.0 * nxz) * ic, r21 = -1.0 * n.z, r22 = (-1.0 * nz2) * ic + 1.0;
  H33 uv[3][2];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    uv[q][0] = r00 * r[q].x + r01 * r[q].y + r02 * r[q].z;
    uv[q][1] = r20 * r[q].x + r21 * r[q].y + r22 * r[q].z;
  }
  const H33 m00 = uv[1][0] - uv[0][0], m01 = uv[2][0] - uv[0][0];
  const H33 m10 = uv[1][1] - uv[0][1], m11 = uv[2][1] - uv[0][1];
  const H33 idet = h33_recip(m00 * m11 - m01 * m10);
  minv[0][0] = m11 * idet;
  minv[0][1] = (-1.0 * m01) * idet;
  minv[1][0] = (-1.0 * m10) * idet;
  minv[1][1] = m00 * idet;
}

__device__ __forceinline__ void membrane_f33(const HV33 (&x)[3], const H33 (&minv)[2][2], HV33& f0, HV33& f1) {
  const HV33 x10 = x[1] - x[0], x20 = x[2] - x[0];
  f0 = scale(minv[0][0], x10) + scale(minv[1][0], x20);
  f1 = scale(minv[0][1], x10) + scale(minv[1][1], x20);
}

__device__ __noinline__ H33 cloth_energy33(const ys_energy_args& a, const HV33 (&q)[4], const HV33 (&p)[4]) {
  if (a.kind == YS_ENERGY_BENDING) {
    const H33 theta = dihedral33(q[0], q[1], q[2], q[3]);
    const H33 theta0 = dihedral33(p[0], p[1], p[2], p[3]);
    const H33 d = theta - theta0;
    const double dt = a.values[1];
    return (a.values[0] * dt * dt) * (norm(p[1] - p[0]) * (d * d));
  }
  const HV33 qx[3] = {q[0], q[1], q[2]}, px[3] = {p[0], p[1], p[2]};
  H33 minv[2][2], area;
  rest_frame33(px, minv, area);
  HV33 f0, f1;
  membrane_f33(qx, minv, f0, f1);
  const double dt = a.values[3];
  if (a.kind == YS_ENERGY_BARAFF_WITKIN) {
    const H33 sh = dot(f0, f1);
    const H33 i5u = norm(f0), i5v = norm(f1);
    const double uc = i5u.v < 1.0 ? 0.01 : 1.0, vc = i5v.v < 1.0 ? 0.01 : 1.0;
    const H33 du = i5u - 1.0, dv = i5v - 1.0;
    const H33 stretch = uc * (du * du) + vc * (dv * dv);
    return (a.values[2] * dt * dt) * (area * (a.values[0] * stretch + a.values[1] * (sh * sh)));
  }
  const H33 e00 = 0.5 * (dot(f0, f0) - 1.0), e11 = 0.5 * (dot(f1, f1) - 1.0), e01 = 0.5 * dot(f0, f1);
  const H33 tr = e00 + e11;
  const H33 psi = a.values[0] * (e00 * e00 + e11 * e11 + 2.0 * (e01 * e01)) + (0.5 * a.values[1]) * (tr * tr);
  return (a.values[2] * dt * dt) * (area * psi);
}

// Unprojected local Hessian over (positions, rest positions) of every
// element, packed upper (6A)x(6A): one H33 evaluation a vertex pair.
template <int A>
__global__ void __launch_bounds__(64) rest_local_hessian_kernel(const ys_energy_args a, double* out) {
  constexpr int M = 2 * A, N = 3 * M;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.num_elements) return;
  double v[M][3];
#pragma unroll
  for (int k = 0; k < A; ++k) {
    const uint32_t id = a.conn[(uint64_t)t * A + k];
    load_point(a.position, id, v[k]);
    load_point(a.rest, id, v[A + k]);
  }
  double* dst = out + (uint64_t)t * (N * (N + 1) / 2);
#pragma unroll 1
  for (int va = 0; va < M; ++va)
#pragma unroll 1
    for (int vb = va; vb < M; ++vb) {
      HV33 w[M];
#pragma unroll
      for (int k = 0; k < M; ++k) {
        H33* c[3] = {&w[k].x, &w[k].y, &w[k].z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          *c[d] = h33c(v[k][d]);
          if (k == va) c[d]->a[d] = 1.0;
          if (k == vb) c[d]->b[d] = 1.0;
        }
      }
      HV33 q[4], p[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        q[k] = w[k < A ? k : 0];
        p[k] = w[k < A ? A + k : A];
      }
      const H33 e = cloth_energy33(a, q, p);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          if (3 * va + i <= 3 * vb + j) dst[utri<N>(3 * va + i, 3 * vb + j)] = e.ab[i][j];
    }
}

// Lagged friction (friction_helpers.py:12-66): with the lagged tangent
// basis (q[2..4], q[5..7]) and lambda_last_h (q[8]), phi of the tangential
// relative displacement y = |(t0.rel, t1.rel)| (smoothed below sqrt(fDhat) dt)
// times frictionRate lambda.  `rest` holds the positions at the start of the
// step, so d(x - x_old)/dx = I.
template <int N>
__device__ __forceinline__ HD<N> lagged_friction(const ys_energy_args& a, const double* q, const HV<N>& rel) {
  const HD<N> u0 = q[2] * rel.x + q[3] * rel.y + q[4] * rel.z;
  const HD<N> u1 = q[5] * rel.x + q[6] * rel.y + q[7] * rel.z;
  const HD<N> y2 = sq(u0) + sq(u1);
  const double fdhat = a.values[0], dt = a.values[1], rate = a.values[2];
  const double eps = sqrt(fdhat) * dt, fric_dhat = fdhat * dt * dt;
  const HD<N> y = hd_sqrt(y2 + 1e-16);
  HD<N> phi;
  if (y2.v > fric_dhat) phi = y;
  else phi = ((1.0 / eps) * y2 + eps / 3.0) - (1.0 / (3.0 * eps * eps)) * (y2 * y);
  return (rate * q[8]) * phi;
}

template <int N, int A>
__device__ __forceinline__ void step_inputs(const Pts<A>& x, const Pts<A>& r, HV<N> (&dx)[A]) {
#pragma unroll
  for (int k = 0; k < A; ++k) {
    const double d[3] = {x.p[k][0] - r.p[k][0], x.p[k][1] - r.p[k][1], x.p[k][2] - r.p[k][2]};
    dx[k] = hv_var<N>(d, 3 * k);
  }
}

// Point-triangle (:73-182): lagged (beta1, beta2) of the closest point.
struct FrictionPT {
  static constexpr int A = 4;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t t, const Pts<A>& x, const Pts<A>& r) {
    const double* q = a.params + (uint64_t)t * a.param_stride;
    HV<N> dx[A];
    step_inputs<N>(x, r, dx);
    return lagged_friction<N>(a, q, dx[0] - (dx[1] + q[0] * (dx[2] - dx[1]) + q[1] * (dx[3] - dx[1])));
  }
};

// Point-edge (:188-276): lagged eta of the closest point on the edge.
struct FrictionPE {
  static constexpr int A = 3;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t t, const Pts<A>& x, const Pts<A>& r) {
    const double* q = a.params + (uint64_t)t * a.param_stride;
    HV<N> dx[A];
    step_inputs<N>(x, r, dx);
    return lagged_friction<N>(a, q, dx[0] - (dx[1] + q[0] * (dx[2] - dx[1])));
  }
};

// Edge-edge (:283-405): lagged (gamma1, gamma2) of the closest points.
struct FrictionEE {
  static constexpr int A = 4;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t t, const Pts<A>& x, const Pts<A>& r) {
    const double* q = a.params + (uint64_t)t * a.param_stride;
    HV<N> dx[A];
    step_inputs<N>(x, r, dx);
    return lagged_friction<N>(a, q, ((dx[0] + q[0] * (dx[1] - dx[0])) - dx[2]) - q[1] * (dx[3] - dx[2]));
  }
};

// Point-point (:411-500).
struct FrictionPP {
  static constexpr int A = 2;
  template <int N>
  __device__ static HD<N> eval(const ys_energy_args& a, uint32_t t, const Pts<A>& x, const Pts<A>& r) {
    const double* q = a.params + (uint64_t)t * a.param_stride;
    HV<N> dx[A];
    step_inputs<N>(x, r, dx);
    return lagged_friction<N>(a, q, dx[0] - dx[1]);
  }
};

// ---- scatter into records --------------------------------------------------

template <int A>
__device__ __forceinline__ void load_arg_codes(const ys_term_plan& p, uint32_t t, uint32_t (&code)[A]) {
#pragma unroll
  for (int k = 0; k < A; ++k) code[k] = p.codes[(uint64_t)t * p.K + (uint64_t)k * p.slot_stride];
}

// Records of the (projected) local Hessian h (packed upper, N = 3A): merged
// per distinct target argument, blocks transposed when the row DoF exceeds
// the column DoF (hessianKernelNoProject.pyx:94-264), in the slot order of
// the coordinates (first occurrence i <= j).
template <int A>
__device__ __forceinline__ void write_records(const uint32_t (&code)[A], uint32_t occ0, const uint32_t* record,
                                              double* out, const double (&h)[3 * A * (3 * A + 1) / 2]) {
  constexpr int N = 3 * A;
  int group[A], first[A];
  int nfirst = 0;
#pragma unroll
  for (int k = 0; k < A; ++k) {
    group[k] = -1;
    if (code[k] < 2) continue;
    int g = -1;
    for (int q = 0; q < nfirst; ++q)
      if (code[first[q]] == code[k]) g = q;
    if (g < 0) { first[nfirst] = k; g = nfirst++; }
    group[k] = g;
  }
  uint32_t occ = occ0;
  for (int gi = 0; gi < nfirst; ++gi)
    for (int gj = gi; gj < nfirst; ++gj) {
      double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
      for (int ai = 0; ai < A; ++ai) {
        if (group[ai] != gi) continue;
#pragma unroll
        for (int bi = 0; bi < A; ++bi) {
          if (group[bi] != gj) continue;
#pragma unroll
          for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int l = 0; l < 3; ++l) acc[k][l] += h[utri<N>(3 * ai + k, 3 * bi + l)];
        }
      }
      double* dst = out + record[occ++];
      const bool upper = code[first[gi]] < code[first[gj]];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) dst[3 * k + l] = upper ? acc[k][l] : acc[l][k];
    }
}

// Threads per CTA of the energy kernels (the projection stash is per thread).
constexpr int kEnergyThreads = 32;

// Energy, gradient records, projection and Hessian records of one element
// from its HD<3A> energy (shared by the vertex-tuple and affine kernels).
template <int A, class Args>
__device__ __forceinline__ void finish_element(const Args& a, uint32_t t, const HD<3 * A>& e, double* stash) {
  constexpr int N = 3 * A;
  if (a.energy) a.energy[t] = e.v;
  uint32_t code[A];
  load_arg_codes<A>(a.plan, t, code);
  uint32_t q = a.plan.grad_outer[t];
#pragma unroll
  for (int k = 0; k < A; ++k) {
    if (code[k] < 2) continue;
    double* dst = a.grad_records + a.plan.grad_record[q++];
    dst[0] = e.g[3 * k];
    dst[1] = e.g[3 * k + 1];
    dst[2] = e.g[3 * k + 2];
  }
  double h[HD<N>::H];
#pragma unroll
  for (int i = 0; i < HD<N>::H; ++i) h[i] = e.h[i];
  if (a.projection_method >= 1) {
    double s[HD<N>::H];  // packed lower copy for the PSD test
#pragma unroll
    for (int rr = 0; rr < N; ++rr)
#pragma unroll
      for (int c = 0; c <= rr; ++c) s[tri(rr, c)] = h[utri<N>(c, rr)];
    if (!psd_test_packed<N>(s)) project_negative_modes<N>(h, a.projection_method, stash, blockDim.x);
  }
  write_records<A>(code, a.plan.coord_outer[t], a.plan.record, a.block_records, h);
}

template <class E>
__global__ void __launch_bounds__(kEnergyThreads) energy_kernel(const ys_energy_args a) {
  constexpr int A = E::A, N = 3 * A;
  extern __shared__ double energy_stash[];
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.num_elements) return;
  Pts<A> x, r;
#pragma unroll
  for (int k = 0; k < A; ++k) {
    const uint32_t id = a.conn[(uint64_t)t * A + k];
    load_point(a.position, id, x.p[k]);
    if (a.rest.num_children) load_point(a.rest, id, r.p[k]);
    else r.p[k][0] = r.p[k][1] = r.p[k][2] = 0.0;
  }
  const HD<N> e = E::template eval<N>(a, t, x, r);
  finish_element<A>(a, t, e, energy_stash + threadIdx.x);
}

// Per-element energy only (line search): the same formulas on HD<0> numbers.
template <class E>
__global__ void __launch_bounds__(128) energy_value_kernel(const ys_energy_args a) {
  constexpr int A = E::A;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.num_elements) return;
  Pts<A> x, r;
#pragma unroll
  for (int k = 0; k < A; ++k) {
    const uint32_t id = a.conn[(uint64_t)t * A + k];
    load_point(a.position, id, x.p[k]);
    if (a.rest.num_children) load_point(a.rest, id, r.p[k]);
    else r.p[k][0] = r.p[k][1] = r.p[k][2] = 0.0;
  }
  a.energy[t] = E::template eval<0>(a, t, x, r).v;
}

// Unprojected local Hessian of every element with respect to its position
// arguments, packed upper (HD<3A>::H doubles an element): the input of the
// rectangular second-order Jacobian, whose reference kernel does not project
// (PKG/kernel/Jacobian/secondOrderJacobianKernelNoProject.pyx).
template <class E>
__global__ void __launch_bounds__(kEnergyThreads) local_hessian_kernel(const ys_energy_args a, double* out) {
  constexpr int A = E::A, N = 3 * A;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.num_elements) return;
  Pts<A> x, r;
#pragma unroll
  for (int k = 0; k < A; ++k) {
    const uint32_t id = a.conn[(uint64_t)t * A + k];
    load_point(a.position, id, x.p[k]);
    if (a.rest.num_children) load_point(a.rest, id, r.p[k]);
    else r.p[k][0] = r.p[k][1] = r.p[k][2] = 0.0;
  }
  const HD<N> e = E::template eval<N>(a, t, x, r);
  double* dst = out + (uint64_t)t * HD<N>::H;
#pragma unroll
  for (int i = 0; i < HD<N>::H; ++i) dst[i] = e.h[i];
}

template <class E>
static int32_t launch_local_hessian(const ys_energy_args& a, double* out, cudaStream_t s) {
  YS_REQUIRE(a.arity == (uint32_t)E::A, YS_ERR_INVALID, "arity does not match the energy kind");
  local_hessian_kernel<E><<<grid_for(a.num_elements, kEnergyThreads), kEnergyThreads, 0, s>>>(a, out);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

template <class E>
static int32_t launch_energy_value(const ys_energy_args& a, cudaStream_t s) {
  YS_REQUIRE(a.arity == (uint32_t)E::A, YS_ERR_INVALID, "arity does not match the energy kind");
  energy_value_kernel<E><<<grid_for(a.num_elements, 128), 128, 0, s>>>(a);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

template <class E>
static int32_t launch_energy(const ys_energy_args& a, cudaStream_t s) {
  YS_REQUIRE(a.arity == (uint32_t)E::A, YS_ERR_INVALID, "arity does not match the energy kind");
  constexpr int N = 3 * E::A;
  const size_t smem = sizeof(double) * project_stash_doubles<N>() * kEnergyThreads;
  YS_CUDA_TRY(cudaFuncSetAttribute(energy_kernel<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  energy_kernel<E><<<grid_for(a.num_elements, kEnergyThreads), kEnergyThreads, smem, s>>>(a);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

// ---- affine (ABD) bodies -------------------------------------------------
// Inputs of an element: the rows of its body's A (inputs 3r + c = A[r][c],
// row-major like the reference attribute) and t (inputs 9 + r).

struct AffineBody {
  double a[3][3];
  double t[3];
};

// x_r = A[r] . xbar + t_r as an HD number: linear in the inputs, so its
// gradient is (xbar at 3r .. 3r+2, 1 at 9 + r) and its Hessian zero.
template <int N>
__device__ __forceinline__ HD<N> affine_coord(const AffineBody& b, const double (&xb)[3], int r) {
  HD<N> x = hd_const<N>(b.a[r][0] * xb[0] + b.a[r][1] * xb[1] + b.a[r][2] * xb[2] + b.t[r]);
  if constexpr (N >= 12) {
#pragma unroll
    for (int c = 0; c < 3; ++c) x.g[3 * r + c] = xb[c];
    x.g[9 + r] = 1.0;
  }
  return x;
}

__device__ __forceinline__ void load_rest3(const double* p, uint64_t i, double (&v)[3]) {
  v[0] = __ldg(p + 3 * i);
  v[1] = __ldg(p + 3 * i + 1);
  v[2] = __ldg(p + 3 * i + 2);
}

// stiffness * 1/2 sum_rows |row(A^T A - I)|^2 (helpers.py:201-211).
struct AffineOrthogonality {
  static constexpr int A = 3;
  template <int N>
  __device__ static HD<N> eval(const ys_affine_args& a, uint32_t, const AffineBody& b) {
    HD<N> m[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) m[r][c] = hd_var<N>(b.a[r][c], 3 * r + c);
    HD<N> acc = hd_const<N>(0.0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        // (A^T A)_ij = sum_k A_ki A_kj
        HD<N> d = m[0][i] * m[0][j] + m[1][i] * m[1][j] + m[2][i] * m[2][j];
        if (i == j) d = d - 1.0;
        acc = acc + sq(d);
      }
    return (0.5 * a.stiffness) * acc;
  }
};

// 1/2 m |A xbar + t - x~|^2, x~ = x_before + v dt + gravity dt^2.
struct AffineInertia {
  static constexpr int A = 4;
  template <int N>
  __device__ static HD<N> eval(const ys_affine_args& a, uint32_t e, const AffineBody& b) {
    double xb[3], x0[3];
    load_rest3(a.rest, e, xb);
    load_rest3(a.x_before, e, x0);
    const double h2 = a.dt * a.dt;
    HD<N> acc = hd_const<N>(0.0);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const double v = a.velocity ? __ldg(a.velocity + 3ull * e + r) : 0.0;
      const double xt = x0[r] + v * a.dt + a.gravity[r] * h2;
      acc = acc + sq(affine_coord<N>(b, xb, r) - xt);
    }
    return (0.5 * __ldg(a.mass + e)) * acc;
  }
};

// Stable Neo-Hookean (helpers.py:102-127) of a tetrahedron of one body whose
// vertices sit at x_k = A xbar_k + t: F rows x_k - x_0 (the edge matrix), TB
// rows xbar_k - xbar_0, IB = (TB^T)^-1, vol = det(TB^T) / 6, FI = F^T IB.
// The energy's argument is the gathered vertex positions, a linear function
// of the body's A and t, so the reference projects the 12x12 Hessian with
// respect to those positions and maps it to the body coordinates
// (PKG/differentiator/differentiator.pyx:795-799): eval<N> gives the energy
// over the 12 position coordinates (N = 12, input 3k + r = x_k[r]) or its
// value (N = 0); the affine kernel projects and maps (affine_positions_to_body).
struct AffineSnh {
  static constexpr int A = 4;
  static constexpr bool kInnerPositions = true;
  // body-frame rest positions xbar, rest edges, IB and det(TB^T) of element e
  __device__ static void rest_frame(const ys_affine_args& a, uint32_t e, double (&ed)[3][3], double (&ib)[3][3],
                                    double& det, double (&xb)[4][3]) {
    const uint4 tv = reinterpret_cast<const uint4*>(a.tets)[e];
    load_rest3(a.rest, tv.x, xb[0]);
    load_rest3(a.rest, tv.y, xb[1]);
    load_rest3(a.rest, tv.z, xb[2]);
    load_rest3(a.rest, tv.w, xb[3]);
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int c = 0; c < 3; ++c) ed[m][c] = xb[m + 1][c] - xb[0][c];
    // (TB^T)^-1 rows: (e1 x e2, e2 x e0, e0 x e1) / det
    const double k0[3] = {ed[1][1] * ed[2][2] - ed[1][2] * ed[2][1], ed[1][2] * ed[2][0] - ed[1][0] * ed[2][2],
                          ed[1][0] * ed[2][1] - ed[1][1] * ed[2][0]};
    const double k1[3] = {ed[2][1] * ed[0][2] - ed[2][2] * ed[0][1], ed[2][2] * ed[0][0] - ed[2][0] * ed[0][2],
                          ed[2][0] * ed[0][1] - ed[2][1] * ed[0][0]};
    const double k2[3] = {ed[0][1] * ed[1][2] - ed[0][2] * ed[1][1], ed[0][2] * ed[1][0] - ed[0][0] * ed[1][2],
                          ed[0][0] * ed[1][1] - ed[0][1] * ed[1][0]};
    det = ed[0][0] * k0[0] + ed[0][1] * k0[1] + ed[0][2] * k0[2];
    const double inv = 1.0 / det;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ib[0][c] = k0[c] * inv;
      ib[1][c] = k1[c] * inv;
      ib[2][c] = k2[c] * inv;
    }
  }

  template <int N>
  __device__ static HD<N> eval(const ys_affine_args& a, uint32_t e, const AffineBody& b) {
    double ed[3][3], ib[3][3], det, xb[4][3];
    rest_frame(a, e, ed, ib, det, xb);
    HD<N> x[4][3];  // positions A xbar_k + t as the inputs
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int r = 0; r < 3; ++r)
        x[k][r] = hd_var<N>(b.a[r][0] * xb[k][0] + b.a[r][1] * xb[k][1] + b.a[r][2] * xb[k][2] + b.t[r], 3 * k + r);
    HD<N> fi[3][3];  // FI = F^T IB, F[m][i] = x_{m+1}[i] - x_0[i]
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        fi[i][j] = ib[0][j] * (x[1][i] - x[0][i]) + ib[1][j] * (x[2][i] - x[0][i]) + ib[2][j] * (x[3][i] - x[0][i]);
    HD<N> ic = hd_const<N>(0.0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) ic = ic + sq(fi[i][j]);
    const HD<N> J = fi[0][0] * (fi[1][1] * fi[2][2] - fi[1][2] * fi[2][1]) -
                    fi[0][1] * (fi[1][0] * fi[2][2] - fi[1][2] * fi[2][0]) +
                    fi[0][2] * (fi[1][0] * fi[2][1] - fi[1][1] * fi[2][0]);
    const double mu = a.mu ? __ldg(a.mu + e) : a.mu_value;
    const double lam = a.lam ? __ldg(a.lam + e) : a.lam_value;
    const double alpha = 1.0 + 0.75 * mu / lam;
    const HD<N> psi = (0.5 * mu) * (ic - 3.0) - (0.5 * mu) * hd_log(ic + 1.0) + (0.5 * lam) * sq(J - alpha);
    return (det / 6.0 * a.dt * a.dt) * psi;
  }
};

// The position-space energy of a body tetrahedron mapped to its body
// coordinates (A row-major at 0..8, t at 9..11): x_k[r] = sum_c A[r][c]
// xbar_k[c] + t[r], so J = dx/dq holds xbar_k at (3k + r, 3r .. 3r + 2) and 1
// at (3k + r, 9 + r); g_q = J^T g_x, H_q = J^T H_x J.
__device__ __forceinline__ double affine_jac(const double (&xb)[4][3], int k, int r, int j) {
  if (j < 9) return (j / 3 == r) ? xb[k][j % 3] : 0.0;
  return (j - 9 == r) ? 1.0 : 0.0;
}

__device__ __forceinline__ void affine_positions_to_body(const HD<12>& ex, const double (&xb)[4][3], HD<12>& q) {
  q.v = ex.v;
#pragma unroll
  for (int j = 0; j < 12; ++j) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int r = 0; r < 3; ++r) acc += affine_jac(xb, k, r, j) * ex.g[3 * k + r];
    q.g[j] = acc;
  }
#pragma unroll
  for (int i = 0; i < 12; ++i)
#pragma unroll
    for (int j = i; j < 12; ++j) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const double ji = affine_jac(xb, k, r, i);
          if (ji == 0.0) continue;
#pragma unroll
          for (int k2 = 0; k2 < 4; ++k2)
#pragma unroll
            for (int r2 = 0; r2 < 3; ++r2) acc += ji * ex.h[sym<12>(3 * k + r, 3 * k2 + r2)] * affine_jac(xb, k2, r2, j);
        }
      q.h[utri<12>(i, j)] = acc;
    }
}

// Body of element e; false (element skipped) when an index is out of range.
__device__ __forceinline__ bool load_affine_body(const ys_affine_args& a, uint32_t e, AffineBody& b) {
  const uint32_t id = a.body ? __ldg(a.body + e) : e;
  if (id >= a.num_bodies) return false;
  if (a.tets) {
    const uint4 tv = reinterpret_cast<const uint4*>(a.tets)[e];
    if (tv.x >= a.num_rest || tv.y >= a.num_rest || tv.z >= a.num_rest || tv.w >= a.num_rest) return false;
  }
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) b.a[r][c] = __ldg(a.affine + 9ull * id + 3 * r + c);
#pragma unroll
  for (int r = 0; r < 3; ++r) b.t[r] = a.translation ? __ldg(a.translation + 3ull * id + r) : 0.0;
  return true;
}

template <class E, class = void>
struct InnerPositions : std::false_type {};
template <class E>
struct InnerPositions<E, std::void_t<decltype(E::kInnerPositions)>> : std::bool_constant<E::kInnerPositions> {};

template <class E>
__global__ void __launch_bounds__(kEnergyThreads) affine_kernel(const ys_affine_args a) {
  constexpr int A = E::A, N = 3 * A;
  extern __shared__ double energy_stash[];
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.num_elements) return;
  AffineBody b;
  if (!load_affine_body(a, e, b)) return;
  if constexpr (InnerPositions<E>::value) {
    // project the Hessian in the vertex positions (12x12), then map it to
    // the body coordinates
    HD<12> ex = E::template eval<12>(a, e, b);
    if (a.projection_method >= 1) {
      double s[HD<12>::H];
#pragma unroll
      for (int rr = 0; rr < 12; ++rr)
#pragma unroll
        for (int c = 0; c <= rr; ++c) s[tri(rr, c)] = ex.h[utri<12>(c, rr)];
      if (!psd_test_packed<12>(s))
        project_negative_modes<12>(ex.h, a.projection_method, energy_stash + threadIdx.x, blockDim.x);
    }
    double ed[3][3], ib[3][3], det, xb[4][3];
    E::rest_frame(a, e, ed, ib, det, xb);
    HD<N> en;
    affine_positions_to_body(ex, xb, en);
    ys_affine_args plain = a;
    plain.projection_method = 0;  // projected already
    finish_element<A>(plain, e, en, energy_stash + threadIdx.x);
  } else {
    const HD<N> en = E::template eval<N>(a, e, b);
    finish_element<A>(a, e, en, energy_stash + threadIdx.x);
  }
}

template <class E>
__global__ void __launch_bounds__(128) affine_value_kernel(const ys_affine_args a) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.num_elements) return;
  AffineBody b;
  if (!load_affine_body(a, e, b)) return;
  a.energy[e] = E::template eval<0>(a, e, b).v;
}

template <class E>
static int32_t launch_affine(const ys_affine_args& a, cudaStream_t s) {
  if (a.block_records == nullptr && a.grad_records == nullptr) {
    YS_REQUIRE(a.energy, YS_ERR_INVALID, "energy-only evaluation needs the energy output");
    affine_value_kernel<E><<<grid_for(a.num_elements, 128), 128, 0, s>>>(a);
    YS_CHECK_LAUNCH();
    return YS_OK;
  }
  YS_REQUIRE(a.block_records && a.grad_records, YS_ERR_INVALID, "block and gradient records go together");
  YS_REQUIRE(a.plan.slot_stride >= 1 && a.plan.K == (uint32_t)E::A * a.plan.slot_stride, YS_ERR_INVALID,
             "K must be the argument count * slot_stride");
  constexpr int N = 3 * E::A;
  const size_t smem = sizeof(double) * project_stash_doubles<N>() * kEnergyThreads;
  YS_CUDA_TRY(cudaFuncSetAttribute(affine_kernel<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  affine_kernel<E><<<grid_for(a.num_elements, kEnergyThreads), kEnergyThreads, smem, s>>>(a);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

// ---- contact through affine-body vertices ----------------------------------
// A barrier element over V union vertices, some of them affine-body vertices
// x = A_b xbar + t_b.  Leaves per vertex: slot 0 the position of a plain
// vertex; slots 0..2 the rows of A and slot 3 t for an affine vertex.  The
// Jacobian block of slot s of vertex v (3 rows of x_v, 3 leaf entries) is
// I3 for a plain position or t, and e_s xbar^T for row s of A.

constexpr uint32_t kNoBody = 0xffffffffu;

struct CoupledVertex {
  double xbar[3];
  uint32_t body;  // kNoBody: plain (free or DATA) vertex
};

struct UnionCodes {
  uint32_t prefix[YS_MAX_UNION + 1];
  int32_t kind[YS_MAX_UNION];
  uint32_t wrt_start[YS_MAX_UNION];
  uint32_t num_children;
};

// Union child of index idx (the last child whose range starts at or before it).
__device__ __forceinline__ uint32_t union_child(const uint32_t* prefix, uint32_t num_children, uint32_t idx) {
  uint32_t c = 0;
#pragma unroll
  for (int k = 1; k < YS_MAX_UNION; ++k)
    if (k < (int)num_children && idx >= prefix[k]) c = k;
  return c;
}

__device__ __forceinline__ uint32_t leaf_code(int32_t kind, uint32_t wrt_start, uint32_t local) {
  return kind == 2 ? wrt_start + 3u * local + 2u : (kind == 1 ? 1u : 0u);
}

__global__ void coupled_codes_kernel(const uint32_t* __restrict__ conn, uint32_t n, uint32_t V, UnionCodes u,
                                     uint32_t affine_child, const uint32_t* __restrict__ vertex_body,
                                     uint32_t num_bodies, int32_t a_kind, uint32_t a_wrt, int32_t t_kind,
                                     uint32_t t_wrt, uint32_t* __restrict__ codes, uint16_t* __restrict__ sizes) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  for (uint32_t v = 0; v < V; ++v) {
    const uint32_t idx = conn[(uint64_t)t * V + v];
    const uint64_t base = (uint64_t)t * 4 * V + 4 * v;
    uint32_t c4[4] = {0u, 0u, 0u, 0u};
    if (idx < u.prefix[u.num_children]) {
      const uint32_t c = union_child(u.prefix, u.num_children, idx);
      const uint32_t local = idx - u.prefix[c];
      if (c == affine_child) {
        const uint32_t b = vertex_body[local];
        if (b < num_bodies) {
#pragma unroll
          for (int r = 0; r < 3; ++r) c4[r] = leaf_code(a_kind, a_wrt, 3u * b + r);
          c4[3] = leaf_code(t_kind, t_wrt, b);
        }
      } else {
        c4[0] = leaf_code(u.kind[c], u.wrt_start[c], local);
      }
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      codes[base + s] = c4[s];
      sizes[base + s] = c4[s] ? (uint16_t)3 : (uint16_t)0;
    }
  }
}

__device__ __forceinline__ bool load_coupled_point(const ys_coupled_args& a, uint32_t idx, double (&p)[3],
                                                   CoupledVertex& cv) {
  const ys_union3& u = a.base.position;
  if (idx >= u.prefix[u.num_children]) return false;
  const uint32_t c = union_child(u.prefix, u.num_children, idx);
  const uint32_t local = idx - u.prefix[c];
  if (c != a.affine_child) {
    const double* s = u.child[c] + 3ull * local;
    p[0] = __ldg(s);
    p[1] = __ldg(s + 1);
    p[2] = __ldg(s + 2);
    cv.body = kNoBody;
    cv.xbar[0] = cv.xbar[1] = cv.xbar[2] = 0.0;
    return true;
  }
  const uint32_t b = __ldg(a.vertex_body + local);
  if (b >= a.num_bodies) return false;
  load_rest3(a.rest, local, cv.xbar);
  cv.body = b;
  const double* A = a.affine + 9ull * b;
  const double* tr = a.translation + 3ull * b;
#pragma unroll
  for (int r = 0; r < 3; ++r)
    p[r] = __ldg(A + 3 * r) * cv.xbar[0] + __ldg(A + 3 * r + 1) * cv.xbar[1] + __ldg(A + 3 * r + 2) * cv.xbar[2] +
           __ldg(tr + r);
  return true;
}

// J^T g for slot s of vertex cv.
__device__ __forceinline__ void coupled_jt_vec(const CoupledVertex& cv, int s, const double* g, double (&out)[3]) {
  if (cv.body != kNoBody && s < 3) {
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = cv.xbar[c] * g[s];
  } else {
    out[0] = g[0];
    out[1] = g[1];
    out[2] = g[2];
  }
}

// Records of the compressed Hessian: target slots merged by code in
// first-occurrence order (the coordinates' order), block (gi, gj) =
// sum over slots k in gi, l in gj of J_k^T H(v_k, v_l) J_l, transposed when
// the row leaf's code exceeds the column leaf's.
template <int V>
__device__ __forceinline__ void coupled_records(const uint32_t (&code)[4 * V], const CoupledVertex (&cv)[V],
                                                uint32_t occ0, const uint32_t* record, double* out,
                                                const double (&h)[3 * V * (3 * V + 1) / 2]) {
  constexpr int N = 3 * V, K = 4 * V;
  int group[K], first[K];
  int nfirst = 0;
  for (int k = 0; k < K; ++k) {
    group[k] = -1;
    if (code[k] < 2) continue;
    int g = -1;
    for (int q = 0; q < nfirst; ++q)
      if (code[first[q]] == code[k]) g = q;
    if (g < 0) { first[nfirst] = k; g = nfirst++; }
    group[k] = g;
  }
  uint32_t occ = occ0;
  for (int gi = 0; gi < nfirst; ++gi)
    for (int gj = gi; gj < nfirst; ++gj) {
      double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int ka = 0; ka < K; ++ka) {
        if (group[ka] != gi) continue;
        const int v = ka >> 2, s = ka & 3;
        const bool rowA = cv[v].body != kNoBody && s < 3;
        for (int kb = 0; kb < K; ++kb) {
          if (group[kb] != gj) continue;
          const int w = kb >> 2, u = kb & 3;
          const bool rowB = cv[w].body != kNoBody && u < 3;
          double hb[3][3], lt[3][3];
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) hb[r][c] = h[sym<N>(3 * v + r, 3 * w + c)];
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) lt[r][c] = rowA ? cv[v].xbar[r] * hb[s][c] : hb[r][c];
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[r][c] += rowB ? lt[r][u] * cv[w].xbar[c] : lt[r][c];
        }
      }
      double* dst = out + record[occ++];
      const bool upper = code[first[gi]] < code[first[gj]];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[3 * r + c] = upper ? acc[r][c] : acc[c][r];
    }
}

template <class E>
__global__ void __launch_bounds__(kEnergyThreads) coupled_kernel(const ys_coupled_args a) {
  constexpr int V = E::A, N = 3 * V, K = 4 * V;
  extern __shared__ double energy_stash[];
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.base.num_elements) return;
  Pts<V> x, r;
  CoupledVertex cv[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const uint32_t id = a.base.conn[(uint64_t)t * V + v];
    if (!load_coupled_point(a, id, x.p[v], cv[v])) {
      if (a.status) atomicCAS(a.status, 0, (int32_t)(t + 1));
      return;
    }
    if (a.base.rest.num_children) load_point(a.base.rest, id, r.p[v]);  // friction: old positions
    else r.p[v][0] = r.p[v][1] = r.p[v][2] = 0.0;
  }
  const HD<N> e = E::template eval<N>(a.base, t, x, r);
  if (a.base.energy) a.base.energy[t] = e.v;
  uint32_t code[K];
#pragma unroll
  for (int k = 0; k < K; ++k) code[k] = a.base.plan.codes[(uint64_t)t * K + k];
  uint32_t q = a.base.plan.grad_outer[t];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (code[k] < 2) continue;
    double gq[3];
    coupled_jt_vec(cv[k >> 2], k & 3, &e.g[3 * (k >> 2)], gq);
    double* dst = a.base.grad_records + a.base.plan.grad_record[q++];
    dst[0] = gq[0];
    dst[1] = gq[1];
    dst[2] = gq[2];
  }
  double h[HD<N>::H];
#pragma unroll
  for (int i = 0; i < HD<N>::H; ++i) h[i] = e.h[i];
  // The leaves map linearly to the vertex positions, so the Hessian with
  // respect to the positions is projected (the inner projection of the
  // reference, PKG/differentiator/differentiator.pyx:795-799) and then mapped
  // to the leaves by coupled_records.
  if (a.base.projection_method >= 1) {
    double s[HD<N>::H];
#pragma unroll
    for (int rr = 0; rr < N; ++rr)
#pragma unroll
      for (int c = 0; c <= rr; ++c) s[tri(rr, c)] = h[utri<N>(c, rr)];
    if (!psd_test_packed<N>(s))
      project_negative_modes<N>(h, a.base.projection_method, energy_stash + threadIdx.x, blockDim.x);
  }
  coupled_records<V>(code, cv, a.base.plan.coord_outer[t], a.base.plan.record, a.base.block_records, h);
}

template <class E>
__global__ void __launch_bounds__(128) coupled_value_kernel(const ys_coupled_args a) {
  constexpr int V = E::A;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.base.num_elements) return;
  Pts<V> x, r;
  CoupledVertex cv[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const uint32_t id = a.base.conn[(uint64_t)t * V + v];
    if (!load_coupled_point(a, id, x.p[v], cv[v])) {
      if (a.status) atomicCAS(a.status, 0, (int32_t)(t + 1));
      a.base.energy[t] = 0.0;
      return;
    }
    if (a.base.rest.num_children) load_point(a.base.rest, id, r.p[v]);
    else r.p[v][0] = r.p[v][1] = r.p[v][2] = 0.0;
  }
  a.base.energy[t] = E::template eval<0>(a.base, t, x, r).v;
}

template <class E>
static int32_t launch_coupled(const ys_coupled_args& a, cudaStream_t s) {
  YS_REQUIRE(a.base.arity == (uint32_t)E::A, YS_ERR_INVALID, "arity does not match the energy kind");
  if (a.base.block_records == nullptr && a.base.grad_records == nullptr) {
    YS_REQUIRE(a.base.energy, YS_ERR_INVALID, "energy-only evaluation needs the energy output");
    coupled_value_kernel<E><<<grid_for(a.base.num_elements, 128), 128, 0, s>>>(a);
    YS_CHECK_LAUNCH();
    return YS_OK;
  }
  YS_REQUIRE(a.base.block_records && a.base.grad_records, YS_ERR_INVALID, "block and gradient records go together");
  YS_REQUIRE(a.base.plan.slot_stride == 1 && a.base.plan.K == 4u * E::A, YS_ERR_INVALID,
             "coupled codes take K = 4 * arity slots, stride 1");
  constexpr int N = 3 * E::A;
  const size_t smem = sizeof(double) * project_stash_doubles<N>() * kEnergyThreads;
  YS_CUDA_TRY(cudaFuncSetAttribute(coupled_kernel<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  coupled_kernel<E><<<grid_for(a.base.num_elements, kEnergyThreads), kEnergyThreads, smem, s>>>(a);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

}  // namespace ys

extern "C" {

int32_t ys_rest_local_hessians(const ys_energy_args* args, double* out, void* stream) {
  YS_REQUIRE(args != nullptr && out != nullptr, YS_ERR_INVALID, "null argument");
  const ys_energy_args& a = *args;
  YS_REQUIRE(a.position.num_children >= 1 && a.position.num_children <= YS_MAX_UNION, YS_ERR_INVALID,
             "bad position union");
  YS_REQUIRE(a.rest.num_children >= 1 && a.rest.num_children <= YS_MAX_UNION, YS_ERR_INVALID,
             "the rest form needs rest positions");
  const int A = a.kind == YS_ENERGY_BENDING ? 4
                : (a.kind == YS_ENERGY_BARAFF_WITKIN || a.kind == YS_ENERGY_STVK_MEMBRANE) ? 3 : 0;
  YS_REQUIRE(A != 0, YS_ERR_INVALID, "rest-position derivatives: bending, Baraff-Witkin and StVK membranes only");
  YS_REQUIRE(a.arity == (uint32_t)A, YS_ERR_INVALID, "arity does not match the energy kind");
  if (a.num_elements == 0) return YS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (A == 4)
    ys::rest_local_hessian_kernel<4><<<ys::grid_for(a.num_elements, 64), 64, 0, s>>>(a, out);
  else
    ys::rest_local_hessian_kernel<3><<<ys::grid_for(a.num_elements, 64), 64, 0, s>>>(a, out);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_local_hessians(const ys_energy_args* args, double* out, void* stream) {
  YS_REQUIRE(args != nullptr && out != nullptr, YS_ERR_INVALID, "null argument");
  const ys_energy_args& a = *args;
  YS_REQUIRE(a.position.num_children >= 1 && a.position.num_children <= YS_MAX_UNION, YS_ERR_INVALID,
             "bad position union");
  YS_REQUIRE(a.rest.num_children <= YS_MAX_UNION, YS_ERR_INVALID, "bad rest union");
  const bool friction = a.kind == YS_ENERGY_FRICTION_PT || a.kind == YS_ENERGY_FRICTION_PE ||
                        a.kind == YS_ENERGY_FRICTION_EE || a.kind == YS_ENERGY_FRICTION_PP;
  const bool needs_rest = a.kind == YS_ENERGY_BENDING || a.kind == YS_ENERGY_BARAFF_WITKIN ||
                          a.kind == YS_ENERGY_STVK_MEMBRANE || friction;
  YS_REQUIRE(!needs_rest || a.rest.num_children >= 1, YS_ERR_INVALID, "this energy needs rest positions");
  YS_REQUIRE(!friction || (a.params && a.param_stride >= 9), YS_ERR_INVALID,
             "friction needs 9 lagged parameters per element");
  if (a.num_elements == 0) return YS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  switch (a.kind) {
    case YS_ENERGY_POINT_POINT: return ys::launch_local_hessian<ys::PointPoint>(a, out, s);
    case YS_ENERGY_POINT_EDGE: return ys::launch_local_hessian<ys::PointEdge>(a, out, s);
    case YS_ENERGY_POINT_TRIANGLE: return ys::launch_local_hessian<ys::PointTriangle>(a, out, s);
    case YS_ENERGY_EDGE_EDGE: return ys::launch_local_hessian<ys::EdgeEdge>(a, out, s);
    case YS_ENERGY_BENDING: return ys::launch_local_hessian<ys::Bending>(a, out, s);
    case YS_ENERGY_BARAFF_WITKIN: return ys::launch_local_hessian<ys::BaraffWitkin>(a, out, s);
    case YS_ENERGY_STVK_MEMBRANE: return ys::launch_local_hessian<ys::StvkMembrane>(a, out, s);
    case YS_ENERGY_FRICTION_PT: return ys::launch_local_hessian<ys::FrictionPT>(a, out, s);
    case YS_ENERGY_FRICTION_PE: return ys::launch_local_hessian<ys::FrictionPE>(a, out, s);
    case YS_ENERGY_FRICTION_EE: return ys::launch_local_hessian<ys::FrictionEE>(a, out, s);
    case YS_ENERGY_FRICTION_PP: return ys::launch_local_hessian<ys::FrictionPP>(a, out, s);
    default: break;
  }
  ys_set_last_error("unknown energy kind", __FILE__, __LINE__);
  return YS_ERR_INVALID;
}

int32_t ys_energy_eval(const ys_energy_args* args, void* stream) {
  YS_REQUIRE(args != nullptr, YS_ERR_INVALID, "null args");
  const ys_energy_args& a = *args;
  YS_REQUIRE(a.position.num_children >= 1 && a.position.num_children <= YS_MAX_UNION, YS_ERR_INVALID,
             "bad position union");
  YS_REQUIRE(a.rest.num_children <= YS_MAX_UNION, YS_ERR_INVALID, "bad rest union");
  if (a.num_elements == 0) return YS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const bool friction = a.kind == YS_ENERGY_FRICTION_PT || a.kind == YS_ENERGY_FRICTION_PE ||
                        a.kind == YS_ENERGY_FRICTION_EE || a.kind == YS_ENERGY_FRICTION_PP;
  const bool needs_rest = a.kind == YS_ENERGY_BENDING || a.kind == YS_ENERGY_BARAFF_WITKIN ||
                          a.kind == YS_ENERGY_STVK_MEMBRANE || friction;
  YS_REQUIRE(!needs_rest || a.rest.num_children >= 1, YS_ERR_INVALID, "this energy needs rest positions");
  YS_REQUIRE(!friction || (a.params && a.param_stride >= 9), YS_ERR_INVALID,
             "friction needs 9 lagged parameters per element");
  if (a.block_records == nullptr && a.grad_records == nullptr) {
    // energy only
    YS_REQUIRE(a.energy, YS_ERR_INVALID, "energy-only evaluation needs the energy output");
    switch (a.kind) {
      case YS_ENERGY_POINT_POINT: return ys::launch_energy_value<ys::PointPoint>(a, s);
      case YS_ENERGY_POINT_EDGE: return ys::launch_energy_value<ys::PointEdge>(a, s);
      case YS_ENERGY_POINT_TRIANGLE: return ys::launch_energy_value<ys::PointTriangle>(a, s);
      case YS_ENERGY_EDGE_EDGE: return ys::launch_energy_value<ys::EdgeEdge>(a, s);
      case YS_ENERGY_BENDING: return ys::launch_energy_value<ys::Bending>(a, s);
      case YS_ENERGY_BARAFF_WITKIN: return ys::launch_energy_value<ys::BaraffWitkin>(a, s);
      case YS_ENERGY_STVK_MEMBRANE: return ys::launch_energy_value<ys::StvkMembrane>(a, s);
      case YS_ENERGY_FRICTION_PT: return ys::launch_energy_value<ys::FrictionPT>(a, s);
      case YS_ENERGY_FRICTION_PE: return ys::launch_energy_value<ys::FrictionPE>(a, s);
      case YS_ENERGY_FRICTION_EE: return ys::launch_energy_value<ys::FrictionEE>(a, s);
      case YS_ENERGY_FRICTION_PP: return ys::launch_energy_value<ys::FrictionPP>(a, s);
      default: break;
    }
    YS_REQUIRE(false, YS_ERR_INVALID, "unknown energy kind");
  }
  YS_REQUIRE(a.plan.slot_stride >= 1 && a.plan.K == a.arity * a.plan.slot_stride, YS_ERR_INVALID,
             "K must be arity * slot_stride");
  switch (a.kind) {
    case YS_ENERGY_POINT_POINT: return ys::launch_energy<ys::PointPoint>(a, s);
    case YS_ENERGY_POINT_EDGE: return ys::launch_energy<ys::PointEdge>(a, s);
    case YS_ENERGY_POINT_TRIANGLE: return ys::launch_energy<ys::PointTriangle>(a, s);
    case YS_ENERGY_EDGE_EDGE: return ys::launch_energy<ys::EdgeEdge>(a, s);
    case YS_ENERGY_BENDING: return ys::launch_energy<ys::Bending>(a, s);
    case YS_ENERGY_BARAFF_WITKIN: return ys::launch_energy<ys::BaraffWitkin>(a, s);
    case YS_ENERGY_STVK_MEMBRANE: return ys::launch_energy<ys::StvkMembrane>(a, s);
    case YS_ENERGY_FRICTION_PT: return ys::launch_energy<ys::FrictionPT>(a, s);
    case YS_ENERGY_FRICTION_PE: return ys::launch_energy<ys::FrictionPE>(a, s);
    case YS_ENERGY_FRICTION_EE: return ys::launch_energy<ys::FrictionEE>(a, s);
    case YS_ENERGY_FRICTION_PP: return ys::launch_energy<ys::FrictionPP>(a, s);
    default: break;
  }
  YS_REQUIRE(false, YS_ERR_INVALID, "unknown energy kind");
}

int32_t ys_affine_eval(const ys_affine_args* args, void* stream) {
  YS_REQUIRE(args != nullptr, YS_ERR_INVALID, "null args");
  const ys_affine_args& a = *args;
  YS_REQUIRE(a.affine != nullptr && a.num_bodies > 0, YS_ERR_INVALID, "affine bodies needed");
  if (a.num_elements == 0) return YS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  switch (a.kind) {
    case YS_AFFINE_ORTHOGONALITY:
      YS_REQUIRE(a.tets == nullptr, YS_ERR_INVALID, "orthogonality takes no tets");
      return ys::launch_affine<ys::AffineOrthogonality>(a, s);
    case YS_AFFINE_INERTIA:
      YS_REQUIRE(a.translation && a.rest && a.x_before && a.mass && a.tets == nullptr, YS_ERR_INVALID,
                 "affine inertia needs translation, rest, x_before and mass");
      return ys::launch_affine<ys::AffineInertia>(a, s);
    case YS_AFFINE_SNH:
      YS_REQUIRE(a.translation && a.rest && a.tets && a.num_rest > 0, YS_ERR_INVALID,
                 "affine SNH needs translation, rest and tets");
      YS_REQUIRE(((uintptr_t)a.tets & 15u) == 0, YS_ERR_INVALID, "tets must be 16-byte aligned");
      YS_REQUIRE(a.lam || a.lam_value != 0.0, YS_ERR_INVALID, "affine SNH needs lambda (per element or a value)");
      return ys::launch_affine<ys::AffineSnh>(a, s);
    default: break;
  }
  YS_REQUIRE(false, YS_ERR_INVALID, "unknown affine kind");
}

int32_t ys_coupled_indices(const uint32_t* connectivity, uint32_t n, uint32_t arity, uint32_t num_children,
                           const uint32_t* child_prefix, const int32_t* child_kind,
                           const uint32_t* child_wrt_start, uint32_t affine_child,
                           const uint32_t* vertex_body, uint32_t num_bodies, int32_t affine_kind,
                           uint32_t affine_wrt_start, int32_t translation_kind,
                           uint32_t translation_wrt_start, uint32_t* codes, uint16_t* sizes,
                           void* stream) {
  YS_REQUIRE(arity >= 2 && arity <= 4, YS_ERR_INVALID, "coupled barriers take 2 to 4 vertices");
  YS_REQUIRE(num_children >= 1 && num_children <= YS_MAX_UNION && affine_child < num_children, YS_ERR_INVALID,
             "bad union or affine child");
  YS_REQUIRE(child_prefix && child_kind && child_wrt_start, YS_ERR_INVALID, "union description needed");
  if (n == 0) return YS_OK;
  YS_REQUIRE(connectivity && vertex_body && codes && sizes, YS_ERR_INVALID, "null pointer");
  ys::UnionCodes u{};
  for (uint32_t c = 0; c <= num_children; ++c) u.prefix[c] = child_prefix[c];
  for (uint32_t c = 0; c < num_children; ++c) { u.kind[c] = child_kind[c]; u.wrt_start[c] = child_wrt_start[c]; }
  u.num_children = num_children;
  ys::coupled_codes_kernel<<<ys::grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
      connectivity, n, arity, u, affine_child, vertex_body, num_bodies, affine_kind, affine_wrt_start,
      translation_kind, translation_wrt_start, codes, sizes);
  YS_CHECK_LAUNCH();
  return YS_OK;
}

int32_t ys_coupled_energy_eval(const ys_coupled_args* args, void* stream) {
  YS_REQUIRE(args != nullptr, YS_ERR_INVALID, "null args");
  const ys_coupled_args& a = *args;
  YS_REQUIRE(a.base.position.num_children >= 1 && a.base.position.num_children <= YS_MAX_UNION, YS_ERR_INVALID,
             "bad position union");
  YS_REQUIRE(a.affine_child < a.base.position.num_children, YS_ERR_INVALID, "affine child outside the union");
  YS_REQUIRE(a.vertex_body && a.rest && a.affine && a.translation && a.num_bodies > 0, YS_ERR_INVALID,
             "affine bodies needed");
  if (a.base.num_elements == 0) return YS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const bool friction = a.base.kind >= YS_ENERGY_FRICTION_PT && a.base.kind <= YS_ENERGY_FRICTION_PP;
  YS_REQUIRE(!friction || (a.base.rest.num_children >= 1 && a.base.params && a.base.param_stride >= 9),
             YS_ERR_INVALID, "friction needs the old positions and 9 lagged parameters per element");
  YS_REQUIRE(a.base.rest.num_children == 0 ||
                 a.base.rest.prefix[a.base.rest.num_children] >= a.base.position.prefix[a.base.position.num_children],
             YS_ERR_INVALID, "old positions must cover the position union");
  switch (a.base.kind) {
    case YS_ENERGY_POINT_POINT: return ys::launch_coupled<ys::PointPoint>(a, s);
    case YS_ENERGY_POINT_EDGE: return ys::launch_coupled<ys::PointEdge>(a, s);
    case YS_ENERGY_POINT_TRIANGLE: return ys::launch_coupled<ys::PointTriangle>(a, s);
    case YS_ENERGY_EDGE_EDGE: return ys::launch_coupled<ys::EdgeEdge>(a, s);
    case YS_ENERGY_FRICTION_PT: return ys::launch_coupled<ys::FrictionPT>(a, s);
    case YS_ENERGY_FRICTION_PE: return ys::launch_coupled<ys::FrictionPE>(a, s);
    case YS_ENERGY_FRICTION_EE: return ys::launch_coupled<ys::FrictionEE>(a, s);
    case YS_ENERGY_FRICTION_PP: return ys::launch_coupled<ys::FrictionPP>(a, s);
    default: break;
  }
  YS_REQUIRE(false, YS_ERR_INVALID, "coupled evaluation takes the contact barriers and the lagged friction kinds");
}

}  // extern "C"
