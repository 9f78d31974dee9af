// Second-order forward-mode automatic differentiation on the device.
//
// HD<N> carries a value, its gradient with respect to N inputs and its
// Hessian (packed upper triangle, utri<N>).  Energies written once with
// these numbers give their exact gradient and Hessian, the role the
// reference's symbolic differentiator and code generator play for its
// energies (PKG/codeGenerator/codeGenerator.pyx:159-369).  All loops have
// compile-time bounds and fully unroll, so the one-hot gradients of the
// inputs and their zero Hessians stay compile-time constants and the
// compiler drops the products with them.
//
// Rules (a, b inputs; f a scalar function):
//   a*b : g = a.g b + b.g a,  H = a.H b + b.H a + a.g b.g^T + b.g a.g^T
//   f(a): g = f' a.g,         H = f' a.H + f'' a.g a.g^T
//   atan2(y, x) with r = x^2 + y^2:
//         g = (x y.g - y x.g) / r,
//         H = (x y.H - y x.H)/r + (-2xy y.g y.g^T + 2xy x.g x.g^T
//             + (y^2 - x^2)(x.g y.g^T + y.g x.g^T)) / r^2
#pragma once

#include <cmath>

#include "ys_eigen.cuh"

namespace ys {

template <int N>
struct HD {
  static constexpr int H = N * (N + 1) / 2;
  double v;
  double g[N];
  double h[H];
};

// Value only (energy evaluation without derivatives): the loops over N = 0
// inputs are empty; the one-element arrays are never touched.
template <>
struct HD<0> {
  static constexpr int H = 0;
  double v;
  double g[1];
  double h[1];
};

template <int N>
__device__ __forceinline__ HD<N> hd_const(double c) {
  HD<N> r;
  r.v = c;
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = 0.0;
#pragma unroll
  for (int i = 0; i < HD<N>::H; ++i) r.h[i] = 0.0;
  return r;
}

template <int N>
__device__ __forceinline__ HD<N> hd_var(double x, int i) {
  HD<N> r = hd_const<N>(x);
#pragma unroll
  for (int k = 0; k < N; ++k) r.g[k] = k == i ? 1.0 : 0.0;
  return r;
}

template <int N>
__device__ __forceinline__ HD<N> operator+(const HD<N>& a, const HD<N>& b) {
  HD<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = a.g[i] + b.g[i];
#pragma unroll
  for (int i = 0; i < HD<N>::H; ++i) r.h[i] = a.h[i] + b.h[i];
  return r;
}

template <int N>
__device__ __forceinline__ HD<N> operator-(const HD<N>& a, const HD<N>& b) {
  HD<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = a.g[i] - b.g[i];
#pragma unroll
  for (int i = 0; i < HD<N>::H; ++i) r.h[i] = a.h[i] - b.h[i];
  return r;
}

template <int N>
__device__ __forceinline__ HD<N> operator*(double s, const HD<N>& a) {
  HD<N> r;
  r.v = s * a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = s * a.g[i];
#pragma unroll
  for (int i = 0; i < HD<N>::H; ++i) r.h[i] = s * a.h[i];
  return r;
}

template <int N>
__device__ __forceinline__ HD<N> operator+(const HD<N>& a, double c) {
  HD<N> r = a;
  r.v += c;
  return r;
}

template <int N>
__device__ __forceinline__ HD<N> operator-(const HD<N>& a, double c) {
  HD<N> r = a;
  r.v -= c;
  return r;
}

template <int N>
__device__ __forceinline__ HD<N> operator*(const HD<N>& a, const HD<N>& b) {
  HD<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = a.g[i] * b.v + b.g[i] * a.v;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = i; j < N; ++j) {
      const int k = utri<N>(i, j);
      r.h[k] = a.h[k] * b.v + b.h[k] * a.v + a.g[i] * b.g[j] + b.g[i] * a.g[j];
    }
  return r;
}

// f(a) from f(a.v), f'(a.v), f''(a.v).
template <int N>
__device__ __forceinline__ HD<N> hd_apply(const HD<N>& a, double f, double df, double d2f) {
  HD<N> r;
  r.v = f;
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = df * a.g[i];
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = i; j < N; ++j) {
      const int k = utri<N>(i, j);
      r.h[k] = df * a.h[k] + d2f * a.g[i] * a.g[j];
    }
  return r;
}

template <int N>
__device__ __forceinline__ HD<N> sq(const HD<N>& a) {
  return hd_apply(a, a.v * a.v, 2.0 * a.v, 2.0);
}

template <int N>
__device__ __forceinline__ HD<N> recip(const HD<N>& a) {
  const double i = 1.0 / a.v;
  return hd_apply(a, i, -i * i, 2.0 * i * i * i);
}

template <int N>
__device__ __forceinline__ HD<N> operator/(const HD<N>& a, const HD<N>& b) {
  return a * recip(b);
}

template <int N>
__device__ __forceinline__ HD<N> hd_sqrt(const HD<N>& a) {
  const double s = sqrt(a.v);
  return hd_apply(a, s, 0.5 / s, -0.25 / (s * a.v));
}

template <int N>
__device__ __forceinline__ HD<N> hd_log(const HD<N>& a) {
  const double i = 1.0 / a.v;
  return hd_apply(a, log(a.v), i, -i * i);
}

template <int N>
__device__ __forceinline__ HD<N> hd_atan2(const HD<N>& y, const HD<N>& x) {
  HD<N> r;
  const double r2 = x.v * x.v + y.v * y.v;
  const double ir = 1.0 / r2, ir2 = ir * ir;
  const double fy = x.v * ir, fx = -y.v * ir;
  const double fyy = -2.0 * x.v * y.v * ir2, fxx = 2.0 * x.v * y.v * ir2;
  const double fxy = (y.v * y.v - x.v * x.v) * ir2;
  r.v = atan2(y.v, x.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = fy * y.g[i] + fx * x.g[i];
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = i; j < N; ++j) {
      const int k = utri<N>(i, j);
      r.h[k] = fy * y.h[k] + fx * x.h[k] + fyy * y.g[i] * y.g[j] + fxx * x.g[i] * x.g[j] +
               fxy * (x.g[i] * y.g[j] + y.g[i] * x.g[j]);
    }
  return r;
}

// 3-vectors of HD numbers.
template <int N>
struct HV {
  HD<N> x, y, z;
};

template <int N>
__device__ __forceinline__ HV<N> hv_var(const double (&p)[3], int first) {
  return {hd_var<N>(p[0], first), hd_var<N>(p[1], first + 1), hd_var<N>(p[2], first + 2)};
}
template <int N>
__device__ __forceinline__ HV<N> operator-(const HV<N>& a, const HV<N>& b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <int N>
__device__ __forceinline__ HV<N> operator+(const HV<N>& a, const HV<N>& b) {
  return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <int N>
__device__ __forceinline__ HV<N> operator*(double s, const HV<N>& a) {
  return {s * a.x, s * a.y, s * a.z};
}
template <int N>
__device__ __forceinline__ HD<N> dot(const HV<N>& a, const HV<N>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <int N>
__device__ __forceinline__ HV<N> cross(const HV<N>& a, const HV<N>& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <int N>
__device__ __forceinline__ HD<N> norm(const HV<N>& a) {
  return hd_sqrt(dot(a, a));
}

// ---- hyper-dual numbers over two sets of 3 directions ----------------------
// H33 carries a value, its first derivatives in two sets of 3 inputs (set a:
// the coordinates of one vertex, set b: those of another, or the same) and
// the mixed second derivatives d2/(da db): one 3x3 block of a Hessian per
// evaluation.  Rules as for HD, with a.g b.g^T split into the two sets:
//   (f g).ab = f.ab g + f g.ab + f.a g.b^T + g.a f.b^T
//   h(f).ab  = h' f.ab + h'' f.a f.b^T
struct H33 {
  double v, a[3], b[3], ab[3][3];
};
__device__ __forceinline__ H33 h33c(double c) {
  H33 r;
  r.v = c;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r.a[i] = r.b[i] = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) r.ab[i][j] = 0.0;
  }
  return r;
}
__device__ __forceinline__ H33 operator+(const H33& f, const H33& g) {
  H33 r;
  r.v = f.v + g.v;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r.a[i] = f.a[i] + g.a[i];
    r.b[i] = f.b[i] + g.b[i];
#pragma unroll
    for (int j = 0; j < 3; ++j) r.ab[i][j] = f.ab[i][j] + g.ab[i][j];
  }
  return r;
}
__device__ __forceinline__ H33 operator*(double s, const H33& f) {
  H33 r;
  r.v = s * f.v;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r.a[i] = s * f.a[i];
    r.b[i] = s * f.b[i];
#pragma unroll
    for (int j = 0; j < 3; ++j) r.ab[i][j] = s * f.ab[i][j];
  }
  return r;
}
__device__ __forceinline__ H33 operator-(const H33& f, const H33& g) { return f + (-1.0) * g; }
__device__ __forceinline__ H33 operator*(const H33& f, const H33& g) {
  H33 r;
  r.v = f.v * g.v;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r.a[i] = f.a[i] * g.v + f.v * g.a[i];
    r.b[i] = f.b[i] * g.v + f.v * g.b[i];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      r.ab[i][j] = f.ab[i][j] * g.v + f.v * g.ab[i][j] + f.a[i] * g.b[j] + g.a[i] * f.b[j];
  return r;
}
// h(f) from h(f.v), h'(f.v), h''(f.v)
__device__ __forceinline__ H33 h33_apply(const H33& f, double h, double dh, double d2h) {
  H33 r;
  r.v = h;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r.a[i] = dh * f.a[i];
    r.b[i] = dh * f.b[i];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.ab[i][j] = dh * f.ab[i][j] + d2h * f.a[i] * f.b[j];
  return r;
}
__device__ __forceinline__ H33 h33_recip(const H33& f) {
  const double i = 1.0 / f.v;
  return h33_apply(f, i, -i * i, 2.0 * i * i * i);
}
__device__ __forceinline__ H33 h33_log(const H33& f) {
  const double i = 1.0 / f.v;
  return h33_apply(f, log(f.v), i, -i * i);
}


__device__ __forceinline__ H33 operator+(const H33& f, double c) {
  H33 r = f;
  r.v += c;
  return r;
}
__device__ __forceinline__ H33 operator-(const H33& f, double c) {
  H33 r = f;
  r.v -= c;
  return r;
}
__device__ __forceinline__ H33 operator/(const H33& f, const H33& g) { return f * h33_recip(g); }
__device__ __forceinline__ H33 h33_sqrt(const H33& f) {
  const double s = sqrt(f.v);
  return h33_apply(f, s, 0.5 / s, -0.25 / (s * f.v));
}
// atan2(y, x), the second-derivative terms of hd_atan2
__device__ __forceinline__ H33 h33_atan2(const H33& y, const H33& x) {
  const double r2 = x.v * x.v + y.v * y.v;
  const double ir = 1.0 / r2, ir2 = ir * ir;
  const double fy = x.v * ir, fx = -y.v * ir;
  const double fyy = -2.0 * x.v * y.v * ir2, fxx = 2.0 * x.v * y.v * ir2;
  const double fxy = (y.v * y.v - x.v * x.v) * ir2;
  H33 r;
  r.v = atan2(y.v, x.v);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r.a[i] = fy * y.a[i] + fx * x.a[i];
    r.b[i] = fy * y.b[i] + fx * x.b[i];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      r.ab[i][j] = fy * y.ab[i][j] + fx * x.ab[i][j] + fyy * y.a[i] * y.b[j] + fxx * x.a[i] * x.b[j] +
                   fxy * (x.a[i] * y.b[j] + y.a[i] * x.b[j]);
  return r;
}

}  // namespace ys
