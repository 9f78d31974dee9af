// Dense symmetric kernels used by the element projection (FP64).
//
// * psd_test_packed<N>: the reference's LDL^T PSD short-circuit
//   (PKG/kernel/Hessian/hessianKernelHeader.pyx:79-141), same operation order
//   (one correctly rounded reciprocal per column, FMA trailing update).
// * jacobi_eigen<N>: cyclic Jacobi eigen-decomposition (Jacobi 1846;
//   Golub & Van Loan, Matrix Computations, 4th ed., Alg. 8.5.2 with the
//   symmetric Schur 2x2 rotation of Alg. 8.5.1).  The reference calls Eigen's
//   SelfAdjointEigenSolver here; the projected matrix is the same to rounding.
#pragma once

#include <cmath>
#include <cstdint>

namespace ys {

// Lower-triangle packed index (row-major over rows, columns 0..row).
__host__ __device__ constexpr int tri(int r, int c) { return r * (r + 1) / 2 + c; }

// In-place test on a packed lower triangle `s` (destroyed).  Returns true when
// the matrix is positive semidefinite within 1e-10 * max(1, max |A_ii|).
template <int N>
__device__ __forceinline__ bool psd_test_packed(double* s) {
  double scale = 1.0;
#pragma unroll
  for (int r = 0; r < N; ++r) scale = fmax(scale, fabs(s[tri(r, r)]));
  const double tol = scale * 1.0e-10;
  bool ok = true;
#pragma unroll
  for (int c = 0; c < N; ++c) {
    const double pivot = s[tri(c, c)];
    if (pivot < -tol) ok = false;
    if (fabs(pivot) <= tol) {
#pragma unroll
      for (int r = c + 1; r < N; ++r)
        if (fabs(s[tri(r, c)]) > tol) ok = false;
      continue;
    }
    const double inv = __drcp_rn(pivot);
#pragma unroll
    for (int r = c + 1; r < N; ++r) {
      const double f = s[tri(r, c)] * inv;
#pragma unroll
      for (int t = c + 1; t <= r; ++t) s[tri(r, t)] = __fma_rn(-f, s[tri(t, c)], s[tri(r, t)]);
    }
  }
  return ok;
}

// Cyclic Jacobi on a full symmetric N x N matrix a (row-major, overwritten
// with a diagonal), eigenvectors in the columns of v.  Bounded sweeps.
template <int N>
__device__ void jacobi_eigen(double (&a)[N][N], double (&v)[N][N]) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) v[i][j] = i == j ? 1.0 : 0.0;
  double total = 0.0;
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) total += a[i][j] * a[i][j];
  if (total == 0.0) return;
  for (int sweep = 0; sweep < 24; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < N; ++p)
      for (int q = p + 1; q < N; ++q) off += a[p][q] * a[p][q];
    if (off <= 0.5e-30 * total) break;
    for (int p = 0; p < N - 1; ++p) {
      for (int q = p + 1; q < N; ++q) {
        const double apq = a[p][q];
        if (apq * apq <= 1.0e-36 * total) continue;
        const double app = a[p][p], aqq = a[q][q];
        const double tau = (aqq - app) / (2.0 * apq);
        double t;
        if (fabs(tau) > 1.0e150) t = 0.5 / tau;
        else t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = rsqrt(1.0 + t * t);
        const double s = t * c;
        a[p][p] = app - t * apq;
        a[q][q] = aqq + t * apq;
        a[p][q] = 0.0;
        a[q][p] = 0.0;
        for (int k = 0; k < N; ++k) {
          if (k == p || k == q) continue;
          const double akp = a[k][p], akq = a[k][q];
          const double nkp = c * akp - s * akq;
          const double nkq = s * akp + c * akq;
          a[k][p] = nkp; a[p][k] = nkp;
          a[k][q] = nkq; a[q][k] = nkq;
        }
        for (int k = 0; k < N; ++k) {
          const double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
    }
  }
}

// a <- V diag(f(lambda)) V^T with lambda = diag(a) after jacobi_eigen.
// method 1: |lambda| for negative eigenvalues, 2: 0 for negative eigenvalues.
template <int N>
__device__ void jacobi_reconstruct(double (&a)[N][N], const double (&v)[N][N], int method) {
  double w[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const double l = a[i][i];
    w[i] = l < 0.0 ? (method == 1 ? -l : 0.0) : l;
  }
  for (int i = 0; i < N; ++i) {
    for (int j = i; j < N; ++j) {
      double acc = 0.0;
      for (int k = 0; k < N; ++k) acc += v[i][k] * w[k] * v[j][k];
      a[i][j] = acc;
      a[j][i] = acc;
    }
  }
}

// Upper-triangle packed index for an N x N symmetric matrix (row <= col).
template <int N>
__host__ __device__ constexpr int utri(int r, int c) {
  return r <= c ? r * N - r * (r - 1) / 2 + (c - r) : c * N - c * (c - 1) / 2 + (r - c);
}

// Cyclic Jacobi with the matrix in registers (packed upper triangle `a`,
// fully unrolled so every index is a compile-time constant) and the
// eigenvectors in shared memory, thread-interleaved: v[(i*N + j) * stride].
// After return, a holds the eigenvalues on its diagonal.
template <int N>
__device__ __forceinline__ void jacobi_eigen_reg(double (&a)[N * (N + 1) / 2], double* __restrict__ v, int stride) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) v[(i * N + j) * stride] = i == j ? 1.0 : 0.0;
  double total = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = i; j < N; ++j) total += (i == j ? 1.0 : 2.0) * a[utri<N>(i, j)] * a[utri<N>(i, j)];
  if (total == 0.0) return;
  for (int sweep = 0; sweep < 24; ++sweep) {
    double off = 0.0;
#pragma unroll
    for (int p = 0; p < N; ++p)
#pragma unroll
      for (int q = p + 1; q < N; ++q) off += a[utri<N>(p, q)] * a[utri<N>(p, q)];
    // Converged when the off-diagonal Frobenius norm is below 1e-15 of the
    // matrix norm (rounding noise keeps it from reaching zero); rotations
    // of entries below 1e-18 of the norm are skipped (threshold Jacobi).
    if (off <= 0.5e-30 * total) break;
    const double skip = 1.0e-36 * total;
#pragma unroll
    for (int p = 0; p < N - 1; ++p) {
#pragma unroll
      for (int q = p + 1; q < N; ++q) {
        // Branch-free: a skipped rotation is the identity (t = 0, c = 1, s = 0),
        // so every thread of a warp runs the same instruction stream.
        const double apq = a[utri<N>(p, q)];
        const bool rot = apq * apq > skip;
        const double app = a[utri<N>(p, p)], aqq = a[utri<N>(q, q)];
        const double tau = (aqq - app) / (rot ? 2.0 * apq : 1.0);
        double t = fabs(tau) > 1.0e150 ? 0.5 / tau
                                       : (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        t = rot ? t : 0.0;
        const double c = rsqrt(1.0 + t * t);
        const double s = t * c;
        a[utri<N>(p, p)] = app - t * apq;
        a[utri<N>(q, q)] = aqq + t * apq;
        a[utri<N>(p, q)] = rot ? 0.0 : apq;
#pragma unroll
        for (int k = 0; k < N; ++k) {
          if (k == p || k == q) continue;
          const double akp = a[utri<N>(k, p)], akq = a[utri<N>(k, q)];
          a[utri<N>(k, p)] = c * akp - s * akq;
          a[utri<N>(k, q)] = s * akp + c * akq;
        }
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const double vkp = v[(k * N + p) * stride], vkq = v[(k * N + q) * stride];
          v[(k * N + p) * stride] = c * vkp - s * vkq;
          v[(k * N + q) * stride] = s * vkp + c * vkq;
        }
      }
    }
  }
}

// Round-robin ("tournament") ordering of the N(N-1)/2 rotations of a sweep
// (Brent & Luk, 1985): with M = N rounded up to even, round r pairs the
// players of the circle method; rotations of one round act on disjoint
// planes, so they commute and their angles depend only on the matrix at the
// start of the round.  Computing all angles of a round first gives the FP64
// pipe independent work instead of one long dependency chain.
__host__ __device__ constexpr int rr_player(int m, int r, int i) { return i == 0 ? 0 : 1 + ((i - 1 + r) % (m - 1)); }

template <int N>
__device__ __forceinline__ void jacobi_eigen_rr(double (&a)[N * (N + 1) / 2], double* __restrict__ v, int stride) {
  constexpr int M = (N % 2) ? N + 1 : N;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) v[(i * N + j) * stride] = i == j ? 1.0 : 0.0;
  double total = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = i; j < N; ++j) total += (i == j ? 1.0 : 2.0) * a[utri<N>(i, j)] * a[utri<N>(i, j)];
  if (total == 0.0) return;
  for (int sweep = 0; sweep < 24; ++sweep) {
    double off = 0.0;
#pragma unroll
    for (int p = 0; p < N; ++p)
#pragma unroll
      for (int q = p + 1; q < N; ++q) off += a[utri<N>(p, q)] * a[utri<N>(p, q)];
    if (off <= 0.5e-30 * total) break;
    const double skip = 1.0e-36 * total;
#pragma unroll
    for (int r = 0; r < M - 1; ++r) {
      double cs[M / 2], sn[M / 2], tt[M / 2];
#pragma unroll
      for (int i = 0; i < M / 2; ++i) {
        const int u = rr_player(M, r, i), w = rr_player(M, r, M - 1 - i);
        const int p = u < w ? u : w, q = u < w ? w : u;
        if (q >= N) continue;
        const double apq = a[utri<N>(p, q)];
        const bool rot = apq * apq > skip;
        const double tau = (a[utri<N>(q, q)] - a[utri<N>(p, p)]) / (rot ? 2.0 * apq : 1.0);
        double t = fabs(tau) > 1.0e150 ? 0.5 / tau
                                       : (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        t = rot ? t : 0.0;
        tt[i] = t;
        cs[i] = rsqrt(1.0 + t * t);
        sn[i] = t * cs[i];
      }
#pragma unroll
      for (int i = 0; i < M / 2; ++i) {
        const int u = rr_player(M, r, i), w = rr_player(M, r, M - 1 - i);
        const int p = u < w ? u : w, q = u < w ? w : u;
        if (q >= N) continue;
        const double t = tt[i], c = cs[i], s = sn[i];
        const double apq = a[utri<N>(p, q)];
        a[utri<N>(p, p)] -= t * apq;
        a[utri<N>(q, q)] += t * apq;
        a[utri<N>(p, q)] = t != 0.0 ? 0.0 : apq;
#pragma unroll
        for (int k = 0; k < N; ++k) {
          if (k == p || k == q) continue;
          const double akp = a[utri<N>(k, p)], akq = a[utri<N>(k, q)];
          a[utri<N>(k, p)] = c * akp - s * akq;
          a[utri<N>(k, q)] = s * akp + c * akq;
        }
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const double vkp = v[(k * N + p) * stride], vkq = v[(k * N + q) * stride];
          v[(k * N + p) * stride] = c * vkp - s * vkq;
          v[(k * N + q) * stride] = s * vkp + c * vkq;
        }
      }
    }
  }
}

// a <- V diag(f(lambda)) V^T in place (packed upper), V in shared memory.
template <int N>
__device__ __forceinline__ void jacobi_reconstruct_reg(double (&a)[N * (N + 1) / 2], const double* __restrict__ v,
                                                       int stride, int method) {
  double w[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const double l = a[utri<N>(i, i)];
    w[i] = l < 0.0 ? (method == 1 ? -l : 0.0) : l;
  }
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double vi[N];
#pragma unroll
    for (int k = 0; k < N; ++k) vi[k] = v[(i * N + k) * stride] * w[k];
#pragma unroll
    for (int j = i; j < N; ++j) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < N; ++k) acc += vi[k] * v[(j * N + k) * stride];
      a[utri<N>(i, j)] = acc;
    }
  }
}

}  // namespace ys
