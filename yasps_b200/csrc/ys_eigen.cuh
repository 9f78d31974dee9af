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

// ---- projection by negative modes -------------------------------------------
//
// proj(A) = A + sum_{lambda_i < 0} (f(lambda_i) - lambda_i) v_i v_i^T with
// f = |.| (method 1) or max(., 0) (method 2): the same matrix as rebuilding
// V diag(f(lambda)) V^T, but only the (few) negative eigenpairs are needed.
//   1. Householder tridiagonalisation A = Q T Q^T (Golub & Van Loan, Matrix
//      Computations, 4th ed., Alg. 8.3.1), reflectors kept in the rows of `a`;
//   2. the negative eigenvalues of T by bisection on the Sturm sign count of
//      the characteristic-polynomial recurrence p_i = (d_i - x) p_{i-1} -
//      e_{i-1}^2 p_{i-2} (GVL 8.4.1), on T scaled to unit size, so no
//      division is needed in the count;
//   3. their eigenvectors of T by inverse iteration (T split at negligible
//      off-diagonals; tridiagonal LU with partial pivoting and pivots of at
//      least eps, two solves, Gram-Schmidt against the vectors found before,
//      which separates clustered eigenvalues), mapped back by Q;
//   4. A rebuilt by `build` and corrected by the rank-one terms.

template <int N>
__host__ __device__ constexpr int sym(int r, int c) { return r <= c ? utri<N>(r, c) : utri<N>(c, r); }

// Number of eigenvalues of the tridiagonal (d, e2 = e^2) below x.
template <int N>
__device__ __forceinline__ int sturm_count(const double (&d)[N], const double (&e2)[N], double x) {
  double p0 = 1.0, p1 = d[0] - x;
  bool neg = p1 <= 0.0;  // p_0 = 1 > 0: a zero p_1 counts as negative
  int count = neg ? 1 : 0;
  bool neg_prev = neg;
#pragma unroll
  for (int i = 1; i < N; ++i) {
    const double p2 = (d[i] - x) * p1 - e2[i - 1] * p0;
    // a zero term takes the sign opposite to the previous one
    neg = p2 < 0.0 || (p2 == 0.0 && !neg_prev);
    count += neg != neg_prev ? 1 : 0;
    neg_prev = neg;
    p0 = p1;
    p1 = p2;
  }
  return count;
}

// Shared-memory stash of one thread (thread-interleaved, stride `stride`):
// the original matrix, the reflectors and their beta, read back only once.
template <int N>
__host__ __device__ constexpr int project_stash_doubles() {
  return N * (N + 1) / 2 + (N - 1) * N / 2 - 1 + (N - 2);
}

template <int N>
__device__ __forceinline__ void project_negative_modes(double (&a)[N * (N + 1) / 2], int method,
                                                       double* __restrict__ stash, int stride) {
  constexpr int KS = N * (N + 1) / 2;        // original matrix
  constexpr int RS = KS;                     // reflector k, entries k+1..N-1
  constexpr int BS = RS + (N - 1) * N / 2 - 1;  // beta_k
  auto refl = [](int k, int i) { return k * (2 * N - k - 1) / 2 + (i - k - 1); };  // rows k = 0..N-3
#pragma unroll
  for (int i = 0; i < KS; ++i) stash[i * stride] = a[i];
  // -- 1. tridiagonalisation ------------------------------------------------------
  double e[N];
#pragma unroll
  for (int k = 0; k < N; ++k) e[k] = 0.0;
#pragma unroll
  for (int k = 0; k < N - 2; ++k) {
    double xn2 = 0.0;
#pragma unroll
    for (int i = k + 1; i < N; ++i) xn2 += a[utri<N>(k, i)] * a[utri<N>(k, i)];
    const double x0 = a[utri<N>(k, k + 1)];
    const double xn = sqrt(xn2);
    const double alpha = x0 >= 0.0 ? -xn : xn;
    const double v0 = x0 - alpha;
    const double vn2 = xn2 - x0 * x0 + v0 * v0;
    const double b = vn2 > 0.0 ? 2.0 / vn2 : 0.0;
    a[utri<N>(k, k + 1)] = v0;  // row k holds v (entries k+1..N-1)
    double pv[N];
#pragma unroll
    for (int i = k + 1; i < N; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int j = k + 1; j < N; ++j) acc += a[sym<N>(i, j)] * a[utri<N>(k, j)];
      pv[i] = b * acc;
    }
    double ptv = 0.0;
#pragma unroll
    for (int i = k + 1; i < N; ++i) ptv += pv[i] * a[utri<N>(k, i)];
    const double half = 0.5 * b * ptv;
#pragma unroll
    for (int i = k + 1; i < N; ++i) pv[i] -= half * a[utri<N>(k, i)];  // w
#pragma unroll
    for (int i = k + 1; i < N; ++i)
#pragma unroll
      for (int j = i; j < N; ++j)
        a[utri<N>(i, j)] -= a[utri<N>(k, i)] * pv[j] + pv[i] * a[utri<N>(k, j)];
#pragma unroll
    for (int i = k + 1; i < N; ++i) stash[(RS + refl(k, i)) * stride] = a[utri<N>(k, i)];
    stash[(BS + k) * stride] = b;
    e[k] = alpha;
  }
  e[N - 2] = a[utri<N>(N - 2, N - 1)];
  double d[N], e2[N];
  double g = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    d[i] = a[utri<N>(i, i)];
    const double r = fabs(d[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < N - 1 ? fabs(e[i]) : 0.0);
    g = fmax(g, r);
  }
  if (!(g > 0.0) || !isfinite(g)) {
#pragma unroll
    for (int i = 0; i < KS; ++i) a[i] = stash[i * stride];
    return;
  }
  // unit scale (Gershgorin bound 1)
  const double sc = 1.0 / g;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    d[i] *= sc;
    // split at negligible off-diagonals (blocks then decouple exactly in the
    // solves below, as in LAPACK's tridiagonal eigenvector routines)
    e[i] = fabs(e[i] * sc) <= 8.9e-16 ? 0.0 : e[i] * sc;
    e2[i] = e[i] * e[i];
  }
  // -- 2. negative eigenvalues ---------------------------------------------------
  const int nneg = sturm_count<N>(d, e2, 0.0);
  double vecs[N][N];  // eigenvectors of T for the negative modes (local memory)
  // The loop runs warp-uniformly to the warp's largest count (lanes past
  // their own count compute a masked dummy mode): every local-memory access
  // of an iteration is then at the same offset in all lanes (coalesced).
  const int mmax = __reduce_max_sync(__activemask(), nneg);
  for (int m = 0; m < mmax; ++m) {
    const bool live = m < nneg;
    double lo = -1.0 - 1e-12, hi = 0.0;
    for (int it = 0; it < 56; ++it) {
      const double mid = 0.5 * (lo + hi);
      const bool up = sturm_count<N>(d, e2, mid) > m;
      hi = up ? mid : hi;
      lo = up ? lo : mid;
    }
    const double lam = 0.5 * (lo + hi);
    // -- 3. inverse iteration on T - lam I ---------------------------------------
    // LU of T - lam I with partial pivoting (rows i, i+1 swapped when the
    // subdiagonal entry is larger), once for both solves; U rows hold
    // (pivot, u1, u2) at columns (i, i+1, i+2), kept as pivot reciprocals.
    // Pivots below eps (unit scale) are raised to eps: every member of a
    // cluster is amplified alike, so Gram-Schmidt can separate them.
    double mlt[N], u1[N], u2[N], ipiv[N];
    bool swp[N];
    {
      double pb = d[0] - lam, pc = e[0], pf = 0.0;
#pragma unroll
      for (int i = 0; i < N - 1; ++i) {
        const double na = e[i], nb = d[i + 1] - lam, nc = i + 1 < N - 1 ? e[i + 1] : 0.0;
        const bool sw = fabs(na) > fabs(pb);
        const double r0 = sw ? na : pb, r1 = sw ? nb : pc, r2 = sw ? nc : pf;
        const double o0 = sw ? pb : na, o1 = sw ? pc : nb, o2 = sw ? pf : nc;
        const double piv = fabs(r0) >= 2.2e-16 ? r0 : (r0 >= 0.0 ? 2.2e-16 : -2.2e-16);
        const double ip = 1.0 / piv;
        const double ml = o0 * ip;
        swp[i] = sw; mlt[i] = ml; u1[i] = r1; u2[i] = r2; ipiv[i] = ip;
        pb = o1 - ml * r1;
        pc = o2 - ml * r2;
        pf = 0.0;
      }
      ipiv[N - 1] = 1.0 / (fabs(pb) >= 2.2e-16 ? pb : (pb >= 0.0 ? 2.2e-16 : -2.2e-16));
    }
    double y[N];
#pragma unroll
    for (int i = 0; i < N; ++i) y[i] = 1.0 + 0.125 * (double)((i * 7 + m * 3) % 5);
    for (int pass = 0; pass < 3; ++pass) {
      // orthogonalise against the vectors found before (twice), normalise
      for (int rep = 0; rep < 2; ++rep)
        for (int j = 0; j < m; ++j) {
          double dot = 0.0;
#pragma unroll
          for (int i = 0; i < N; ++i) dot += vecs[j][i] * y[i];
#pragma unroll
          for (int i = 0; i < N; ++i) y[i] -= dot * vecs[j][i];
        }
      double n2 = 0.0;
#pragma unroll
      for (int i = 0; i < N; ++i) n2 += y[i] * y[i];
      const double inv = rsqrt(n2);
#pragma unroll
      for (int i = 0; i < N; ++i) y[i] *= inv;
      if (pass == 2) break;
      // solve (T - lam I) y' = y with the factors: the row swaps and
      // eliminations on y, then back substitution
      double py = y[0];
#pragma unroll
      for (int i = 0; i < N - 1; ++i) {
        const double ny = y[i + 1];
        const double ry = swp[i] ? ny : py, oy = swp[i] ? py : ny;
        y[i] = ry;
        py = oy - mlt[i] * ry;
      }
      y[N - 1] = py;
#pragma unroll
      for (int i = N - 1; i >= 0; --i) {
        double t = y[i];
        if (i + 1 < N) t -= u1[i] * y[i + 1];
        if (i + 2 < N) t -= u2[i] * y[i + 2];
        y[i] = t * ipiv[i];
      }
    }
    // map back, v = H_0 H_1 ... H_{N-3} y
#pragma unroll
    for (int i = 0; i < N; ++i) vecs[m][i] = y[i];
#pragma unroll
    for (int k = N - 3; k >= 0; --k) {
      double t = 0.0;
#pragma unroll
      for (int i = k + 1; i < N; ++i) t += stash[(RS + refl(k, i)) * stride] * y[i];
      t *= stash[(BS + k) * stride];
#pragma unroll
      for (int i = k + 1; i < N; ++i) y[i] -= t * stash[(RS + refl(k, i)) * stride];
    }
    // -- 4. A += w v v^T on the stashed original, mode by mode -----------------
    if (live) {
      const double l = lam * g;  // original scale
      const double w = method == 1 ? -2.0 * l : -l;
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = i; j < N; ++j) stash[utri<N>(i, j) * stride] += w * y[i] * y[j];
    }
  }
#pragma unroll
  for (int i = 0; i < KS; ++i) a[i] = stash[i * stride];
}

}  // namespace ys
