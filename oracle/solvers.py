"""Linear solvers of the hot path, restated in FP64 NumPy (oracle only)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .projection import diagonal_block_pseudo_inverse


def block_jacobi_apply(inverse_blocks: np.ndarray, x: np.ndarray, counts, sizes) -> np.ndarray:
  """``z = D^-1 x`` per variable block (``PKG/kernel/Solver/solverKernel.pyx:282-323``)."""
  z = np.empty_like(x)
  seg = dstart = 0
  for n, s in zip(counts, sizes):
    inv = inverse_blocks[dstart:dstart + n * s * s].reshape(n, s, s)
    z[seg:seg + n * s] = np.einsum("bij,bj->bi", inv, x[seg:seg + n * s].reshape(n, s)).ravel()
    seg += n * s
    dstart += n * s * s
  return z


def diagonal_inverse(diag_blocks: np.ndarray, counts, sizes) -> np.ndarray:
  """Per-attribute pseudo-inverse of the diagonal blocks (``diagonalBlockInverseKernel.pyx:201-215``)."""
  out = np.empty_like(diag_blocks)
  dstart = 0
  for n, s in zip(counts, sizes):
    if n:
      out[dstart:dstart + n * s * s] = diagonal_block_pseudo_inverse(
          diag_blocks[dstart:dstart + n * s * s].reshape(n, s, s)).ravel()
    dstart += n * s * s
  return out


@dataclass
class JacobiResult:
  status: int
  iterations: int
  solution: np.ndarray
  delta_new: float


def jacobi_pcg(matvec, rhs, inverse_blocks, counts, sizes, threshold, max_iterations,
               initial_guess=None, zero_initial_guess=True) -> JacobiResult:
  """Block-Jacobi PCG with the reference's recurrence and return codes.

  Restates ``computeSolution`` (``PKG/kernel/Solver/solverKernel.pyx:534-686``):
  stop when ``r^T M^-1 r <= threshold * delta_0`` (a squared, preconditioned
  ratio); return ``0`` when already converged, the iteration count on
  convergence, ``-4`` when the budget runs out, ``-(it + 4)`` on a
  non-positive curvature or recurrence value, ``-5`` on an invalid initial
  residual.
  """
  g = np.asarray(rhs, dtype=np.float64)
  prec = lambda v: block_jacobi_apply(inverse_blocks, v, counts, sizes)
  if zero_initial_guess:
    x = np.zeros_like(g)
    r = g.copy()
    c = prec(g)
    delta0 = float(c @ g)
    delta_new = delta0
  else:
    x = np.asarray(initial_guess, dtype=np.float64).copy()
    delta0 = float(prec(g) @ g)
    r = g - matvec(x)
    c = prec(r)
    delta_new = float(r @ c)
  if not (np.isfinite(delta0) and delta0 >= 0 and np.isfinite(delta_new) and delta_new >= 0):
    return JacobiResult(-5, 0, x, delta_new)
  tol = threshold * delta0
  if not (np.isfinite(tol) and tol >= 0):
    return JacobiResult(-5, 0, x, delta_new)
  if delta_new <= tol:
    return JacobiResult(0, 0, x, delta_new)
  for it in range(1, max_iterations + 1):
    q = matvec(c)
    den = float(c @ q)
    delta_old = delta_new
    if not np.isfinite(den) or den <= 0.0:
      return JacobiResult(-it - 4, it, x, delta_new)
    alpha = delta_new / den
    x = x + c * alpha
    r = r - q * alpha
    s = prec(r)
    delta_new = float(r @ s)
    if not np.isfinite(delta_new) or delta_new < 0.0 or not np.isfinite(delta_old) or delta_old <= 0.0:
      return JacobiResult(-it - 4, it, x, delta_new)
    beta = delta_new / delta_old
    converged = delta_new <= tol
    c = s + c * beta
    if converged:
      return JacobiResult(it, it, x, delta_new)
  return JacobiResult(-4, max_iterations, x, delta_new)


@dataclass
class PCGResult:
  solution: np.ndarray
  iterations: int
  relative_residual: float
  converged: bool
  breakdown: str | None = None


def mas_pcg(matvec, rhs, precondition, tolerance, max_iterations, initial_guess=None,
            restart=False) -> PCGResult:
  """MAS-preconditioned CG (``PKG/solver/mas/pcg.py:23-102``).

  Stops when ``r^T z <= tolerance * reference`` with ``reference = r_0^T z_0``
  for a zero initial guess (``rhs^T M^-1 rhs`` otherwise).

  ``restart=True`` follows the reference's device loop instead of its NumPy
  one on a finite non-positive curvature (``mas/cuda/pcg.cu:183-189,
  236-240``): a zero step, then the direction restarts from ``M^-1 r``
  (beta = 0); the iteration counts.  The NumPy loop ends the solve there.
  """
  rhs = np.asarray(rhs, dtype=np.float64).reshape(-1)
  x = np.zeros_like(rhs) if initial_guess is None else np.asarray(initial_guess, dtype=np.float64).copy()
  residual = rhs - matvec(x)
  denom = max(float(np.linalg.norm(rhs)), np.finfo(np.float64).tiny)
  z = precondition(residual)
  rz = float(residual @ z)
  reference = rz if initial_guess is None else float(rhs @ precondition(rhs))
  if np.isfinite(rz) and rz >= 0 and np.isfinite(reference) and reference > 0 and rz <= tolerance * reference:
    return PCGResult(x, 0, float(np.linalg.norm(residual)) / denom, True)
  if max_iterations == 0:
    return PCGResult(x, 0, float(np.linalg.norm(residual)) / denom, False)
  if not np.isfinite(rz) or rz <= 0 or not np.isfinite(reference) or reference <= 0:
    return PCGResult(x, 0, float(np.linalg.norm(residual)) / denom, False, "preconditioner is not positive definite")
  direction = z.copy()
  for it in range(1, max_iterations + 1):
    product = matvec(direction)
    curvature = float(direction @ product)
    restarted = restart and np.isfinite(curvature) and curvature <= 0
    if not restarted and (not np.isfinite(curvature) or curvature <= 0):
      return PCGResult(x, it - 1, float(np.linalg.norm(residual)) / denom, False, "matrix is not positive definite")
    alpha = 0.0 if restarted else rz / curvature
    x += alpha * direction
    residual -= alpha * product
    z = precondition(residual)
    next_rz = float(residual @ z)
    rel = float(np.linalg.norm(residual)) / denom
    if not np.isfinite(next_rz) or next_rz < 0:
      return PCGResult(x, it, rel, False, "preconditioner is not positive definite")
    if next_rz <= tolerance * reference:
      return PCGResult(x, it, rel, True)
    if next_rz == 0.0:
      return PCGResult(x, it, rel, False, "preconditioner is not positive definite")
    direction = z + (0.0 if restarted else next_rz / rz) * direction
    rz = next_rz
  return PCGResult(x, max_iterations, float(np.linalg.norm(residual)) / denom, False)


def relative_residual(matvec, rhs, x) -> float:
  """True FP64 2-norm ratio ``||g - H x|| / ||g||``."""
  r = np.asarray(rhs) - matvec(np.asarray(x))
  return float(np.linalg.norm(r) / max(np.linalg.norm(rhs), np.finfo(np.float64).tiny))
