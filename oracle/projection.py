"""SPD projection and diagonal-block pseudo-inverse rules (oracle only)."""

from __future__ import annotations

import numpy as np


def is_psd_reference(a: np.ndarray) -> np.ndarray:
  """Packed-Schur LDL^T PSD test, vectorised over a stack of matrices.

  Restates ``is_positive_semidefinite<N>`` of
  ``PKG/kernel/Hessian/hessianKernelHeader.pyx:79-141``: the scale is
  ``max(1, max |A_ii|)``, the tolerance ``1e-10 * scale``; a pivot below
  ``-tol`` fails, a pivot within ``tol`` requires its remaining column to be
  within ``tol``; otherwise the trailing lower triangle is updated with one
  reciprocal per column.  Only the lower triangle of ``a`` is read.
  """
  a = np.asarray(a, dtype=np.float64)
  squeeze = a.ndim == 2
  if squeeze:
    a = a[None]
  t, n, _ = a.shape
  schur = np.tril(a).copy()
  diag = np.abs(np.diagonal(schur, axis1=1, axis2=2))
  scale = np.maximum(1.0, diag.max(axis=1))
  tol = scale * 1.0e-10
  ok = np.ones(t, dtype=bool)
  for c in range(n):
    pivot = schur[:, c, c]
    ok &= ~(pivot < -tol)
    small = np.abs(pivot) <= tol
    if c + 1 < n:
      col = schur[:, c + 1:, c]
      bad_col = np.any(np.abs(col) > tol[:, None], axis=1)
      ok &= ~(small & bad_col)
      active = ~small
      inv = np.where(active, 1.0 / np.where(active, pivot, 1.0), 0.0)
      factor = col * inv[:, None]
      # schur[r, tc] -= factor[r] * schur[tc, c] for c < tc <= r
      upd = factor[:, :, None] * col[:, None, :]
      upd = np.tril(upd)
      upd[~active] = 0.0
      schur[:, c + 1:, c + 1:] -= upd
  return ok[0] if squeeze else ok


def project_spd(a: np.ndarray, method: int) -> np.ndarray:
  """Project a stack of symmetric matrices as the reference does.

  ``method`` follows ``scene.addEnergy(projection_method=...)``
  (``PKG/scene/scene.pyx:155-158``): ``<= 0`` leaves the matrix unchanged;
  ``1`` replaces negative eigenvalues by their absolute value; ``2`` by zero.
  Matrices that pass :func:`is_psd_reference` are returned unchanged
  (``hessianKernelHeader.pyx:200-203,229``).  1x1 matrices follow the scalar
  SPD code path (``PKG/codeGenerator/codeGenerator.pyx:816-818``).
  """
  a = np.array(a, dtype=np.float64, copy=True)
  squeeze = a.ndim == 2
  if squeeze:
    a = a[None]
  if method <= 0:
    return a[0] if squeeze else a
  n = a.shape[1]
  if n == 1:
    out = np.abs(a) if method == 1 else np.maximum(a, 0.0)
    return out[0] if squeeze else out
  psd = is_psd_reference(a)
  todo = np.flatnonzero(~psd)
  if todo.size:
    sym = a[todo]
    w, v = np.linalg.eigh(0.5 * (sym + np.swapaxes(sym, 1, 2)))
    w = np.abs(w) if method == 1 else np.where(w < 0.0, 0.0, w)
    a[todo] = np.einsum("tik,tk,tjk->tij", v, w, v)
  return a[0] if squeeze else a


def diagonal_block_pseudo_inverse(blocks: np.ndarray) -> np.ndarray:
  """Eigen pseudo-inverse used by the block-Jacobi preconditioner.

  ``PKG/kernel/Solver/diagonalBlockInverseKernel.pyx:69,91``: every
  eigenvalue maps to ``|l|`` when ``|l| < 1e-6`` and to ``|1/l|`` otherwise
  (blocks of size <= 4 are padded with identity, which leaves the leading
  block unchanged).
  """
  w, v = np.linalg.eigh(np.asarray(blocks, dtype=np.float64))
  inv = np.where(np.abs(w) < 1e-6, np.abs(w), np.abs(1.0 / np.where(w == 0.0, 1.0, w)))
  return np.einsum("tik,tk,tjk->tij", v, inv, v)
