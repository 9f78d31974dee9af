"""Rectangular second-order Jacobians (oracle; test infrastructure only).

Restates the reference's rectangular Jacobian of a scalar energy,
``d2E / (d rows d cols)`` (``PKG/differentiator/differentiator.pyx:367-489``):
every (row slot, column slot) pair of an instance whose slots carry target
codes ``>= 2`` contributes the block of the instance's local second
derivative between those arguments
(``PKG/kernel/Coordinate/secondOrderJacobianIndicesKernel.pyx:16-84``), no
projection (``PKG/kernel/Jacobian/secondOrderJacobianKernelNoProject.pyx``);
repeated targets add up.  Dense, for small cases.
"""

from __future__ import annotations

import numpy as np


def dense(local_h, row_codes, col_codes, rows, cols):
  """Dense ``rows x cols`` matrix from local Hessians ``[n, 3A, 3A]`` and
  per-argument codes ``[n, A]`` (code - 2 = scalar start, < 2: no target)."""
  local_h = np.asarray(local_h, dtype=np.float64)
  row_codes = np.asarray(row_codes, dtype=np.int64)
  col_codes = np.asarray(col_codes, dtype=np.int64)
  J = np.zeros((rows, cols))
  n, A = row_codes.shape
  for t in range(n):
    for a in range(A):
      r = row_codes[t, a]
      if r < 2:
        continue
      for b in range(A):
        c = col_codes[t, b]
        if c < 2:
          continue
        J[r - 2:r + 1, c - 2:c + 1] += local_h[t, 3 * a:3 * a + 3, 3 * b:3 * b + 3]
  return J


def inertia_local(mass, dt, with_velocity=True):
  """Local Hessians of 1/2 m |x - x_before - dt v - dt^2 g|^2 over
  (x, x_before[, v]) (``examples/dropping_in_container_mixed/helpers.py:138-141``)."""
  c = np.array([1.0, -1.0, -dt])[:3 if with_velocity else 2]
  blk = np.kron(np.outer(c, c), np.eye(3))
  return np.asarray(mass, dtype=np.float64)[:, None, None] * blk[None]
