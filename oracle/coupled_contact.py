"""Contact through affine-body vertices (oracle; test infrastructure only).

Restates how the reference differentiates a contact pair whose vertices come
from the collision union ``[soft, abd, container]`` of
``examples/dropping_in_container_mixed/dropping_in_container.py:344``, where
an abd vertex sits at ``x = A xbar + t`` (``:270``): the leaves of a plain
vertex are its position, those of an abd vertex its body's A (three rows
here, the reference's 9 entries in the same row-major order) and t.

The map from the leaves to the gathered vertex positions is linear, so the
second-order chain term vanishes and the reference projects the *inner*
Hessian -- the one with respect to the pair's vertex positions, 3V x 3V,
with the reference's PSD test and eigen-projection -- and then forms
``J^T proj(H) J`` (``PKG/differentiator/differentiator.pyx:795-799``,
``project_entire_hessian = False``; its own GPU test expects exactly
``J^T _project(H_inner) J`` for linear JOIN/UNION maps,
``tests/differentiator/test_hessian_sparsity_permutation_gpu.py:150,216,269``).
Repeated leaves (two vertices of one body) add up in the columns of J.
"""

from __future__ import annotations

import numpy as np

from oracle import projection
from oracle import vertex_energies as ve


def slot_codes(verts, plain_code, body_codes):
  """Slot codes [4V] of one element (four slots a vertex).

  ``verts``: per vertex ``("p", index)`` or ``("a", body)``; ``plain_code(index)``
  gives the code of a plain vertex's position, ``body_codes(body)`` the four
  codes (A rows, t) of a body."""
  out = []
  for kind, i in verts:
    out.extend([plain_code(i), 0, 0, 0] if kind == "p" else list(body_codes(i)))
  return np.asarray(out, dtype=np.int64)


def local_compressed(kind, verts, codes, params, method, lagged=None, rest=None):
  """Energy and the compressed gradient / Hessian of one element.

  ``verts``: per vertex ``("p", x[3])`` or ``("a", A[9], t[3], xbar[3], ...)``;
  ``codes``: [4V].  The vertex-space Hessian is projected (``method``), then
  mapped through the merged leaf Jacobian of :func:`jacobian`.  ``rest`` and
  ``lagged`` feed the friction kinds (positions at the start of the step and
  the lagged data).  Returns ``(e, codes_c, sizes_c, g_c, H_c)``: repeated
  target codes become padding (code 0, size 0) in ``codes_c``; ``g_c`` and
  ``H_c`` follow the kept slots in first-occurrence order."""
  x = _positions(verts)
  e, g_x, h_x = ve.energy_grad_hess(kind, x[None], None if rest is None else np.asarray(rest)[None], params,
                                    None if lagged is None else np.asarray(lagged)[None])
  h_x = h_x[0]
  if method >= 1:
    h_x = projection.project_spd(h_x, method)
  J = jacobian(verts, codes)
  g_c = J.T @ g_x[0]
  h_c = J.T @ h_x @ J
  codes_c = np.zeros(len(codes), dtype=np.int64)
  sizes_c = np.zeros(len(codes), dtype=np.int64)
  seen = set()
  for k, c in enumerate(np.asarray(codes, dtype=np.int64)):
    if c == 0 or (c >= 2 and c in seen):
      continue
    seen.add(int(c))
    codes_c[k] = c
    sizes_c[k] = 3
  return float(e[0]), codes_c, sizes_c, g_c, h_c


def _positions(verts):
  xs = []
  for d in verts:
    if d[0] == "p":
      xs.append(np.asarray(d[1], dtype=np.float64))
    else:
      xs.append(np.asarray(d[1], dtype=np.float64).reshape(3, 3) @ np.asarray(d[3], dtype=np.float64) +
                np.asarray(d[2], dtype=np.float64))
  return np.asarray(xs)


def jacobian(verts, codes):
  """Jhat [3V, 3 * kept] of the merged leaves (vertex coordinates <- leaves),
  columns in first-occurrence slot order as in :func:`local_compressed`."""
  cols = []
  first = {}
  blocks = []  # (vertex, column, 3x3)
  for v, d in enumerate(verts):
    for s in range(4):
      c = int(codes[4 * v + s])
      if c == 0:
        continue
      if c >= 2 and c in first:
        col = first[c]
      else:
        col = len(cols)
        cols.append(c)
        if c >= 2:
          first[c] = col
      if d[0] == "p" or s == 3:
        j = np.eye(3)
      else:
        j = np.zeros((3, 3))
        j[s] = d[3]
      blocks.append((v, col, j))
  J = np.zeros((3 * len(verts), 3 * len(cols)))
  for v, col, j in blocks:
    J[3 * v:3 * v + 3, 3 * col:3 * col + 3] += j
  return J
