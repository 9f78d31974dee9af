"""Barriers through affine-body vertices (oracle; test infrastructure only).

Restates how the reference differentiates a contact pair whose vertices come
from the collision union ``[soft, abd, container]`` of
``examples/dropping_in_container_mixed/dropping_in_container.py:344``, where
an abd vertex sits at ``x = A xbar + t`` (``:270``): the leaves of a plain
vertex are its position, those of an abd vertex its body's A (three rows
here, the reference's 9 entries in the same row-major order) and t.  The
energy is differentiated with respect to every slot separately (torch
autograd, float64), the slots that repeat one leaf are merged by summing
their rows and columns (``PKG/kernel/Hessian/hessianKernelFullProject.pyx:95-131``),
and the compressed matrix is projected as a whole with the reference's PSD
test and eigen-projection (``:133-139``, :func:`oracle.projection.project_spd`)
-- up to 24x24 -- with no use of its low rank.

:func:`projected_via_gram` restates the device's route to the same matrix
(a 3V x 3V projection of ``L^T H L``, L the Cholesky factor of the vertices'
Gram matrix) so the two can be compared on the CPU.
"""

from __future__ import annotations

import numpy as np

from oracle import projection
from oracle import vertex_energies as ve


def _t():
  import torch
  return torch


def slot_codes(verts, plain_code, body_codes):
  """Slot codes [4V] of one element (four slots a vertex).

  ``verts``: per vertex ``("p", index)`` or ``("a", body)``; ``plain_code(index)``
  gives the code of a plain vertex's position, ``body_codes(body)`` the four
  codes (A rows, t) of a body."""
  out = []
  for kind, i in verts:
    out.extend([plain_code(i), 0, 0, 0] if kind == "p" else list(body_codes(i)))
  return np.asarray(out, dtype=np.int64)


def local_compressed(kind, verts, codes, params, method):
  """Energy and the compressed, projected gradient / Hessian of one element.

  ``verts``: per vertex ``("p", x[3])`` or ``("a", A[9], t[3], xbar[3])``;
  ``codes``: [4V].  Returns ``(e, codes_c, sizes_c, g_c, H_c)``: repeated
  target codes become padding (code 0, size 0) in ``codes_c``; ``g_c`` and
  ``H_c`` follow the kept slots in order."""
  torch = _t()
  fn = ve.KINDS[kind]
  slots = []  # (slot k, vertex, s, values)
  for v, d in enumerate(verts):
    for s in range(4):
      k = 4 * v + s
      if codes[k] == 0:
        continue
      if d[0] == "p":
        val = np.asarray(d[1], dtype=np.float64)
      else:
        val = np.asarray(d[1], dtype=np.float64)[3 * s:3 * s + 3] if s < 3 else np.asarray(d[2], dtype=np.float64)
      slots.append((k, v, s, val))
  where = {k: i for i, (k, _, _, _) in enumerate(slots)}

  def f(z):
    xs = []
    for v, d in enumerate(verts):
      if d[0] == "p":
        i = where[4 * v]
        xs.append(z[3 * i:3 * i + 3])
      else:
        xbar = torch.tensor(np.asarray(d[3], dtype=np.float64))
        rows = [z[3 * where[4 * v + r]:3 * where[4 * v + r] + 3] for r in range(3)]
        tt = z[3 * where[4 * v + 3]:3 * where[4 * v + 3] + 3]
        xs.append(torch.stack([torch.dot(rows[r], xbar) + tt[r] for r in range(3)]))
    x = torch.stack(xs)
    return fn(x, torch.zeros_like(x), params)

  z0 = torch.tensor(np.concatenate([sl[3] for sl in slots]))
  e = float(f(z0))
  g = torch.autograd.functional.jacobian(f, z0).numpy()
  h = torch.autograd.functional.hessian(f, z0).numpy()
  h = 0.5 * (h + h.T)
  # merge repeated target leaves into their first occurrence
  first = {}
  keep = []
  owner = np.zeros(len(slots), dtype=np.int64)
  for i, (k, _, _, _) in enumerate(slots):
    c = int(codes[k])
    if c >= 2 and c in first:
      owner[i] = first[c]
      continue
    if c >= 2:
      first[c] = len(keep)
    owner[i] = len(keep)
    keep.append(i)
  P = np.zeros((3 * len(slots), 3 * len(keep)))
  for i in range(len(slots)):
    P[3 * i:3 * i + 3, 3 * owner[i]:3 * owner[i] + 3] = np.eye(3)
  g_c = P.T @ g
  h_c = P.T @ h @ P
  if method >= 1:
    h_c = projection.project_spd(h_c, method)
  codes_c = np.zeros(len(codes), dtype=np.int64)
  sizes_c = np.zeros(len(codes), dtype=np.int64)
  for i in keep:
    k = slots[i][0]
    codes_c[k] = codes[k]
    sizes_c[k] = 3
  return e, codes_c, sizes_c, g_c, h_c


def gram_factor(verts):
  """Cholesky factor of the Gram matrix m (m_vw = xbar_v . xbar_w + 1 for two
  vertices of one body, 1 on a plain vertex's diagonal, 0 otherwise)."""
  V = len(verts)
  m = np.zeros((V, V))
  for v in range(V):
    for w in range(V):
      dv, dw = verts[v], verts[w]
      if v == w and dv[0] == "p":
        m[v, w] = 1.0
      elif dv[0] == "a" and dw[0] == "a" and dv[4] == dw[4]:
        m[v, w] = float(np.dot(dv[3], dw[3])) + 1.0
  return np.linalg.cholesky(m)


def projected_via_gram(h_x, verts, method):
  """Vertex-space Hessian h_x [3V, 3V] after the projection of its compressed
  form, by way of ``S = L^T h_x L``: ``h_x + L^-T (proj(S) - S) L^-1`` with
  ``L = chol(m) (x) I3``.  ``verts`` entries: ``("p",)`` or
  ``("a", A, t, xbar, body)``."""
  L = np.kron(gram_factor(verts), np.eye(3))
  S = L.T @ h_x @ L
  if projection.is_psd_reference(S):
    return h_x.copy()
  D = projection.project_spd(S, method) - S
  Li = np.linalg.inv(L)
  return h_x + Li.T @ D @ Li


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
