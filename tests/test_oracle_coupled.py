"""Contact through affine-body vertices, on the CPU.

The reference projects the Hessian of a pair with respect to its vertex
positions (3V x 3V) and maps it to the leaves (plain positions, body A rows
and t) through the linear Jacobian of x = A xbar + t, merging repeated
leaves: ``J^T proj(H) J``.  These tests check on random elements that the
oracle's unprojected result equals autograd in the leaves (the chain rule,
merged), that the projected one is ``J^T proj(H) J`` and positive
semidefinite, and that the projection is exercised.  Tolerance: 1e-11
relative to the largest entry.
"""

import numpy as np
import pytest

from oracle import coupled_contact as cc
from oracle import vertex_energies as ve

def rel(a, b):
  return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _element(kind, layout, rng):
  """Vertices of one element: layout entries 'p' (plain) or a body index."""
  bodies = {}
  verts = []
  for v, lab in enumerate(layout):
    if lab == "p":
      verts.append(("p", rng.uniform(-0.05, 0.05, 3) + 0.02 * v))
    else:
      if lab not in bodies:
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        bodies[lab] = ((q @ (np.eye(3) + rng.uniform(-0.05, 0.05, (3, 3)))).ravel(), rng.uniform(-0.02, 0.02, 3))
      A, t = bodies[lab]
      verts.append(("a", A, t, rng.uniform(-0.3, 0.3, 3), lab))
  return verts


def _codes(verts):
  plain = iter(range(100))
  out = []
  for d in verts:
    if d[0] == "p":
      out.extend([2 + 3 * next(plain), 0, 0, 0])
    else:
      b = d[4]
      out.extend([1000 + 12 * b + 3 * r for r in range(3)] + [2000 + 3 * b])
  return np.asarray(out, dtype=np.int64)


def _positions(verts):
  xs = []
  for d in verts:
    if d[0] == "p":
      xs.append(d[1])
    else:
      xs.append(d[1].reshape(3, 3) @ d[3] + d[2])
  return np.asarray(xs)


LAYOUTS = [
    (1, ["p", 0]), (1, [0, 1]), (2, ["p", 0, 0]), (2, [0, 1, 1]), (3, ["p", 0, 0, 0]), (3, [0, "p", "p", "p"]),
    (3, [0, 1, 1, 1]), (4, ["p", "p", 0, 0]), (4, [0, 0, 1, 1]), (4, [0, "p", 1, "p"]), (3, ["p", "p", "p", "p"]),
]


def _leaf_autograd(kind, verts, codes, params):
  """Gradient and Hessian by autograd directly in the leaves, repeated
  leaves merged (sum of their rows and columns)."""
  import torch
  fn = ve.KINDS[kind]
  slots = []
  for v, d in enumerate(verts):
    for s in range(4):
      k = 4 * v + s
      if codes[k] == 0:
        continue
      val = d[1] if d[0] == "p" else (d[1][3 * s:3 * s + 3] if s < 3 else d[2])
      slots.append((k, np.asarray(val, dtype=np.float64)))
  where = {k: i for i, (k, _) in enumerate(slots)}

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

  z0 = torch.tensor(np.concatenate([v for _, v in slots]))
  g = torch.autograd.functional.jacobian(f, z0).numpy()
  h = torch.autograd.functional.hessian(f, z0).numpy()
  first, owner, keep = {}, [], []
  for k, _ in slots:
    c = int(codes[k])
    if c >= 2 and c in first:
      owner.append(first[c])
      continue
    if c >= 2:
      first[c] = len(keep)
    owner.append(len(keep))
    keep.append(k)
  P = np.zeros((3 * len(slots), 3 * len(keep)))
  for i, o in enumerate(owner):
    P[3 * i:3 * i + 3, 3 * o:3 * o + 3] = np.eye(3)
  return P.T @ g, P.T @ h @ P


@pytest.mark.parametrize("kind,layout", LAYOUTS)
@pytest.mark.parametrize("method", [1, 2])
def test_inner_projection_through_the_leaf_jacobian(kind, layout, method):
  from oracle import projection
  rng = np.random.default_rng(7 + 13 * kind + len(layout) + 101 * method)
  projected = 0
  for trial in range(6):
    verts = _element(kind, layout, rng)
    codes = _codes(verts)
    x = _positions(verts)
    # barrier parameters (dHat, kappa): dHat above the element's squared distance, so the term is active
    dist = _squared_distance(kind, x)
    params = (2.5 * dist, 1.0)
    e0, g_x, h_x = ve.energy_grad_hess(kind, x[None], None, params)
    e, codes_c, sizes_c, g_c, h_c = cc.local_compressed(kind, verts, codes, params, method)
    J = cc.jacobian(verts, codes)
    assert abs(e - e0[0]) <= 1e-13 * abs(e0[0])
    g_leaf, h_leaf = _leaf_autograd(kind, verts, codes, params)
    assert rel(g_c, g_leaf) <= 1e-11
    _, _, _, _, h_raw = cc.local_compressed(kind, verts, codes, params, 0)
    assert rel(h_raw, h_leaf) <= 1e-11
    assert rel(h_c, J.T @ projection.project_spd(h_x[0], method) @ J) <= 1e-11
    assert np.linalg.eigvalsh(0.5 * (h_c + h_c.T)).min() >= -1e-9 * np.abs(h_c).max()
    projected += int(rel(h_c, h_raw) > 1e-9)
  assert projected >= 1, "no element reached the projection"


def _squared_distance(kind, x):
  import torch
  t = torch.tensor(x)
  if kind == 1:
    e = t[1] - t[0]
    return float(torch.dot(e, e))
  if kind == 2:
    c = torch.linalg.cross(t[1] - t[0], t[2] - t[0])
    e = t[2] - t[1]
    return float(torch.dot(c, c) / torch.dot(e, e))
  if kind == 3:
    b = torch.linalg.cross(t[2] - t[1], t[3] - t[1])
    return float(torch.dot(t[0] - t[1], b) ** 2 / torch.dot(b, b))
  b = torch.linalg.cross(t[1] - t[0], t[3] - t[2])
  return float(torch.dot(t[2] - t[0], b) ** 2 / torch.dot(b, b))


def test_slot_codes_follow_the_four_slot_layout():
  codes = cc.slot_codes([("p", 5), ("a", 1)], lambda i: 2 + 3 * i, lambda b: (100 + b, 200 + b, 300 + b, 400 + b))
  assert codes.tolist() == [17, 0, 0, 0, 101, 201, 301, 401]
