"""Contact through affine-body vertices, on the CPU.

The reference projects the compressed local Hessian of a pair (leaves of
plain vertices and of the bodies of abd vertices, repeated leaves merged) as
a whole, up to 24x24.  The device projects ``S = L^T H L`` (3V x 3V, L from
the Gram matrix of the element's body vertices) instead.  These tests check
on random elements that both routes give the same compressed matrix, that
the chain rule through ``x = A xbar + t`` matches autograd in the leaves,
and that the projection is exercised.  Tolerance: 1e-11 relative to the
largest entry.
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


@pytest.mark.parametrize("kind,layout", LAYOUTS)
@pytest.mark.parametrize("method", [1, 2])
def test_gram_route_matches_the_merged_projection(kind, layout, method):
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
    assert rel(J.T @ g_x[0], g_c) <= 1e-11
    _, _, _, _, h_raw = cc.local_compressed(kind, verts, codes, params, 0)
    assert rel(J.T @ h_x[0] @ J, h_raw) <= 1e-11
    via = J.T @ cc.projected_via_gram(h_x[0], verts, method) @ J
    assert rel(via, h_c) <= 1e-11
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
