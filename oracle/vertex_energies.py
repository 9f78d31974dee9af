"""Vertex-tuple energies of the mixed scenes (oracle; test infrastructure only).

Float64 restatements of the reference example formulas, differentiated by
torch autograd on the CPU (the reference validates its energies with
float64 PyTorch and SymPy scripts the same way):

* barriers ``point_point`` / ``point_edge`` / ``point_triangle`` /
  ``edge_edge``: ``examples/dropping_in_container_mixed/helpers.py:143-199``;
* ``bending``: ``helpers.py:213-234`` (the half-angle ``atan2`` form);
* ``baraff_witkin`` and its rest frame ``compute_rest_shape``:
  ``helpers.py:240-292``;
* lagged point-triangle friction: ``examples/dropping_in_container/
  friction_helpers.py:12-66`` (smoothing) and ``:73-182`` (point-triangle);
* a StVK membrane on the Baraff-Witkin rest frame (the reference ships none:
  parity unpinned for it).

Each function takes ``x`` (and ``rest``) as ``[A, 3]`` tensors of one element
and returns the scalar energy; :func:`energy_grad_hess` batches the
gradient and Hessian over elements.
"""

from __future__ import annotations

import numpy as np


def _t():
  import torch
  return torch


def _barrier(d, dhat, kappa):
  torch = _t()
  i5 = d / dhat
  lenE = d - dhat
  l = torch.log(i5)
  return kappa * lenE * lenE * l * l


def point_point(x, rest, p):
  d = (x[1] - x[0]).dot(x[1] - x[0])
  return _barrier(d, p[0], p[1])


def point_edge(x, rest, p):
  torch = _t()
  c = torch.linalg.cross(x[1] - x[0], x[2] - x[0])
  d = c.dot(c) / (x[2] - x[1]).dot(x[2] - x[1])
  return _barrier(d, p[0], p[1])


def point_triangle(x, rest, p):
  torch = _t()
  b = torch.linalg.cross(x[2] - x[1], x[3] - x[1])
  atb = (x[0] - x[1]).dot(b)
  return _barrier(atb * atb / b.dot(b), p[0], p[1])


def edge_edge(x, rest, p):
  torch = _t()
  b = torch.linalg.cross(x[1] - x[0], x[3] - x[2])
  atb = (x[2] - x[0]).dot(b)
  return _barrier(atb * atb / b.dot(b), p[0], p[1])


def _angle(v, w, axis):
  torch = _t()
  return 2.0 * torch.atan2(torch.linalg.cross(v, w).dot(axis) / torch.linalg.norm(axis),
                           v.dot(w) + torch.linalg.norm(v) * torch.linalg.norm(w))


def _edge_theta(q0, q1, q2, q3):
  torch = _t()
  n0 = torch.linalg.cross(q0 - q2, q1 - q2)
  n1 = torch.linalg.cross(q1 - q3, q0 - q3)
  return _angle(n0, n1, q1 - q0)


def bending(x, rest, p):
  torch = _t()
  t = _edge_theta(x[0], x[1], x[2], x[3])
  t0 = _edge_theta(rest[0], rest[1], rest[2], rest[3])
  return p[0] * (t - t0) * (t - t0) * torch.linalg.norm(rest[1] - rest[0]) * p[1] * p[1]


def compute_rest_shape(v0, v1, v2):
  """2x2 rest shape matrix (``helpers.py:240-270``)."""
  torch = _t()
  n = torch.linalg.cross(v1 - v0, v2 - v0)
  n = n / torch.linalg.norm(n)
  target = torch.tensor([0.0, 1.0, 0.0], dtype=v0.dtype)
  vec = torch.linalg.cross(n, target)
  cos = n.dot(target)
  cv = torch.stack([torch.stack([vec[0] * 0, -vec[2], vec[1]]), torch.stack([vec[2], vec[0] * 0, -vec[0]]),
                    torch.stack([-vec[1], vec[0], vec[0] * 0])])
  rot = torch.eye(3, dtype=v0.dtype) + cv + cv @ cv / (1.0 + cos)
  uv = [torch.stack([(rot @ v)[0], (rot @ v)[2]]) for v in (v0, v1, v2)]
  a, b = uv[1] - uv[0], uv[2] - uv[0]
  return torch.stack([torch.stack([a[0], b[0]]), torch.stack([a[1], b[1]])])


def _membrane_f(x, rest):
  torch = _t()
  f = torch.stack([x[1] - x[0], x[2] - x[0]], dim=1)  # 3x2, columns x10, x20
  return f @ torch.linalg.inv(compute_rest_shape(rest[0], rest[1], rest[2]))


def _rest_area(rest):
  torch = _t()
  return torch.linalg.norm(torch.linalg.cross(rest[1] - rest[0], rest[2] - rest[0])) / 2.0


def baraff_witkin(x, rest, p):
  torch = _t()
  stretch_s, shear_s, thickness, dt = p
  f = _membrane_f(x, rest)
  i6 = f[:, 0].dot(f[:, 1])
  i5u, i5v = torch.linalg.norm(f[:, 0]), torch.linalg.norm(f[:, 1])
  uc = 0.01 if float(i5u.detach()) < 1.0 else 1.0
  vc = 0.01 if float(i5v.detach()) < 1.0 else 1.0
  stretch = uc * (i5u - 1.0) ** 2 + vc * (i5v - 1.0) ** 2
  return (stretch_s * stretch + shear_s * i6 * i6) * thickness * _rest_area(rest) * dt * dt


def stvk_membrane(x, rest, p):
  mu, lam, thickness, dt = p
  f = _membrane_f(x, rest)
  e00 = 0.5 * (f[:, 0].dot(f[:, 0]) - 1.0)
  e11 = 0.5 * (f[:, 1].dot(f[:, 1]) - 1.0)
  e01 = 0.5 * f[:, 0].dot(f[:, 1])
  psi = mu * (e00 * e00 + e11 * e11 + 2.0 * e01 * e01) + 0.5 * lam * (e00 + e11) ** 2
  return psi * thickness * _rest_area(rest) * dt * dt


def friction_pt(x, rest, p, lagged):
  """``friction_energy_pt`` with the lagged (beta1, beta2, t0, t1, lambda)."""
  torch = _t()
  fdhat, dt, rate = p
  b1, b2 = lagged[0], lagged[1]
  t0, t1, lam = lagged[2:5], lagged[5:8], lagged[8]
  dx = x - rest
  rel = dx[0] - (dx[1] + b1 * (dx[2] - dx[1]) + b2 * (dx[3] - dx[1]))
  u0, u1 = t0.dot(rel), t1.dot(rel)
  y2 = u0 * u0 + u1 * u1
  eps = np.sqrt(fdhat) * dt
  fric_dhat = fdhat * dt * dt
  y = torch.sqrt(y2 + 1e-16)
  if float(y2.detach()) > fric_dhat:
    phi = y
  else:
    phi = eps / 3.0 + y2 / eps - y2 * y / (3.0 * eps * eps)
  return rate * lam * phi


def lagged_friction_pt(x_old, dhat, kappa):
  """Lagged data of a point-triangle pair at the start of the step
  (``closest_point_coord_and_tangent_basis_pt``, ``lambda_last_h_pt``,
  ``friction_helpers.py:73-141``): (beta1, beta2, tangent0, tangent1, lambda)."""
  p, t0, t1, t2 = (np.asarray(v, dtype=np.float64) for v in x_old)
  e01, e02 = t1 - t0, t2 - t0
  B = np.stack([e01, e02], axis=1)
  beta = np.linalg.inv(B.T @ B) @ B.T @ (p - t0)
  tan0 = e01 / np.linalg.norm(e01)
  c = np.cross(np.cross(e01, e02), e01)
  tan1 = c / np.linalg.norm(c)
  q = t0 + beta[0] * e01 + beta[1] * e02
  d2 = (p - q) @ (p - q)
  i5log = np.log(d2 / dhat)
  lenE = d2 - dhat
  inner = i5log * i5log * (2.0 * d2 - 2.0 * dhat) + 2.0 * i5log * lenE * lenE / d2
  lam = -kappa * 2.0 * np.sqrt(d2) * inner
  return np.concatenate([beta, tan0, tan1, [lam]])


KINDS = {1: point_point, 2: point_edge, 3: point_triangle, 4: edge_edge, 5: bending, 6: baraff_witkin,
         7: stvk_membrane, 8: friction_pt}


def energy_grad_hess(kind, x, rest, params, lagged=None):
  """Energy [n], gradient [n, 3A] and Hessian [n, 3A, 3A] of ``n`` elements.

  ``x``, ``rest``: [n, A, 3]; ``params``: the scalar parameters of the kind;
  ``lagged``: [n, 9] for friction.
  """
  torch = _t()
  fn = KINDS[kind]
  x = np.asarray(x, dtype=np.float64)
  n, arity = x.shape[0], x.shape[1]
  rest = np.zeros_like(x) if rest is None else np.asarray(rest, dtype=np.float64)
  e = np.zeros(n)
  g = np.zeros((n, 3 * arity))
  h = np.zeros((n, 3 * arity, 3 * arity))
  for t in range(n):
    r = torch.tensor(rest[t])
    lag = None if lagged is None else torch.tensor(np.asarray(lagged[t], dtype=np.float64))

    def f(v):
      xx = v.reshape(arity, 3)
      return fn(xx, r, params) if lag is None else fn(xx, r, params, lag)

    v = torch.tensor(x[t].reshape(-1))
    e[t] = float(f(v))
    g[t] = torch.autograd.functional.jacobian(f, v).numpy()
    h[t] = torch.autograd.functional.hessian(f, v).numpy()
  return e, g, 0.5 * (h + np.transpose(h, (0, 2, 1)))
