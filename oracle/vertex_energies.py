"""Vertex-tuple energies of the mixed scenes (oracle; test infrastructure only).

Float64 restatements of the reference example formulas, differentiated by
torch autograd on the CPU (the reference validates its energies with
float64 PyTorch and SymPy scripts the same way):

* barriers ``point_point`` / ``point_edge`` / ``point_triangle`` /
  ``edge_edge``: ``examples/dropping_in_container_mixed/helpers.py:143-199``;
* ``bending``: ``helpers.py:213-234`` (the half-angle ``atan2`` form);
* ``baraff_witkin`` and its rest frame ``compute_rest_shape``:
  ``helpers.py:240-292``;
* lagged friction of the four contact kinds: ``examples/dropping_in_container/
  friction_helpers.py:12-66`` (smoothing), ``:73-182`` (point-triangle),
  ``:188-276`` (point-edge), ``:283-405`` (edge-edge), ``:411-500``
  (point-point);
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
  # selects between float64 constants (python scalars would give float32)
  lo, one = i5u.new_tensor(0.01), i5u.new_tensor(1.0)
  uc = torch.where(i5u < 1.0, lo, one)
  vc = torch.where(i5v < 1.0, lo, one)
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


def _friction(rel, p, lagged):
  """``friction_energy_from_rel_dx`` with ``smooth_friction_phi``
  (``friction_helpers.py:26-66``): the lagged tangent basis (t0, t1) and
  lambda are ``lagged[2:5]``, ``lagged[5:8]``, ``lagged[8]``."""
  torch = _t()
  fdhat, dt, rate = p
  t0, t1, lam = lagged[2:5], lagged[5:8], lagged[8]
  u0, u1 = t0.dot(rel), t1.dot(rel)
  y2 = u0 * u0 + u1 * u1
  eps = np.sqrt(fdhat) * dt
  fric_dhat = fdhat * dt * dt
  y = torch.sqrt(y2 + 1e-16)
  # the branch as a select (both sides finite), so the formula batches
  phi = torch.where(y2 > fric_dhat, y, eps / 3.0 + y2 / eps - y2 * y / (3.0 * eps * eps))
  return rate * lam * phi


def friction_pt(x, rest, p, lagged):
  """``friction_energy_pt`` (``friction_helpers.py:124-182``) with the lagged
  (beta1, beta2, t0, t1, lambda); ``rest`` holds the positions of the last step."""
  b1, b2 = lagged[0], lagged[1]
  dx = x - rest
  return _friction(dx[0] - (dx[1] + b1 * (dx[2] - dx[1]) + b2 * (dx[3] - dx[1])), p, lagged)


def friction_pe(x, rest, p, lagged):
  """``friction_energy_pe`` (``friction_helpers.py:235-276``): lagged (eta, 0, t0, t1, lambda)."""
  eta = lagged[0]
  dx = x - rest
  return _friction(dx[0] - (dx[1] + eta * (dx[2] - dx[1])), p, lagged)


def friction_ee(x, rest, p, lagged):
  """``friction_energy_ee`` (``friction_helpers.py:355-405``): lagged (gamma1, gamma2, t0, t1, lambda)."""
  g1, g2 = lagged[0], lagged[1]
  dx = x - rest
  return _friction(dx[0] + g1 * (dx[1] - dx[0]) - dx[2] - g2 * (dx[3] - dx[2]), p, lagged)


def friction_pp(x, rest, p, lagged):
  """``friction_energy_pp`` (``friction_helpers.py:469-500``): lagged (0, 0, t0, t1, lambda)."""
  dx = x - rest
  return _friction(dx[0] - dx[1], p, lagged)


def _lambda_last_h(d2, dhat, kappa):
  """``lambda_last_h_rank2`` (``friction_helpers.py:12-23``)."""
  i5log = np.log(d2 / dhat)
  lenE = d2 - dhat
  inner = i5log * i5log * (2.0 * d2 - 2.0 * dhat) + 2.0 * i5log * lenE * lenE / d2
  return -kappa * 2.0 * np.sqrt(d2) * inner


def _unit(v):
  return v / np.linalg.norm(v)


def lagged_friction_pe(x_old, dhat, kappa):
  """(eta, 0, tangent0, tangent1, lambda) of a point-edge pair
  (``closest_point_coord_and_tangent_basis_pe``, ``lambda_last_h_pe``,
  ``friction_helpers.py:188-232``)."""
  p, e0, e1 = (np.asarray(v, dtype=np.float64) for v in x_old)
  edge = e1 - e0
  eta = (p - e0) @ edge / (edge @ edge)
  q = e0 + eta * edge
  d2 = (p - q) @ (p - q)
  return np.concatenate([[eta, 0.0], _unit(edge), _unit(np.cross(edge, p - e0)), [_lambda_last_h(d2, dhat, kappa)]])


def lagged_friction_ee(x_old, dhat, kappa):
  """(gamma1, gamma2, tangent0, tangent1, lambda) of an edge-edge pair
  (``closest_point_coord_and_tangent_basis_ee``, ``lambda_last_h_ee``,
  ``friction_helpers.py:283-352``)."""
  a0, a1, b0, b1 = (np.asarray(v, dtype=np.float64) for v in x_old)
  e20, e01, e23 = a0 - b0, a1 - a0, b1 - b0
  A = np.array([[e01 @ e01, -(e23 @ e01)], [-(e23 @ e01), e23 @ e23]])
  gamma = np.linalg.inv(A) @ np.array([-(e20 @ e01), e20 @ e23])
  r = (a0 + gamma[0] * e01) - (b0 + gamma[1] * e23)
  return np.concatenate([gamma, _unit(e01), _unit(np.cross(np.cross(e01, e23), e01)),
                         [_lambda_last_h(r @ r, dhat, kappa)]])


def lagged_friction_pp(x_old, dhat, kappa):
  """(0, 0, tangent0, tangent1, lambda) of a point-point pair
  (``closest_point_coord_and_tangent_basis_pp``, ``lambda_last_h_pp``,
  ``friction_helpers.py:411-466``)."""
  p0, p1 = (np.asarray(v, dtype=np.float64) for v in x_old)
  v = p1 - p0
  xc, yc = np.array([0.0, -v[2], v[1]]), np.array([v[2], 0.0, -v[0]])
  raw = xc if xc @ xc > yc @ yc else yc
  r = p0 - p1
  return np.concatenate([[0.0, 0.0], _unit(raw), _unit(np.cross(v, raw)), [_lambda_last_h(r @ r, dhat, kappa)]])


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
         7: stvk_membrane, 8: friction_pt, 9: friction_pe, 10: friction_ee, 11: friction_pp}
FRICTION_KINDS = (8, 9, 10, 11)
LAGGED = {8: lagged_friction_pt, 9: lagged_friction_pe, 10: lagged_friction_ee, 11: lagged_friction_pp}


def energy_grad_hess(kind, x, rest, params, lagged=None, chunk=16384):
  """Energy [n], gradient [n, 3A] and Hessian [n, 3A, 3A] of ``n`` elements.

  ``x``, ``rest``: [n, A, 3]; ``params``: the scalar parameters of the kind;
  ``lagged``: [n, 9] for friction.  The elements are differentiated in
  batches of ``chunk`` (``torch.func`` over the same formulas as
  :func:`energy_grad_hess_loop`, which takes them one at a time).
  """
  torch = _t()
  from torch.func import grad, hessian, vmap
  fn = KINDS[kind]
  x = np.asarray(x, dtype=np.float64)
  n, arity = x.shape[0], x.shape[1]
  rest = np.zeros_like(x) if rest is None else np.asarray(rest, dtype=np.float64)
  lag = np.zeros((n, 9)) if lagged is None else np.asarray(lagged, dtype=np.float64).reshape(n, -1)
  fric = kind in FRICTION_KINDS

  def f(v, r, lg):
    xx = v.reshape(arity, 3)
    return fn(xx, r, params, lg) if fric else fn(xx, r, params)

  e = np.zeros(n)
  g = np.zeros((n, 3 * arity))
  h = np.zeros((n, 3 * arity, 3 * arity))
  for a in range(0, n, chunk):
    b = min(n, a + chunk)
    v = torch.from_numpy(np.ascontiguousarray(x[a:b].reshape(b - a, -1)))
    r = torch.from_numpy(np.ascontiguousarray(rest[a:b]))
    lg = torch.from_numpy(np.ascontiguousarray(lag[a:b]))
    e[a:b] = vmap(f)(v, r, lg).numpy()
    g[a:b] = vmap(grad(f))(v, r, lg).numpy()
    h[a:b] = vmap(hessian(f))(v, r, lg).numpy()
  return e, g, 0.5 * (h + np.transpose(h, (0, 2, 1)))


def energy_grad_hess_loop(kind, x, rest, params, lagged=None):
  """:func:`energy_grad_hess` one element at a time (``torch.autograd.functional``)."""
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
