"""Energies of affine (ABD) bodies (oracle; test infrastructure only).

Float64 restatements of the reference's affine-body terms, differentiated by
torch autograd on the CPU with respect to the body's 12 coordinates in the
reference's order: the 9 entries of the affine matrix A (row-major, the
``affine_matrices`` attribute of
``examples/dropping_in_container_mixed/dropping_in_container.py:241-245``)
followed by the translation t (``:243``).

* :func:`orthogonality` -- ``affine_energy`` (``examples/dropping_in_container_mixed/
  helpers.py:201-211``): ``1/2 sum_rows |row(A^T A - I)|^2``, times a stiffness;
* :func:`inertia` -- ``inertia`` (``helpers.py:138-141``) of a vertex at
  ``x = A xbar + t`` (``dropping_in_container.py:261-270``, ``:378``);
* :func:`snh` -- ``stable_neo_hookean_modified`` (``helpers.py:129-136``) on
  the tet positions ``xbar A^T + t`` (``dropping_in_container.py:280-320``,
  ``:370``); :func:`snh_projected` with the reference's projection (in the
  vertex positions, then mapped to the body coordinates).

:func:`grad_hess` batches the gradient and Hessian over elements.
"""

from __future__ import annotations

import numpy as np


def _t():
  import torch
  return torch


def orthogonality(q, data, stiffness):
  torch = _t()
  a = q[:9].reshape(3, 3)
  diff = a.T @ a - torch.eye(3, dtype=q.dtype)
  return stiffness * 0.5 * (diff[0].dot(diff[0]) + diff[1].dot(diff[1]) + diff[2].dot(diff[2]))


def inertia(q, data, params):
  """data: xbar (3), x_before (3), velocity (3), mass (1); params: dt, gravity (3)."""
  torch = _t()
  a, t = q[:9].reshape(3, 3), q[9:12]
  xbar, xb, v, m = data[0:3], data[3:6], data[6:9], data[9]
  dt = params[0]
  g = torch.as_tensor(params[1:4], dtype=q.dtype)
  x = a @ xbar + t
  xt = xb + v * dt + g * dt * dt
  return 0.5 * m * (x - xt).dot(x - xt)


def snh(q, data, params):
  """data: the 4 body-frame rest positions (12); params: mu, lam, dt."""
  torch = _t()
  a, t = q[:9].reshape(3, 3), q[9:12]
  rest = data[:12].reshape(4, 3)
  mu, lam, dt = params
  pos = rest @ a.T + t[None, :]
  tb = torch.stack([rest[1] - rest[0], rest[2] - rest[0], rest[3] - rest[0]])
  f = torch.stack([pos[1] - pos[0], pos[2] - pos[0], pos[3] - pos[0]])
  ib = torch.linalg.inv(tb.T)
  vol = torch.linalg.det(tb.T) / 6.0
  fi = f.T @ ib
  j = torch.linalg.det(fi)
  ic = torch.trace(fi.T @ fi)
  i3 = ic + 1.0
  alpha = 1.0 + 0.75 * mu / lam
  return vol * (0.5 * mu * (ic - 3.0) - 0.5 * mu * torch.log(i3) + 0.5 * lam * ((j - alpha) * (j - alpha))) * dt * dt


def snh_projected(q, rest, params, method):
  """Energies, gradients [n, 12] and Hessians [n, 12, 12] of the affine SNH in
  the body coordinates with the reference's projection: the energy's
  argument is the tetrahedron's gathered vertex positions ``xbar A^T + t``,
  linear in the body coordinates, so the 12x12 Hessian with respect to the
  positions is projected and mapped by J = dx/dq
  (``PKG/differentiator/differentiator.pyx:795-799``)."""
  from . import energies, projection
  q = np.asarray(q, dtype=np.float64)
  rest = np.asarray(rest, dtype=np.float64).reshape(len(q), 4, 3)
  mu, lam, dt = params
  a = q[:, :9].reshape(-1, 3, 3)
  t = q[:, 9:12]
  x = np.einsum("nkc,nrc->nkr", rest, a) + t[:, None, :]
  e, gx, hx = energies.snh_from_rest(x, rest, mu, lam, dt)
  if method >= 1:
    hx = projection.project_spd(hx, method)
  J = np.zeros((len(q), 12, 12))  # row 3k + r: xbar_k at columns 3r .. 3r + 2, 1 at 9 + r
  for k in range(4):
    for r in range(3):
      J[:, 3 * k + r, 3 * r:3 * r + 3] = rest[:, k]
      J[:, 3 * k + r, 9 + r] = 1.0
  g = np.einsum("nij,ni->nj", J, gx)
  h = np.einsum("nia,nij,njb->nab", J, hx, J)
  return e, g, h


def grad_hess(fn, q, data, params, size=12):
  """Energies [n], gradients [n, size], Hessians [n, size, size] of ``fn`` at
  the body coordinates ``q`` [n, >= size] with per-element ``data``."""
  torch = _t()
  q = np.asarray(q, dtype=np.float64)
  data = np.asarray(data, dtype=np.float64)
  n = q.shape[0]
  e, g, h = np.zeros(n), np.zeros((n, size)), np.zeros((n, size, size))
  for i in range(n):
    qi = torch.tensor(q[i, :size], dtype=torch.float64)
    di = torch.tensor(data[i], dtype=torch.float64)
    f = lambda v: fn(v, di, params)
    val = f(qi.clone().requires_grad_(True))
    e[i] = float(val.detach())
    g[i] = torch.autograd.functional.jacobian(f, qi).numpy()
    h[i] = torch.autograd.functional.hessian(f, qi).numpy()
  return e, g, h
