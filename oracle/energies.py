"""Element energies of the hot path, restated in FP64 NumPy (oracle only).

Every routine is vectorised over elements and returns the local gradient and
the *unprojected* local Hessian over the element's natural arguments in
argument-major order (argument a, component k -> row ``s*a + k``), which is
the order in which the reference's generated device functions lay out their
packed ``[upper H | g]`` result (``PKG/matrixAndVector/matrix/hessian.pyx:926-934``).
"""

from __future__ import annotations

import numpy as np

# Levi-Civita symbol eps[i, j, k].
_EPS = np.zeros((3, 3, 3))
for _i, _j, _k in ((0, 1, 2), (1, 2, 0), (2, 0, 1)):
  _EPS[_i, _j, _k] = 1.0
  _EPS[_i, _k, _j] = -1.0


def snh_rest_invariants(rest: np.ndarray):
  """Rest inverse edge matrix and signed volume of each tetrahedron.

  Follows ``examples/dropping_in_container_mixed/helpers.py:102-114``:
  ``TB`` has rows ``X1-X0, X2-X0, X3-X0``; ``vol = det(TB^T)/6`` (signed) and
  ``IB = (TB^T)^-1``.  Identical to ``precompute_rest_invariants`` in
  ``examples/backup/pytorch_energy_hessian_and_gradient/stable_neo_hookean.py:40-55``.
  """
  rest = np.asarray(rest, dtype=np.float64)
  dm = np.stack([rest[:, 1] - rest[:, 0], rest[:, 2] - rest[:, 0], rest[:, 3] - rest[:, 0]], axis=2)
  return np.linalg.inv(dm), np.linalg.det(dm) / 6.0


def snh_local(x: np.ndarray, ib: np.ndarray, vol: np.ndarray, mu, lam, dt: float = 1.0):
  """Stable Neo-Hookean energy, gradient (T,12) and Hessian (T,12,12).

  Energy (``examples/dropping_in_container_mixed/helpers.py:116-127``)::

      FI = F^T IB,  J = det FI,  IC = tr(FI^T FI)
      E  = vol * (mu/2 (IC-3) - mu/2 log(IC+1) + lam/2 (J - (1 + 3/4 mu/lam))^2) * dt^2

  Derivatives are the exact first and second derivatives of this expression
  with respect to the 12 gathered vertex coordinates (the reference obtains
  them symbolically, ``PKG/differentiator/differentiator.pyx:506-595``).
  """
  x = np.asarray(x, dtype=np.float64)
  t = x.shape[0]
  mu = np.broadcast_to(np.asarray(mu, dtype=np.float64), (t,))
  lam = np.broadcast_to(np.asarray(lam, dtype=np.float64), (t,))
  vol = np.broadcast_to(np.asarray(vol, dtype=np.float64), (t,))
  g = np.empty((t, 4, 3))
  g[:, 1:, :] = ib
  g[:, 0, :] = -ib.sum(axis=1)
  f = np.einsum("tak,taj->tkj", x, g)
  ic = np.einsum("tkj,tkj->t", f, f)
  j = np.linalg.det(f)
  cof = np.stack([np.cross(f[:, :, 1], f[:, :, 2]), np.cross(f[:, :, 2], f[:, :, 0]),
                  np.cross(f[:, :, 0], f[:, :, 1])], axis=2)
  alpha = 1.0 + 0.75 * mu / lam
  scale = vol * dt * dt
  energy = scale * (0.5 * mu * (ic - 3.0) - 0.5 * mu * np.log(ic + 1.0) + 0.5 * lam * (j - alpha) ** 2)
  c1 = mu * (1.0 - 1.0 / (ic + 1.0))
  c2 = 2.0 * mu / (ic + 1.0) ** 2
  c3 = lam * (j - alpha)
  p = c1[:, None, None] * f + (lam * (j - alpha))[:, None, None] * cof
  grad = scale[:, None, None] * np.einsum("tkj,taj->tak", p, g)
  eye = np.eye(3)
  hf = (c1[:, None, None, None, None] * np.einsum("kl,jm->kjlm", eye, eye)[None]
        + c2[:, None, None, None, None] * np.einsum("tkj,tlm->tkjlm", f, f)
        + lam[:, None, None, None, None] * np.einsum("tkj,tlm->tkjlm", cof, cof)
        + c3[:, None, None, None, None] * np.einsum("klp,jmq,tpq->tkjlm", _EPS, _EPS, f))
  hess = scale[:, None, None, None, None] * np.einsum("taj,tbm,tkjlm->takbl", g, g, hf)
  return energy, grad.reshape(t, 12), hess.reshape(t, 12, 12)


def snh_from_rest(x, rest, mu, lam, dt):
  """SNH with the rest invariants computed from rest positions per element."""
  ib, vol = snh_rest_invariants(rest)
  return snh_local(x, ib, vol, mu, lam, dt)


def inertia_local(x, x_tilde, mass):
  """Implicit-Euler inertia 1/2 (x - x~)^T m (x - x~) per vertex.

  Follows ``examples/dropping_in_container_mixed/helpers.py:138-141`` with a
  scalar lumped mass; ``x~`` is supplied by the caller (the reference builds
  it as ``x_before + v dt + gravity dt^2``).
  """
  x = np.asarray(x, dtype=np.float64)
  d = x - np.asarray(x_tilde, dtype=np.float64)
  m = np.broadcast_to(np.asarray(mass, dtype=np.float64), (x.shape[0],))
  energy = 0.5 * m * np.einsum("ti,ti->t", d, d)
  grad = m[:, None] * d
  hess = m[:, None, None] * np.eye(3)[None]
  return energy, grad, hess


def linear_quadratic_local(y, jac, offset, inner, linear, project=None):
  """Quadratic energy of a linear boundary map (the reference KAT energy).

  ``b = J y + o``, ``E = l^T b + 1/2 b^T H b``; gradient ``J^T (H b + l)`` and
  Hessian ``J^T P(H) J`` where ``P`` is the inner SPD projection applied by
  the reference when the boundary map is linear
  (``PKG/differentiator/differentiator.pyx:794-799``).  ``project`` maps a
  matrix to its projection (``None`` leaves it raw).
  """
  y = np.asarray(y, dtype=np.float64)
  b = y @ jac.T + offset
  energy = b @ linear + 0.5 * np.einsum("ti,ij,tj->t", b, inner, b)
  grad = (b @ inner.T + linear) @ jac
  h = inner if project is None else project(inner)
  hess = np.broadcast_to(jac.T @ h @ jac, (y.shape[0], jac.shape[1], jac.shape[1])).copy()
  return energy, grad, hess


def snh_hessian_with_rest(x, rest, mu, lam, dt):
  """Hessians [T, 24, 24] of the Stable Neo-Hookean energy (``helpers.py:116-127``)
  with respect to the tet's positions and its rest positions together
  (``[x (12), X (12)]``, argument-major), by torch autograd over the same
  expression (``FI = F^T IB`` with ``IB`` the inverse of the rest edge
  matrix, ``vol`` from the rest edges).  The position-position block equals
  :func:`snh_from_rest`'s Hessian."""
  import torch
  from torch.func import hessian, vmap
  x = torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, 12)))
  r = torch.from_numpy(np.ascontiguousarray(np.asarray(rest, dtype=np.float64).reshape(-1, 12)))
  t = x.shape[0]
  mu = torch.from_numpy(np.broadcast_to(np.asarray(mu, dtype=np.float64), (t,)).copy())
  lam = torch.from_numpy(np.broadcast_to(np.asarray(lam, dtype=np.float64), (t,)).copy())

  def det3(a):
    return (a[0, 0] * (a[1, 1] * a[2, 2] - a[1, 2] * a[2, 1]) - a[0, 1] * (a[1, 0] * a[2, 2] - a[1, 2] * a[2, 0])
            + a[0, 2] * (a[1, 0] * a[2, 1] - a[1, 1] * a[2, 0]))

  def inv3(a):
    c = torch.stack([torch.linalg.cross(a[:, 1], a[:, 2]), torch.linalg.cross(a[:, 2], a[:, 0]),
                     torch.linalg.cross(a[:, 0], a[:, 1])])   # rows: the inverse's rows times det
    return c / det3(a)

  def energy(z, m, l):
    p, q = z[:12].reshape(4, 3), z[12:].reshape(4, 3)
    dm = torch.stack([q[1] - q[0], q[2] - q[0], q[3] - q[0]], dim=1)   # columns: rest edges
    ds = torch.stack([p[1] - p[0], p[2] - p[0], p[3] - p[0]], dim=1)
    f = ds @ inv3(dm)
    ic = (f * f).sum()
    j = det3(f)
    alpha = 1.0 + 0.75 * m / l
    vol = det3(dm) / 6.0
    return vol * (0.5 * m * (ic - 3.0) - 0.5 * m * torch.log(ic + 1.0) + 0.5 * l * (j - alpha) ** 2) * dt * dt

  z = torch.cat([x, r], dim=1)
  h = vmap(hessian(energy))(z, mu, lam).numpy()
  return 0.5 * (h + np.transpose(h, (0, 2, 1)))


def snh_parameter_jacobian(x, rest, mu, lam, dt, which):
  """d(dE/dx)/d mu (``which`` 0) or d(dE/dx)/d lambda (1) of the Stable
  Neo-Hookean energy per tet, [T, 12], by torch autograd (forward over
  reverse) of the same expression as :func:`snh_hessian_with_rest`."""
  import torch
  from torch.func import grad, jacfwd, vmap
  x = torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, 12)))
  r = torch.from_numpy(np.ascontiguousarray(np.asarray(rest, dtype=np.float64).reshape(-1, 12)))
  t = x.shape[0]
  mu = torch.from_numpy(np.broadcast_to(np.asarray(mu, dtype=np.float64), (t,)).copy())
  lam = torch.from_numpy(np.broadcast_to(np.asarray(lam, dtype=np.float64), (t,)).copy())

  def energy(p12, q12, m, l):
    p, q = p12.reshape(4, 3), q12.reshape(4, 3)
    dm = torch.stack([q[1] - q[0], q[2] - q[0], q[3] - q[0]], dim=1)
    ds = torch.stack([p[1] - p[0], p[2] - p[0], p[3] - p[0]], dim=1)
    ib = torch.stack([torch.linalg.cross(dm[:, 1], dm[:, 2]), torch.linalg.cross(dm[:, 2], dm[:, 0]),
                      torch.linalg.cross(dm[:, 0], dm[:, 1])])
    det = (dm[:, 0] * ib[0]).sum()
    f = ds @ (ib / det)
    ic = (f * f).sum()
    j = (f[:, 0] * torch.linalg.cross(f[:, 1], f[:, 2])).sum()
    alpha = 1.0 + 0.75 * m / l
    return det / 6.0 * (0.5 * m * (ic - 3.0) - 0.5 * m * torch.log(ic + 1.0) + 0.5 * l * (j - alpha) ** 2) * dt * dt

  argnum = 2 if which == 0 else 3
  d = vmap(jacfwd(grad(energy, argnums=0), argnums=argnum))(x, r, mu, lam)
  return d.numpy()
