"""The cloth-over-obstacle scene with affine bodies, matrix-free (oracle; test
infrastructure only).

Restates, term by term in FP64, the Newton system of the scene that
``yasps_b200.scenes.cloth_contact_scene`` builds -- the energies of
``examples/dropping_in_container_mixed/helpers.py`` (StVK membrane, dihedral
bending, IPC point-triangle and edge-edge barriers, inertia), the lagged
point-triangle friction of ``examples/dropping_in_container/friction_helpers.py``
and, with bodies, the affine-body terms of
``examples/dropping_in_container_mixed/dropping_in_container.py:241-395``
(vertex inertia through ``x = A xbar + t``, the orthogonality energy, and
body-cloth point-triangle barriers through the collision union
``[cloth, abd, obstacle]``, ``:344``).

Every element is differentiated with respect to its vertex positions (the
energy's argument), its Hessian projected there (method 1 for the cloth and
contact terms, none for inertia, method 2 for the orthogonality energy on A)
and mapped to the targets by the linear leaf Jacobian ``J``: a cloth vertex
is its own 3 coordinates, a body vertex ``dx = dA xbar + dt`` over the
body's 9 entries of A (row-major) and t, an obstacle vertex is no target
(``PKG/differentiator/differentiator.pyx:795-799``).  The system is never
assembled: ``g = sum_e J_e^T g_e`` and ``H x = sum_e J_e^T H_e J_e x``.

DoF order: the cloth positions, then A of every body (9 each), then t (3
each) -- the order of ``scene.minimizeEnergy``'s solution segments.
"""

from __future__ import annotations

import numpy as np

from oracle import affine_energies as ae
from oracle import energies as oe
from oracle import projection
from oracle import vertex_energies as ve


def _layout(cc):
  nc = len(cc.cloth_position)
  nb = 0 if cc.bodies is None else cc.bodies.num_bodies
  return nc, nb, 3 * nc, 3 * nc + 9 * nb, 3 * nc + 12 * nb


class _Vertices:
  """Vertex ids of a union mapped to their leaf Jacobians: ``kind`` 0 cloth,
  1 body vertex, 2 obstacle (no target)."""

  def __init__(self, cc, ids, union):
    nc, nb, a0, t0, _ = _layout(cc)
    ids = np.asarray(ids, dtype=np.int64)
    no = len(cc.obstacle)
    nbv = 0 if cc.bodies is None else len(cc.bodies.rest)
    self.kind = np.full(ids.shape, 2)
    self.index = np.zeros(ids.shape, dtype=np.int64)
    if union == "obstacle_cloth":
      cl = ids >= no
      self.kind[cl] = 0
      self.index[cl] = ids[cl] - no
    elif union == "cloth_abd_obstacle":
      cl = ids < nc
      bv = (ids >= nc) & (ids < nc + nbv)
      self.kind[cl] = 0
      self.index[cl] = ids[cl]
      self.kind[bv] = 1
      self.index[bv] = ids[bv] - nc
    else:  # cloth-local ids
      self.kind[:] = 0
      self.index = ids
    self.cc = cc
    self.a0, self.t0 = a0, t0

  def gather(self, v):
    """J v: the vertex displacements [..., 3] of the DoF vector ``v``."""
    out = np.zeros(self.kind.shape + (3,))
    cl, bv = self.kind == 0, self.kind == 1
    out[cl] = v[:self.a0].reshape(-1, 3)[self.index[cl]]
    if bv.any():
      b = self.cc.bodies.vertex_body[self.index[bv]]
      dA = v[self.a0:self.t0].reshape(-1, 3, 3)[b]
      dt = v[self.t0:].reshape(-1, 3)[b]
      out[bv] = np.einsum("nrc,nc->nr", dA, self.cc.bodies.rest[self.index[bv]]) + dt
    return out

  def scatter(self, w, out):
    """out += J^T w for vertex vectors ``w`` [..., 3]."""
    cl, bv = self.kind == 0, self.kind == 1
    np.add.at(out[:self.a0].reshape(-1, 3), self.index[cl], w[cl])
    if bv.any():
      b = self.cc.bodies.vertex_body[self.index[bv]]
      xbar = self.cc.bodies.rest[self.index[bv]]
      np.add.at(out[self.a0:self.t0].reshape(-1, 3, 3), b, np.einsum("nr,nc->nrc", w[bv], xbar))
      np.add.at(out[self.t0:].reshape(-1, 3), b, w[bv])


def _union_positions(cc, ids, union):
  vs = _Vertices(cc, ids, union)
  ids = np.asarray(ids, dtype=np.int64)
  x = np.zeros(ids.shape + (3,))
  cl, bv, ob = vs.kind == 0, vs.kind == 1, vs.kind == 2
  x[cl] = cc.cloth_position[vs.index[cl]]
  if bv.any():
    x[bv] = cc.bodies.positions()[vs.index[bv]]
  if ob.any():
    no = len(cc.obstacle)
    oid = ids[ob] if union == "obstacle_cloth" else ids[ob] - (len(cc.cloth_position) +
                                                               (0 if cc.bodies is None else len(cc.bodies.rest)))
    x[ob] = cc.obstacle[oid]
    assert np.all(oid < no)
  return vs, x


def _element_term(cc, kind, ids, union, params, method, rest=None, lagged=None, g=None, hx=None, v=None):
  if len(ids) == 0:
    return 0.0
  vs, x = _union_positions(cc, ids, union)
  e, ge, he = ve.energy_grad_hess(kind, x, rest, params, lagged)
  if method >= 1:
    he = projection.project_spd(he, method)
  n, ar = x.shape[0], x.shape[1]
  vs.scatter(ge.reshape(n, ar, 3), g)
  dx = vs.gather(v).reshape(n, 3 * ar)
  vs.scatter(np.einsum("nij,nj->ni", he, dx).reshape(n, ar, 3), hx)
  return float(e.sum())


def system_times(cc, v, projection_method: int = 1):
  """``(g, H v, energy)`` of the scene's Newton system at its built state."""
  nc, nb, a0, t0, n = _layout(cc)
  v = np.asarray(v, dtype=np.float64)
  g, hv = np.zeros(n), np.zeros(n)
  energy = 0.0
  pm = projection_method
  rest_t = cc.cloth_rest[cc.tris]
  energy += _element_term(cc, 7, cc.tris, "cloth", (cc.mu, cc.lam, cc.thickness, cc.dt), pm, rest=rest_t,
                          g=g, hx=hv, v=v)
  energy += _element_term(cc, 5, cc.bend, "cloth", (cc.bend_stiff, cc.dt), pm, rest=cc.cloth_rest[cc.bend],
                          g=g, hx=hv, v=v)
  barrier = (cc.dhat, cc.kappa)
  energy += _element_term(cc, 3, cc.pt, "obstacle_cloth", barrier, pm, g=g, hx=hv, v=v)
  energy += _element_term(cc, 4, cc.ee, "obstacle_cloth", barrier, pm, g=g, hx=hv, v=v)
  # friction: the last step's positions are the built ones (old = position)
  if len(cc.pt):
    _, x_old = _union_positions(cc, cc.pt, "obstacle_cloth")
    energy += _element_term(cc, 8, cc.pt, "obstacle_cloth", (cc.fdhat, cc.dt, cc.friction), pm, rest=x_old,
                            lagged=cc.lagged, g=g, hx=hv, v=v)
  # cloth inertia (x~ = x_old + dt^2 gravity, no projection)
  x_tilde = cc.cloth_position + np.array([0.0, -9.8, 0.0]) * cc.dt * cc.dt
  e, gi, hi = oe.inertia_local(cc.cloth_position, x_tilde, cc.mass)
  energy += float(e.sum())
  g[:a0] += gi.reshape(-1)
  hv[:a0] += (cc.mass[:, None] * v[:a0].reshape(-1, 3)).reshape(-1)
  if cc.bodies is None:
    return g, hv, energy
  bodies = cc.bodies
  energy += _element_term(cc, 3, cc.body_pt, "cloth_abd_obstacle", barrier, pm, g=g, hx=hv, v=v)
  # body vertex inertia through x = A xbar + t
  nbv = len(bodies.rest)
  vs = _Vertices(cc, nc + np.arange(nbv), "cloth_abd_obstacle")
  xb = bodies.positions()
  x_tilde = xb + bodies.velocity * bodies.dt + bodies.gravity[None] * bodies.dt * bodies.dt
  e, gi, _ = oe.inertia_local(xb, x_tilde, bodies.mass)
  energy += float(e.sum())
  vs.scatter(gi, g)
  vs.scatter(bodies.mass[:, None] * vs.gather(v), hv)
  # orthogonality on A (projection 2)
  q = np.concatenate([bodies.affine, bodies.translation], axis=1)
  e, go, ho = ae.grad_hess(ae.orthogonality, q, np.zeros((nb, 1)), bodies.stiffness)
  ho = projection.project_spd(ho, 2)
  energy += float(e.sum())
  g[a0:t0] += go[:, :9].reshape(-1)
  g[t0:] += go[:, 9:].reshape(-1)
  qv = np.concatenate([v[a0:t0].reshape(nb, 9), v[t0:].reshape(nb, 3)], axis=1)
  w = np.einsum("nij,nj->ni", ho, qv)
  hv[a0:t0] += w[:, :9].reshape(-1)
  hv[t0:] += w[:, 9:].reshape(-1)
  return g, hv, energy


def relative_residual(cc, x, projection_method: int = 1) -> float:
  """``||g - H x|| / ||g||`` of the solution ``x`` (DoF order above)."""
  g, hx, _ = system_times(cc, x, projection_method)
  return float(np.linalg.norm(g - hx) / np.linalg.norm(g))
