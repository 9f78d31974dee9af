"""The matrix-free oracle of the cloth-over-obstacle scene with affine
bodies: its Hessian product is linear and symmetric, and its gradient and
Hessian product agree with the element oracles assembled densely for the
barrier-only body coupling (the coupled-contact oracle, which differentiates
each pair through its leaf Jacobian independently)."""

import numpy as np

from oracle import cloth_scene
from yasps_b200 import scenes


def _scene():
  return scenes.cloth_contact(8, 120, num_bodies=2, body_subdivisions=1, body_radius=0.12, seed=4)


def test_hessian_product_is_symmetric_and_linear():
  cc = _scene()
  assert cc.bodies is not None and len(cc.body_pt) > 0
  n = 3 * len(cc.cloth_position) + 12 * cc.bodies.num_bodies
  rng = np.random.default_rng(0)
  u, v = rng.normal(size=n), rng.normal(size=n)
  g, hu, _ = cloth_scene.system_times(cc, u)
  _, hv, _ = cloth_scene.system_times(cc, v)
  _, huv, _ = cloth_scene.system_times(cc, 2.0 * u - 3.0 * v)
  scale = np.abs(hu).max() + np.abs(hv).max()
  assert abs(u @ hv - v @ hu) <= 1e-12 * scale * (np.abs(u).sum() + np.abs(v).sum())
  assert np.abs(huv - (2.0 * hu - 3.0 * hv)).max() <= 1e-12 * scale * 5.0
  assert np.all(np.isfinite(g)) and np.abs(g).max() > 0.0


def test_body_coupling_matches_the_coupled_contact_oracle():
  """The body-cloth point-triangle pairs through ``J^T proj(H) J``: the
  matrix-free product equals the dense matrix of ``coupled_contact``'s
  per-pair compressed blocks."""
  from oracle import coupled_contact as occ
  cc = _scene()
  nc, nb = len(cc.cloth_position), cc.bodies.num_bodies
  a0, t0, n = 3 * nc, 3 * nc + 9 * nb, 3 * nc + 12 * nb
  rng = np.random.default_rng(1)
  v = rng.normal(size=n)
  g_dense, h_dense = np.zeros(n), np.zeros((n, n))
  nbv = len(cc.bodies.rest)
  for row in cc.body_pt.astype(np.int64):
    verts, dofs = [], []
    for idx in row:
      if idx < nc:
        verts.append(("p", cc.cloth_position[idx]))
        dofs.append([3 * idx + k for k in range(3)])
      elif idx < nc + nbv:
        i = idx - nc
        b = int(cc.bodies.vertex_body[i])
        verts.append(("a", cc.bodies.affine[b], cc.bodies.translation[b], cc.bodies.rest[i], b))
        dofs.append(None)
      else:
        verts.append(("p", cc.obstacle[idx - nc - nbv]))
        dofs.append("obstacle")
    # leaf Jacobian columns: every DoF of the scene, J [12, n]
    J = np.zeros((12, n))
    for k, (d, ds) in enumerate(zip(verts, dofs)):
      if ds == "obstacle":
        continue
      if ds is not None:
        J[3 * k:3 * k + 3, ds] = np.eye(3)
      else:
        b, xbar = d[4], d[3]
        for r in range(3):
          J[3 * k + r, a0 + 9 * b + 3 * r:a0 + 9 * b + 3 * r + 3] = xbar
          J[3 * k + r, t0 + 3 * b + r] = 1.0
    x = occ._positions(verts)
    from oracle import projection
    from oracle import vertex_energies as ve
    _, gx, hx = ve.energy_grad_hess_loop(3, x[None], None, (cc.dhat, cc.kappa))
    g_dense += J.T @ gx[0]
    h_dense += J.T @ projection.project_spd(hx[0], 1) @ J
  g_all, hv_all, _ = cloth_scene.system_times(cc, v)
  # remove every other term by differencing against the scene without body pairs
  bare = scenes.cloth_contact(8, 120, num_bodies=2, body_subdivisions=1, body_radius=0.12, seed=4)
  bare.body_pt = np.zeros((0, 4), dtype=np.uint32)
  g_bare, hv_bare, _ = cloth_scene.system_times(bare, v)
  assert np.abs((g_all - g_bare) - g_dense).max() <= 1e-10 * np.abs(g_dense).max()
  ref = h_dense @ v
  assert np.abs((hv_all - hv_bare) - ref).max() <= 1e-10 * np.abs(ref).max()
