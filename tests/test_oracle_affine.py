"""The affine-body oracle against the pinned vertex-space oracle (CPU).

The affine energies are the vertex energies composed with ``x = A xbar + t``;
their gradient and Hessian in the body coordinates q = [A (row-major), t]
must be ``J^T g_x`` and ``J^T H_x J`` with ``J = dx/dq``.  The SNH and inertia
restatements in ``oracle.energies`` are pinned to the reference's own SNH
scripts (golden fixtures), so this check pins the affine oracle too.
"""

import numpy as np
import pytest

from oracle import affine_energies as ae
from oracle import energies as oe


def _jac(xbar):
  """dx/dq for one point x = A xbar + t, q = [A row-major, t]."""
  j = np.zeros((3, 12))
  for r in range(3):
    j[r, 3 * r:3 * r + 3] = xbar
    j[r, 9 + r] = 1.0
  return j


def _bodies(rng, n):
  out = []
  for _ in range(n):
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    a = q @ (np.eye(3) + 0.1 * rng.uniform(-1, 1, size=(3, 3)))
    out.append(np.concatenate([a.ravel(), rng.uniform(-1, 1, size=3)]))
  return np.asarray(out)


def test_affine_snh_is_vertex_snh_through_the_affine_map():
  rng = np.random.default_rng(11)
  q = _bodies(rng, 5)
  rest = rng.uniform(-0.1, 0.1, size=(5, 4, 3))
  mu, lam, dt = 3.5e4, 1.4e5, 0.01
  e, g, h = ae.grad_hess(ae.snh, q, rest.reshape(5, 12), (mu, lam, dt))
  for i in range(5):
    a, t = q[i, :9].reshape(3, 3), q[i, 9:]
    x = rest[i] @ a.T + t
    ev, gv, hv = oe.snh_from_rest(x[None], rest[i][None], mu, lam, dt)
    jj = np.concatenate([_jac(rest[i, k]) for k in range(4)])  # [12 vertex coords, 12 q]
    assert abs(e[i] - ev[0]) <= 1e-12 * abs(ev[0])
    np.testing.assert_allclose(g[i], jj.T @ gv[0], rtol=0, atol=1e-11 * np.abs(gv).max())
    ref = jj.T @ hv[0] @ jj
    np.testing.assert_allclose(h[i], ref, rtol=0, atol=1e-11 * np.abs(ref).max())
    # t does not enter F: its rows and columns vanish
    assert np.abs(h[i][9:]).max() <= 1e-12 * np.abs(ref).max()


def test_affine_inertia_is_vertex_inertia_through_the_affine_map():
  rng = np.random.default_rng(12)
  q = _bodies(rng, 4)
  xbar = rng.uniform(-0.2, 0.2, size=(4, 3))
  xb = rng.uniform(-1, 1, size=(4, 3))
  v = rng.uniform(-0.1, 0.1, size=(4, 3))
  m = rng.uniform(0.5, 2.0, size=4)
  dt, grav = 0.01, (0.0, -9.8, 0.0)
  data = np.concatenate([xbar, xb, v, m[:, None]], axis=1)
  e, g, h = ae.grad_hess(ae.inertia, q, data, (dt, *grav))
  for i in range(4):
    a, t = q[i, :9].reshape(3, 3), q[i, 9:]
    x = a @ xbar[i] + t
    xt = xb[i] + v[i] * dt + np.asarray(grav) * dt * dt
    ev, gv, hv = oe.inertia_local(x[None], xt[None], m[i])
    jj = _jac(xbar[i])
    assert abs(e[i] - ev[0]) <= 1e-13 * max(abs(ev[0]), 1e-300)
    np.testing.assert_allclose(g[i], jj.T @ gv[0], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(h[i], jj.T @ hv[0] @ jj, rtol=1e-12, atol=1e-15)


def test_orthogonality_vanishes_on_rotations_and_matches_finite_differences():
  rng = np.random.default_rng(13)
  q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
  e, g, h = ae.grad_hess(ae.orthogonality, q.reshape(1, 9), np.zeros((1, 1)), 7.0, size=9)
  assert abs(e[0]) < 1e-24 and np.abs(g).max() < 1e-12
  a = (q @ (np.eye(3) + 0.2 * rng.uniform(-1, 1, size=(3, 3)))).reshape(1, 9)
  e, g, h = ae.grad_hess(ae.orthogonality, a, np.zeros((1, 1)), 7.0, size=9)
  s = a[0].reshape(3, 3)
  ref = 7.0 * 0.5 * np.sum((s.T @ s - np.eye(3)) ** 2)
  assert abs(e[0] - ref) <= 1e-13 * ref
  eps = 1e-6
  for k in range(9):
    d = np.zeros(9)
    d[k] = eps
    ep, gp, _ = ae.grad_hess(ae.orthogonality, a + d, np.zeros((1, 1)), 7.0, size=9)
    em, gm, _ = ae.grad_hess(ae.orthogonality, a - d, np.zeros((1, 1)), 7.0, size=9)
    assert abs((ep[0] - em[0]) / (2 * eps) - g[0, k]) <= 1e-6 * np.abs(g).max()
    np.testing.assert_allclose((gp[0] - gm[0]) / (2 * eps), h[0, k], rtol=0, atol=1e-6 * np.abs(h).max())


@pytest.mark.parametrize("method", [1, 2])
def test_oracle_scene_assembly_is_symmetric_and_projected(method):
  from tests.abd_scene import oracle_assembly
  from yasps_b200 import scenes
  cube = scenes.fem_cube(3, seed=1)
  bodies = scenes.affine_bodies(num_bodies=2, m=2, seed=1)
  dense, grad, diag, energy, pat = oracle_assembly(cube, bodies, projection_method=method)
  assert np.allclose(dense, dense.T, rtol=0, atol=1e-12 * np.abs(dense).max())
  # reference layout: 9x9, 3x9 and 9x3 blocks sit beside the 3x3 ones
  dims = {tuple(d) for d in pat.dims.tolist()}
  assert (9, 9) in dims and (3, 3) in dims and ((9, 3) in dims or (3, 9) in dims)
  assert np.linalg.eigvalsh(dense).min() > 0.0
  assert np.isfinite(energy) and np.isfinite(grad).all() and np.isfinite(diag).all()
