"""The rectangular-Jacobian oracle on closed forms: the inertia term's
blocks d2E/(dx dx_before) = -m I and d2E/(dx dv) = -m dt I, repeated
targets of one instance adding up, and non-target slots dropped."""

import numpy as np

from oracle import rect_jacobian as orj


def test_inertia_blocks_and_merging():
  m = np.array([2.0, 3.0])
  dt = 0.01
  loc = orj.inertia_local(m, dt)
  i = np.arange(2)
  rc = np.stack([2 + 3 * i, 0 * i, 0 * i], axis=1)
  cc = np.stack([0 * i, 2 + 3 * i, 0 * i], axis=1)
  J = orj.dense(loc, rc, cc, 6, 6)
  assert np.allclose(J, np.kron(np.diag(-m), np.eye(3)))
  cv = np.stack([0 * i, 0 * i, 2 + 3 * i], axis=1)
  assert np.allclose(orj.dense(loc, rc, cv, 6, 6), np.kron(np.diag(-m * dt), np.eye(3)))
  # x_before and v both mapped to one column target: the blocks add up
  cboth = np.stack([0 * i, 2 + 3 * i, 2 + 3 * i], axis=1)
  assert np.allclose(orj.dense(loc, rc, cboth, 6, 6), np.kron(np.diag(-m * (1 + dt)), np.eye(3)))


def test_snh_hessian_with_rest_matches_the_position_hessian():
  """The (x, X) Hessian's position block is the SNH oracle's Hessian, and its
  position-rest block is the derivative of the oracle gradient in X
  (central differences of the closed-form gradient, 1e-6)."""
  from oracle import energies as oe
  from yasps_b200 import scenes
  cube = scenes.fem_cube(3, noise=0.01, seed=2)
  tets = cube.tets.astype(np.int64)[:5]
  x, X = cube.positions_all()[tets], cube.rest_all()[tets]
  h = oe.snh_hessian_with_rest(x, X, cube.mu, cube.lam, cube.dt)
  _, g, hxx = oe.snh_from_rest(x, X, cube.mu, cube.lam, cube.dt)
  assert np.abs(h[:, :12, :12] - hxx).max() <= 1e-12 * np.abs(hxx).max()
  eps = 1e-6
  for k in range(12):
    Xp, Xm = X.reshape(-1, 12).copy(), X.reshape(-1, 12).copy()
    Xp[:, k] += eps
    Xm[:, k] -= eps
    gp = oe.snh_from_rest(x, Xp.reshape(-1, 4, 3), cube.mu, cube.lam, cube.dt)[1]
    gm = oe.snh_from_rest(x, Xm.reshape(-1, 4, 3), cube.mu, cube.lam, cube.dt)[1]
    fd = (gp - gm) / (2 * eps)
    assert np.abs(h[:, :12, 12 + k] - fd).max() <= 1e-6 * np.abs(h[:, :12, 12:]).max()


def test_snh_parameter_jacobian_matches_differences():
  """The oracle's d(dE/dx)/d mu and d(dE/dx)/d lambda against central
  differences of the closed-form SNH gradient (1e-6)."""
  from oracle import energies as oe
  from yasps_b200 import scenes
  cube = scenes.fem_cube(3, noise=0.01, seed=2)
  tets = cube.tets.astype(np.int64)[:6]
  x, X = cube.positions_all()[tets], cube.rest_all()[tets]
  for which in (0, 1):
    d = oe.snh_parameter_jacobian(x, X, cube.mu, cube.lam, cube.dt, which)
    h = 1e-6 * (cube.mu if which == 0 else cube.lam)
    args = lambda s: (cube.mu + s, cube.lam) if which == 0 else (cube.mu, cube.lam + s)
    gp = oe.snh_from_rest(x, X, *args(h), cube.dt)[1]
    gm = oe.snh_from_rest(x, X, *args(-h), cube.dt)[1]
    fd = (gp - gm) / (2 * h)
    assert np.abs(d - fd).max() <= 1e-6 * np.abs(d).max()
