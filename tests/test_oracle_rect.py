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
