"""Oracle vertex-tuple energies: pinned to the reference's float64 PyTorch
scripts (bending, Baraff-Witkin) and checked for derivative consistency.

The reference scripts guard norms with +1e-8 terms, which move these
values by up to ~5e-7 relative, so the pin tolerance is 2e-6 relative.  The
barriers and the four friction kinds are pinned at 1e-12 to the reference's
own helper code in ``test_oracle_golden.py``; StVK has no reference
counterpart (parity unpinned).  Every kind's Hessian is also checked against
finite differences of its autograd gradient.
"""

import os

import numpy as np
import pytest

from oracle import vertex_energies as ve

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def cloth():
  return np.load(os.path.join(HERE, "cloth_torch.npz"))


def test_bending_matches_reference_torch(cloth):
  e, g, _ = ve.energy_grad_hess(5, cloth["bend_x"], cloth["bend_rest"], (float(cloth["bend_stiff"]), 1.0))
  assert np.allclose(e, cloth["bend_energy"], rtol=2e-6, atol=0)
  ref = cloth["bend_grad"].reshape(len(e), -1)
  assert np.abs(g - ref).max() <= 2e-6 * np.abs(ref).max()


def test_baraff_witkin_matches_reference_torch(cloth):
  e, g, _ = ve.energy_grad_hess(6, cloth["bw_x"], cloth["bw_rest"], tuple(cloth["bw_params"]))
  assert np.allclose(e, cloth["bw_energy"], rtol=2e-6, atol=0)
  ref = cloth["bw_grad"].reshape(len(e), -1)
  assert np.abs(g - ref).max() <= 2e-6 * np.abs(ref).max()


def _elements(kind, rng):
  arity = {1: 2, 2: 3, 3: 4, 4: 4, 5: 4, 6: 3, 7: 3, 8: 4}[kind]
  base = np.array([[0.0, 0.0, 0.0], [0.1, 0.0, 0.01], [0.02, 0.0, 0.1], [0.05, 0.03, 0.04]])[:arity]
  rest = base[None] + rng.uniform(-1e-3, 1e-3, size=(3, arity, 3))
  x = rest * 1.1 + rng.uniform(-2e-3, 2e-3, size=rest.shape)
  if kind in (1, 2, 3, 4):
    x[:, 0] += np.array([0.0, 0.02, 0.0])  # keep the pair apart
  return x, rest


@pytest.mark.parametrize("kind", [1, 2, 3, 4, 5, 6, 7, 8])
def test_hessian_is_the_derivative_of_the_gradient(kind):
  rng = np.random.default_rng(kind)
  x, rest = _elements(kind, rng)
  params = {1: (1e-3, 1e3), 2: (1e-3, 1e3), 3: (1e-3, 1e3), 4: (1e-3, 1e3), 5: (1e-3, 0.01),
            6: (2000.0, 1000.0, 1e-3, 0.01), 7: (5e3, 2e3, 1e-3, 0.01), 8: (1e-6, 0.01, 0.3)}[kind]
  lagged = None
  if kind == 8:
    lagged = np.stack([ve.lagged_friction_pt(x[t] + 1e-4, 1e-3, 1e3) for t in range(len(x))])
    rest = x - rng.uniform(-1e-3, 1e-3, size=x.shape)  # previous positions: a sliding step
  _, g, h = ve.energy_grad_hess(kind, x, rest, params, lagged)
  step = 1e-7
  for t in range(len(x)):
    for i in range(x.shape[1] * 3):
      xp, xm = x.copy(), x.copy()
      xp[t].reshape(-1)[i] += step
      xm[t].reshape(-1)[i] -= step
      _, gp, _ = ve.energy_grad_hess(kind, xp[t:t + 1], rest[t:t + 1], params,
                                     None if lagged is None else lagged[t:t + 1])
      _, gm, _ = ve.energy_grad_hess(kind, xm[t:t + 1], rest[t:t + 1], params,
                                     None if lagged is None else lagged[t:t + 1])
      fd = (gp[0] - gm[0]) / (2 * step)
      assert np.abs(fd - h[t, i]).max() <= 1e-5 * max(np.abs(h[t]).max(), 1e-300)


_ARITY = {1: 2, 2: 3, 3: 4, 4: 4, 5: 4, 6: 3, 7: 3, 8: 4, 9: 3, 10: 4, 11: 2}


@pytest.mark.parametrize("kind", sorted(_ARITY))
def test_batched_differentiation_matches_one_element_at_a_time(kind):
  """The batched path (torch.func over the same formulas) agrees with the
  element-by-element autograd path to rounding, on both sides of the
  friction and Baraff-Witkin selects."""
  rng = np.random.default_rng(kind)
  n, ar = 9, _ARITY[kind]
  if kind in (6, 7):
    tri = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.1], [0.1, 0.0, 0.0]])  # +y normal
    x = tri[None] + rng.uniform(-3e-3, 3e-3, size=(n, 3, 3))
    x[::2] *= 1.2  # stretched: the other side of the Baraff-Witkin select
    rest = tri[None] + rng.uniform(-1e-3, 1e-3, size=(n, 3, 3))
    rest[:, :, 1] = 0.0
  else:
    x = rng.uniform(-1.0, 1.0, size=(n, ar, 3)) * 0.03
    rest = x + rng.uniform(-1e-3, 1e-3, size=x.shape)
    rest[::2] = x[::2] + rng.uniform(-1e-7, 1e-7, size=x[::2].shape)  # inside the friction smoothing
  params = {5: (1e-3, 0.01), 6: (2000.0, 1000.0, 1e-3, 0.01), 7: (5e3, 2e3, 1e-3, 0.01)}.get(
      kind, (1e-3, 1e3) if kind <= 4 else (1e-6, 0.01, 0.3))
  lagged = rng.uniform(0.1, 0.9, size=(n, 9)) if kind >= 8 else None
  batched = ve.energy_grad_hess(kind, x, rest, params, lagged, chunk=4)
  single = ve.energy_grad_hess_loop(kind, x, rest, params, lagged)
  for a, b in zip(batched, single):
    assert np.all(np.isfinite(a))
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_baraff_witkin_select_keeps_float64():
  """The stretch weights (0.01 below unit stretch, else 1) are float64
  constants: the energy equals its direct float64 evaluation to rounding
  (a float32 0.01 would be off by 2e-8 relative)."""
  import torch
  rng = np.random.default_rng(3)
  tri = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.1], [0.1, 0.0, 0.0]])
  x = tri + rng.uniform(-3e-3, 3e-3, size=(3, 3))
  rest = tri.copy()
  p = (2000.0, 1000.0, 1e-3, 0.01)
  e = float(ve.baraff_witkin(torch.tensor(x), torch.tensor(rest), p))
  f = ve._membrane_f(torch.tensor(x), torch.tensor(rest)).numpy()
  u, v = np.linalg.norm(f[:, 0]), np.linalg.norm(f[:, 1])
  cu, cv = (0.01 if u < 1.0 else 1.0), (0.01 if v < 1.0 else 1.0)
  area = 0.5 * np.linalg.norm(np.cross(rest[1] - rest[0], rest[2] - rest[0]))
  ref = (p[0] * (cu * (u - 1.0) ** 2 + cv * (v - 1.0) ** 2) + p[1] * (f[:, 0] @ f[:, 1]) ** 2) * p[2] * area * p[3] ** 2
  assert abs(e - ref) <= 1e-14 * abs(ref)
