"""The cloth-over-obstacle scene with affine bodies (the c2 scene type)
against the matrix-free FP64 oracle: the device gradient and the product of
the assembled FP64 Hessian with a random vector within 1e-12 of the
largest entry, and both precision forms' solutions at the stated true
relative residual of the oracle's system."""

import numpy as np
import pytest

from oracle import cloth_scene
from yasps_b200 import scenes

pytestmark = pytest.mark.gpu


def _csr(H):
  import scipy.sparse as sp
  pos3, val3 = H.blocks3()
  pos = pos3.cpu().numpy().astype(np.int64).reshape(-1, 2)
  v = val3.cpu().numpy()[:9 * len(pos)].reshape(-1, 3, 3)
  n = H.rows
  k = np.arange(3)
  rows = (pos[:, 0, None, None] + k[None, :, None]).repeat(3, axis=2)
  cols = (pos[:, 1, None, None] + k[None, None, :]).repeat(3, axis=1)
  up = sp.coo_matrix((v.ravel(), (rows.ravel(), cols.ravel())), shape=(n, n)).tocsr()
  off = pos[:, 0] != pos[:, 1]
  lo = sp.coo_matrix((v[off].ravel(), (rows[off].ravel(), cols[off].ravel())), shape=(n, n)).tocsr().T
  return (up + lo).tocsr()


@pytest.mark.parametrize("bodies", [0, 2])
def test_cloth_scene_system_matches_oracle(bodies):
  cc = scenes.cloth_contact(24, 2000, num_bodies=bodies, body_subdivisions=2, body_radius=0.25, seed=3)
  sc, _ = scenes.cloth_contact_scene(cc)
  H = sc.minimizer.computeNumericValue()
  g = H.gradient.value.cpu().numpy()
  A = _csr(H)
  v = np.random.default_rng(0).normal(size=H.rows)
  g_o, hv_o, _ = cloth_scene.system_times(cc, v)
  assert np.abs(g - g_o).max() <= 1e-12 * np.abs(g_o).max()
  assert np.abs(A @ v - hv_o).max() <= 1e-12 * np.abs(hv_o).max()


@pytest.mark.parametrize("mixed", [True, False])
def test_cloth_scene_solutions_against_oracle(mixed):
  cc = scenes.cloth_contact(24, 2000, num_bodies=2, body_subdivisions=2, body_radius=0.25, seed=3)
  sc, _ = scenes.cloth_contact_scene(cc)
  sc.minimizer.setSolver("mas", mixed_spmv=mixed, stop_rule="residual")
  segs = sc.minimizeEnergy(tolerance=1e-6, maxIterations=5000)
  x = np.concatenate([s.cpu().numpy().reshape(-1) for s in segs])
  assert cloth_scene.relative_residual(cc, x) <= 1e-6
