"""Affine (ABD) bodies beside a soft cube on the GPU against the oracle.

The device stores each body's affine matrix as three 3-DoF rows (every block
3x3); the oracle keeps the reference's 9-DoF slot (9x9 / 9x3 blocks).  They
are compared as dense matrices, gradients and per-variable diagonal blocks.
Tolerances: FP64 gradient and projected Hessian 1e-12 relative to the largest
magnitude; energy total 1e-12 relative; the MAS solve at the stated true
relative residual.
"""

import numpy as np
import pytest

from oracle import solvers
from tests.abd_scene import oracle_assembly

pytestmark = pytest.mark.gpu


def rel(a, b):
  a, b = np.asarray(a), np.asarray(b)
  return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _dense(H):
  pos = H.block_positions.cpu().numpy().astype(np.int64).reshape(-1, 2)
  vals = H.blocks_flattened.cpu().numpy()[:9 * pos.shape[0]].reshape(-1, 3, 3)
  d = np.zeros((H.rows, H.rows))
  for (r, c), b in zip(pos, vals):
    d[r:r + 3, c:c + 3] += b
    if r != c:
      d[c:c + 3, r:r + 3] += b.T
  return d


def _scene(method, seed=1, nb=3, m=3):
  from yasps_b200 import scenes
  cube = scenes.fem_cube(4, seed=seed)
  bodies = scenes.affine_bodies(num_bodies=nb, m=m, seed=seed, deform=0.05)
  sc, hd = scenes.affine_scene(cube, bodies, projection_method=method)
  return cube, bodies, sc, hd


@pytest.mark.parametrize("method", [1, 0])
def test_affine_assembly_matches_oracle(method):
  cube, bodies, sc, _ = _scene(method)
  H = sc.minimizer.computeNumericValue()
  dense, grad, diag, energy, _ = oracle_assembly(cube, bodies, projection_method=method)
  assert H.block_dimensions == [3, 3]
  assert rel(H.gradient.value.cpu().numpy(), grad) <= 1e-12
  assert rel(_dense(H), dense) <= 1e-12
  assert rel(H.diagonal_blocks.cpu().numpy(), diag) <= 1e-12
  assert rel(H.diagonal.cpu().numpy(), np.diag(dense)) <= 1e-12
  assert abs(sc.computeTotalEnergy() - energy) <= 1e-12 * abs(energy)


def test_affine_projection_is_exercised():
  cube, bodies, _, _ = _scene(1)
  d1, *_ = oracle_assembly(cube, bodies, projection_method=1)
  d0, *_ = oracle_assembly(cube, bodies, projection_method=0)
  assert rel(d1, d0) > 1e-9, "the affine SNH terms must reach the projection"


def test_affine_scene_mas_solve():
  cube, bodies, sc, hd = _scene(1, seed=2, nb=4)
  sc.minimizer.setSolver("mas", stop_rule="residual")
  segs = sc.minimizeEnergy(tolerance=1e-8, maxIterations=4000)
  x = np.concatenate([s.cpu().numpy().reshape(-1) for s in segs])
  dense, grad, *_ = oracle_assembly(cube, bodies, projection_method=1)
  assert solvers.relative_residual(lambda v: dense @ v, grad, x) <= 1e-8
  assert [s.numel() for s in segs] == [3 * cube.free_count, 9 * bodies.num_bodies, 3 * bodies.num_bodies]


def test_affine_bodies_reject_mixed_tets():
  from yasps_b200 import scenes
  cube = scenes.fem_cube(3, seed=0)
  bodies = scenes.affine_bodies(num_bodies=2, m=2, seed=0)
  bad = bodies.tets.copy()
  bad[0, 3] = bodies.tets[-1, 0]  # a vertex of the other body
  bodies.tets = bad
  sc, _ = scenes.affine_scene(cube, bodies)
  with pytest.raises(ValueError, match="one body"):
    sc.minimizer.computeNumericValue()
