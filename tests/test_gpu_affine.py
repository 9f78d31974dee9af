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
  """Dense matrix from the public block attributes (any block categories)."""
  pos = H.block_positions.cpu().numpy().astype(np.int64).reshape(-1, 2)
  vals = H.blocks_flattened.cpu().numpy()
  dims = np.asarray(H.block_dimensions, dtype=np.int64).reshape(-1, 2)
  d = np.zeros((H.rows, H.rows))
  k = 0
  for (h, w), cnt, start in zip(dims, H.block_counts, H.blocks_start_indices):
    for j in range(cnt):
      r, c = pos[k]
      b = vals[start + j * h * w:start + (j + 1) * h * w].reshape(h, w)
      d[r:r + h, c:c + w] += b
      if r != c:
        d[c:c + w, r:r + h] += b.T
      k += 1
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
  dense, grad, diag, energy, pat = oracle_assembly(cube, bodies, projection_method=method)
  assert rel(H.gradient.value.cpu().numpy(), grad) <= 1e-12
  assert rel(_dense(H), dense) <= 1e-12
  assert rel(H.diagonal_blocks.cpu().numpy(), diag) <= 1e-12
  assert rel(H.diagonal.cpu().numpy(), np.diag(dense)) <= 1e-12
  assert abs(sc.computeTotalEnergy() - energy) <= 1e-12 * abs(energy)


def test_affine_reference_layout_bit_exact():
  """The public block attributes of a scene with 9-DoF affine targets carry
  the reference's layout: categories (9x9, 9x3, 3x9, 3x3 ...) in (h, w, row,
  col) order, block positions, category counts and value starts, and the
  lookup of every element block, bit-exact against the oracle pattern built
  with 9-DoF slots; the values at 1e-12."""
  cube, bodies, sc, _ = _scene(1)
  H = sc.minimizer.computeNumericValue()
  _, _, _, _, pat = oracle_assembly(cube, bodies, projection_method=1)
  pos = H.block_positions.cpu().numpy().astype(np.int64).reshape(-1, 2)
  assert np.array_equal(pos, pat.positions)
  assert H.block_dimensions == pat.category_dims.reshape(-1).tolist()
  assert sorted(set(map(tuple, pat.category_dims.tolist()))) >= [(3, 3), (3, 9), (9, 3), (9, 9)]
  assert H.block_counts == pat.category_counts.tolist()
  assert H.blocks_start_indices == pat.category_starts.tolist()
  assert np.array_equal(H.lookups.cpu().numpy().astype(np.int64), np.concatenate(pat.lookups))
  # values: the same matrix through both layouts
  dense, *_ = oracle_assembly(cube, bodies, projection_method=1)
  assert rel(_dense(H), dense) <= 1e-12


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


def test_affine_scene_block_jacobi_with_9x9_blocks():
  """Block-Jacobi PCG with the 9x9 diagonal blocks of the affine matrices
  (pseudo-inverted whole, diagonalBlockInverseKernel.pyx:40-215) and 3x3
  blocks elsewhere, against the oracle's block-Jacobi PCG on the same
  system: the reference's return code within one iteration and the solution
  at the reference's squared preconditioned stopping rule."""
  cube, bodies, sc, _ = _scene(1, seed=2, nb=4)
  sc.minimizer.setSolver("jacobian")
  H = sc.minimizer.computeNumericValue()
  dense, grad, diag, _, pat = oracle_assembly(cube, bodies, projection_method=1)
  nf, nb = cube.free_count, bodies.num_bodies
  counts, sizes = [nf, nb, nb], [3, 9, 3]
  inv = solvers.diagonal_inverse(diag, counts, sizes)
  ref = solvers.jacobi_pcg(lambda v: dense @ v, grad, inv, counts, sizes, 1e-14, 4000)
  code = sc.minimizer.linearSolver.computeSolution(H, H.gradient, None, tolerance=1e-14, maxIterations=4000,
                                                   zero_initial_guess=True)
  assert ref.status > 0 and abs(code - ref.status) <= 1
  x = sc.minimizer.linearSolver.solution.cpu().numpy()
  assert solvers.relative_residual(lambda v: dense @ v, grad, x) <= 10 * solvers.relative_residual(
      lambda v: dense @ v, grad, ref.solution) + 1e-9
