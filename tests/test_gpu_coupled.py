"""Barrier contact through affine-body vertices on the GPU against the oracle.

The device and the oracle evaluate each pair in vertex coordinates, project
that Hessian (the reference's inner projection for a linear map from the
leaves) and apply the chain rule to the body leaves, merging repeated ones.  Compared: dense assembled matrix and gradient at 1e-12 relative to
the largest entry, energy total at 1e-12 relative; the rerun is
bit-identical; a solve of the full scene (with inertia and orthogonality)
through MAS reaches the stated true relative residual.
"""

import numpy as np
import pytest

from tests import coupled_scene as cs

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


@pytest.mark.parametrize("method", [0, 1, 2])
def test_coupled_assembly_matches_oracle(method):
  s = cs.make(seed=3)
  sc, _ = cs.scene(s, method)
  H = sc.minimizer.computeNumericValue()
  dense, grad, energy = cs.oracle_assembly(s, method)
  assert rel(H.gradient.value.cpu().numpy(), grad) <= 1e-12
  assert rel(_dense(H), dense) <= 1e-12
  assert abs(sc.computeTotalEnergy() - energy) <= 1e-12 * abs(energy)


@pytest.mark.parametrize("method", [1, 2])
def test_coupled_friction_matches_oracle(method):
  """Lagged friction of the four kinds through affine-body vertices (the
  old positions through the same union), beside the barriers."""
  s = cs.add_friction(cs.make(seed=3))
  sc, _ = cs.scene(s, method)
  H = sc.minimizer.computeNumericValue()
  dense, grad, energy = cs.oracle_assembly(s, method)
  assert rel(H.gradient.value.cpu().numpy(), grad) <= 1e-12
  assert rel(_dense(H), dense) <= 1e-12
  assert abs(sc.computeTotalEnergy() - energy) <= 1e-12 * abs(energy)


def test_separate_hessian_jacobian_flag_gives_the_same_matrix():
  """addEnergy(separate_hessian_jacobian=True) (the reference's explicit
  J-block evaluation of J^T H J) assembles the same values bit for bit."""
  s = cs.add_friction(cs.make(seed=3))
  sc, _ = cs.scene(s, 2)
  first = sc.minimizer.computeNumericValue().blocks_flattened.clone()
  sc2, _ = cs.scene(s, 2, separate_hessian_jacobian=True)
  assert bool((sc2.minimizer.computeNumericValue().blocks_flattened == first).all())


def test_coupled_projection_is_exercised_and_reruns_bit_identical():
  s = cs.make(seed=3)
  d0, *_ = cs.oracle_assembly(s, 0)
  d2, *_ = cs.oracle_assembly(s, 2)
  assert rel(d2, d0) > 1e-9, "the coupled pairs must reach the projection"
  sc, _ = cs.scene(s, 2)
  H = sc.minimizer.computeNumericValue()
  first = H.blocks_flattened.clone()
  H = sc.minimizer.computeNumericValue()
  assert bool((H.blocks_flattened == first).all())


def test_coupled_scene_mas_solve():
  from yasps_b200 import scenes
  s = cs.make(seed=4)
  sc, _ = scenes.contact_with_bodies_scene(s["cloth"], s["bodies"], s["container"], s["pairs"], s["dhat"],
                                           s["kappa"], projection_method=2, cloth_mass=s["mass"])
  sc.minimizer.setSolver("mas", stop_rule="residual")
  segs = sc.minimizeEnergy(tolerance=1e-8, maxIterations=4000)
  x = np.concatenate([v.cpu().numpy().reshape(-1) for v in segs])
  H = sc.minimizer.computeNumericValue()
  dense = _dense(H)
  g = H.gradient.value.cpu().numpy()
  assert np.linalg.norm(g - dense @ x) <= 1e-8 * np.linalg.norm(g)
  assert [v.numel() for v in segs] == [3 * len(s["cloth"]), 9 * s["bodies"].num_bodies,
                                        3 * s["bodies"].num_bodies]


def test_cloth_with_bodies_newton_step():
  """The mixed scene (cloth membrane, bending, barriers and friction against
  an obstacle, icosphere affine bodies coupled to the cloth by PT pairs)
  in both precision forms: the solution meets the true relative residual of
  the assembled FP64 system."""
  from yasps_b200 import scenes
  cc = scenes.cloth_contact(24, 2_000, num_bodies=2, body_subdivisions=2, body_radius=0.25)
  assert len(cc.body_pt) > 0
  sc, _ = scenes.cloth_contact_scene(cc)
  mz = sc.minimizer
  for mixed in (True, False):
    mz.setSolver("mas", mixed_spmv=mixed, stop_rule="residual")
    segs = sc.minimizeEnergy(tolerance=1e-6, maxIterations=5000)
    x = np.concatenate([v.cpu().numpy().reshape(-1) for v in segs])
    H = mz.computeNumericValue()
    g = H.gradient.value.cpu().numpy()
    assert np.linalg.norm(g - _dense(H) @ x) <= 1e-6 * np.linalg.norm(g)
    assert [v.numel() for v in segs] == [3 * 24 * 24, 18, 6]
