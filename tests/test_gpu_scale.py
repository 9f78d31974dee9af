"""GPU parity beyond the small cubes: a cube of the c1 class (32^3 vertices,
the 64^3 workload's material and noise) and the precision form of the mixed
cloth + contact + friction scenes, against the FP64 oracle.

Tolerances: FP64 gradient and Hessian 1e-12 relative to the largest entry;
the FP32 block copy 1e-5 relative to the largest entry; every solve at the
stated true relative residual ||g - H x|| / ||g|| with g and H assembled by
the oracle.
"""

import numpy as np
import pytest

from oracle import baseline
from oracle import pattern as opattern
from oracle import solvers
from tests.vertex_scene import VertexScene
from yasps_b200 import scenes

pytestmark = pytest.mark.gpu


def blocks_to_csr(pos, vals, n):
  import scipy.sparse as sp
  pos = np.asarray(pos, dtype=np.int64).reshape(-1, 2)
  v = np.asarray(vals, dtype=np.float64)[:9 * len(pos)].reshape(-1, 3, 3)
  k = np.arange(3)
  rows = (pos[:, 0, None, None] + k[None, :, None]).repeat(3, axis=2)
  cols = (pos[:, 1, None, None] + k[None, None, :]).repeat(3, axis=1)
  up = sp.coo_matrix((v.ravel(), (rows.ravel(), cols.ravel())), shape=(n, n)).tocsr()
  off = pos[:, 0] != pos[:, 1]
  lo = sp.coo_matrix((v[off].ravel(), (rows[off].ravel(), cols[off].ravel())), shape=(n, n)).tocsr().T
  return (up + lo).tocsr()


@pytest.fixture(scope="module")
def c1_class():
  cube = scenes.fem_cube(32, spacing=0.1, young=1e6, poisson=0.45, noise=0.005, seed=0)
  g, H = baseline.system_from_cube(cube)
  return cube, g, H


def test_c1_class_gradient_and_hessian(c1_class):
  cube, g_o, H_o = c1_class
  sc, _ = scenes.fem_scene(cube)
  H = sc.minimizer.computeNumericValue()
  g = H.gradient.value.cpu().numpy()
  assert np.abs(g - g_o).max() <= 1e-12 * np.abs(g_o).max()
  A = blocks_to_csr(H.block_positions.cpu().numpy(), H.blocks_flattened.cpu().numpy(), H.rows)
  assert abs(A - H_o).max() <= 1e-12 * abs(H_o).max()
  H.ensure_fp32()
  nu = H._static.pattern.num_unique
  v32 = H._static.values32.cpu().numpy().reshape(-1, 12)[:nu, :9].astype(np.float64).reshape(-1)
  A32 = blocks_to_csr(H.block_positions.cpu().numpy(), v32, H.rows)
  assert abs(A32 - H_o).max() <= 1e-5 * abs(H_o).max()


@pytest.mark.parametrize("mixed", [True, False])
def test_c1_class_solve_against_oracle(c1_class, mixed):
  cube, g_o, H_o = c1_class
  sc, _ = scenes.fem_scene(cube)
  sc.minimizer.setSolver("mas", mixed_spmv=mixed, stop_rule="residual")
  segs = sc.minimizeEnergy(tolerance=1e-6, maxIterations=3000)
  x = segs[0].cpu().numpy()
  assert np.linalg.norm(g_o - H_o @ x) <= 1e-6 * np.linalg.norm(g_o)


def test_cloth_contact_precision_form_against_oracle():
  """FP32 SpMV and MAS with FP64 barrier, friction and membrane element
  Hessians and FP64 refinement, on the cloth + contact + four friction kinds
  scene: the solution meets the residual under the oracle's g and H.  The
  vertex masses are raised to 1 (condition number ~2e5): FP32 products
  carry ~1e-7 relative error, so a refinement step gains only while
  cond * 1e-7 < 1 (with the scene's 1e-3 masses the condition number is
  ~2e8 and only the FP64 path converges)."""
  vs = VertexScene(m=8, seed=5)
  vs.mass[:] = 1.0
  sc = vs.build(projection_method=1)
  sc.minimizer.setSolver("mas", mixed_spmv=True, stop_rule="residual")
  segs = sc.minimizeEnergy(tolerance=1e-8, maxIterations=4000)
  x = segs[0].cpu().numpy()
  pat, values, grad = vs.oracle_assembly(projection_method=1)
  assert solvers.relative_residual(lambda v: opattern.spmv(pat, values, v), grad, x) <= 1e-8
  assert sc.minimizer.linearSolver.statistics["refinements"] >= 1


def test_cloth_with_bodies_precision_form():
  """The c2 scene type at small size (cloth, affine icosphere bodies coupled
  by point-triangle pairs, barriers and friction against an obstacle): both
  precision forms reach the residual of the FP64 system, checked on the
  host in FP64; the FP32 form takes its refinements."""
  cc = scenes.cloth_contact(24, 2000, num_bodies=2, seed=3)
  sc, _ = scenes.cloth_contact_scene(cc)
  mz = sc.minimizer
  for mixed in (True, False):
    mz.setSolver("mas", mixed_spmv=mixed, stop_rule="residual")
    mz.computeHessianAndGradient(tolerance=1e-6, maxIterations=5000)
    Hc = mz.activeHessian()
    pos3, val3 = Hc.blocks3()
    A = blocks_to_csr(pos3.cpu().numpy(), val3.cpu().numpy(), Hc.rows)
    g = Hc.gradient.value.cpu().numpy()
    x = mz.linearSolver.implementation.solution.cpu().numpy()
    assert np.linalg.norm(g - A @ x) <= 1e-6 * np.linalg.norm(g)
