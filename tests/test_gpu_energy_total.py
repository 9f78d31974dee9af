"""Total energy (energy-only element kernels + deterministic device sums)
against the oracle, and the backtracking line search on a Newton step.
Tolerance: 1e-12 relative to the total."""

import numpy as np
import pytest

from tests.oracle_scene import OracleCube
from tests.vertex_scene import VertexScene
from oracle import vertex_energies as ve
from oracle import energies as oe
from yasps_b200 import scenes

pytestmark = pytest.mark.gpu


def test_fem_total_energy_matches_oracle():
  cube = scenes.fem_cube(8, noise=0.02, seed=3)
  ora = OracleCube(cube)
  sc, _ = scenes.fem_scene(cube)
  total = sc.computeTotalEnergy()
  expected = float(np.sum(ora.energy_snh)) + float(np.sum(ora.energy_inertia))
  assert abs(total - expected) <= 1e-12 * abs(expected)


def test_vertex_energies_total_matches_oracle():
  vs = VertexScene(m=6, seed=3)
  sc = vs.build(projection_method=1)
  total = sc.computeTotalEnergy()
  expected = 0.0
  for kind, conn, params, aux, lag in vs.terms():
    src = None if aux is None else (vs.rest if aux == "rest" else vs.x_old)
    e, _, _ = ve.energy_grad_hess(kind, vs.x[conn], None if src is None else src[conn], params, lag)
    expected += float(e.sum())
  x_tilde = vs.x_old + vs.gravity[None] * vs.dt * vs.dt
  ei, _, _ = oe.inertia_local(vs.x, x_tilde, vs.mass)
  expected += float(ei.sum())
  assert abs(total - expected) <= 1e-12 * abs(expected)


def test_line_search_decreases_energy_along_the_newton_step():
  cube = scenes.fem_cube(8, noise=0.02, seed=4)
  sc, _ = scenes.fem_scene(cube)
  before = sc.computeTotalEnergy()
  sc.minimizeEnergy(tolerance=1e-10, maxIterations=2000)
  alpha = sc.backtrackingLineSearch()
  after = sc.computeTotalEnergy()
  assert alpha > 0.0 and after < before
