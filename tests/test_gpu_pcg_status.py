"""Failure and breakdown paths of the device PCG loop (no fault, no hang).

* Non-positive curvature under MAS: the reference's device loop takes a zero
  step and restarts the direction from M^-1 r (``PKG/solver/mas/cuda/pcg.cu:183-189``).
  The case scales the blocks that couple two level-0 domains of a one-level
  hierarchy: the domain matrices (and so the preconditioner) are unchanged
  and SPD, while the first direction sees a negative curvature.  Every
  iteration then restarts from the same direction, so the solve runs to its
  iteration budget with x = 0, as the oracle's restarting loop does.
* The grid barrier of the MAS loop gives up after a host-set number of polls:
  a limit of zero makes every waiting block give up at once, the solve is
  reported void (YS_ERR_CUDA) and the context stays usable.
"""

import numpy as np
import pytest

from oracle import mas as omas
from oracle import solvers
from tests.oracle_scene import OracleCube
from yasps_b200 import _lib as L
from yasps_b200 import scenes

pytestmark = pytest.mark.gpu


def test_mas_restarts_on_non_positive_curvature():
  import torch
  cube = scenes.fem_cube(8, spacing=0.1, young=1e5, poisson=0.4, noise=0.01, seed=3)
  ora = OracleCube(cube)
  sc, _ = scenes.fem_scene(cube)
  sc.minimizer.setSolver("mas", max_levels=1, global_coarse_domain=False)
  H = sc.minimizer.computeNumericValue()
  impl = sc.minimizer.linearSolver.implementation
  impl._ensure_hierarchy(H)
  assert len(impl.hierarchy.levels) == 1 and len(impl.hierarchy.levels[0].domains) > 1
  p = ora.pattern
  nv = ora.n // 3
  edges = [(r // 3, c // 3) for r, c in p.positions if r != c]
  h = omas.build_hierarchy(np.full(nv, 3), edges, max_levels=1, global_coarse_domain=False)
  dom = np.full(nv, -1)
  for d, nodes in enumerate(h.levels[0].domains):
    dom[np.asarray(nodes)] = d
  rows, cols = p.positions[:, 0] // 3, p.positions[:, 1] // 3
  cross = dom[rows] != dom[cols]
  assert cross.any()
  blocks = lambda vals: [(r // 3, c // 3, vals[o:o + 9].reshape(3, 3)) for (r, c), o in zip(p.positions,
                                                                                             p.value_offsets)]
  pre = omas.MASPreconditioner(h, omas.level_local_matrices(h, blocks(ora.values)))
  p0 = pre.apply(ora.gradient)
  cross_vals = np.zeros_like(ora.values)
  for o in p.value_offsets[cross]:
    cross_vals[o:o + 9] = ora.values[o:o + 9]
  a = float(p0 @ pattern_matvec(p, cross_vals, p0))
  base = float(p0 @ ora.matvec(p0))
  assert base > 0 and a != 0
  scale = 1.0 - 10.0 * base / abs(a) * np.sign(a)  # curvature of p0: base + (scale - 1) a = -9 base
  vals = ora.values.copy()
  for o in p.value_offsets[cross]:
    vals[o:o + 9] *= scale
  mv = lambda x: pattern_matvec(p, vals, x)
  assert float(p0 @ mv(p0)) < 0
  # the oracle: the NumPy loop breaks down at once, the restarting loop runs out its budget
  pre2 = omas.MASPreconditioner(h, omas.level_local_matrices(h, blocks(vals)))
  assert np.allclose(pre2.apply(ora.gradient), p0, rtol=0, atol=1e-12 * np.abs(p0).max())
  stop = solvers.mas_pcg(mv, ora.gradient, pre2.apply, 1e-12, 7)
  assert stop.breakdown == "matrix is not positive definite" and stop.iterations == 0
  ref = solvers.mas_pcg(mv, ora.gradient, pre2.apply, 1e-12, 7, restart=True)
  assert not ref.converged and ref.iterations == 7 and not ref.solution.any()
  # the device, with the same scaled blocks
  bs = H.block_sets[0]
  off = bs.pattern.value_offset[:bs.pattern.num_unique].cpu().numpy().astype(np.int64)
  dpos = bs.pattern.positions[:2 * bs.pattern.num_unique].cpu().numpy().astype(np.int64).reshape(-1, 2)
  assert np.array_equal(dpos, p.positions)
  factor = np.ones(bs.values.numel())
  for o in off[cross]:
    factor[o:o + 9] = scale
  bs.values.mul_(torch.from_numpy(factor).cuda())
  solver = sc.minimizer.linearSolver
  code = solver.computeSolution(H, H.gradient, None, tolerance=1e-12, maxIterations=7, zero_initial_guess=True)
  res = solver.implementation.last_result
  assert code == -4 and res.status == L.YS_ERR_NOT_CONVERGED and res.iterations == 7
  assert not solver.solution.cpu().numpy().any()


def pattern_matvec(p, vals, x):
  from oracle import pattern
  return pattern.spmv(p, vals, x)


def test_mas_grid_barrier_poll_limit_voids_the_solve():
  cube = scenes.fem_cube(10, spacing=0.1, young=1e5, poisson=0.4, noise=0.01, seed=0)
  ora = OracleCube(cube)
  sc, _ = scenes.fem_scene(cube)
  sc.minimizer.setSolver("mas")
  H = sc.minimizer.computeNumericValue()
  solver = sc.minimizer.linearSolver
  solve = lambda: solver.computeSolution(H, H.gradient, None, tolerance=1e-12, maxIterations=40,
                                         zero_initial_guess=True)
  assert solve() == 0
  handle = solver.implementation._cache.handle
  assert handle is not None
  L.call("ys_pcg_set_barrier_poll_limit", handle, 0)
  with pytest.raises(L.YsError) as err:
    solve()
  assert err.value.code == L.YS_ERR_CUDA
  assert b"barrier" in L.load().ys_last_error()
  assert solver.implementation._cache.handle.value == handle.value  # the same graph ran
  L.call("ys_pcg_set_barrier_poll_limit", handle, 1 << 24)
  assert solve() == 0
  x = solver.solution.cpu().numpy()
  assert solvers.relative_residual(ora.matvec, ora.gradient, x) <= 1e-5
