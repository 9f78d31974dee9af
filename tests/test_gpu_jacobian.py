"""Rectangular second-order Jacobians (``differentiator.diff2`` with
different row and column targets) against the oracle: the pattern (unique
block positions, row-major) bit-exact, the blocks within 1e-12 of the
largest entry, and ``spmv`` / ``spmv(transpose=True)`` against the dense
oracle matrix.  Cases: the barrier coupling of cloth and obstacle vertices
(a union's two leaves), the inertia term's adjoint blocks (x against
x_before and against the velocity), the SNH coupling of free and pinned
vertices; and the square / gradient forms of the same front end."""

import numpy as np
import pytest

from oracle import energies as oe
from oracle import rect_jacobian as orj
from oracle import vertex_energies as ve
from yasps_b200 import scenes
from yasps_b200.hessian import vector
from yasps_b200.jacobian import differentiator, secondOrderJacobian

pytestmark = pytest.mark.gpu


def device_dense(J):
  pos = J.block_positions.cpu().numpy().astype(np.int64).reshape(-1, 2)
  vals = J.blocks_flattened.cpu().numpy().reshape(-1, 3, 3)
  D = np.zeros((J.rows, J.cols))
  for (r, c), b in zip(pos, vals):
    D[r:r + 3, c:c + 3] += b
  return D, pos


def expected_positions(row_codes, col_codes):
  pairs = {(int(r) - 2, int(c) - 2) for rr, cc in zip(row_codes, col_codes) for r in rr if r >= 2 for c in cc if c >= 2}
  return np.array(sorted(pairs), dtype=np.int64).reshape(-1, 2)


def check(J, D_oracle, row_codes, col_codes):
  D, pos = device_dense(J)
  assert np.array_equal(pos, expected_positions(row_codes, col_codes))
  scale = np.abs(D_oracle).max()
  assert np.abs(D - D_oracle).max() <= 1e-12 * scale
  rng = np.random.default_rng(0)
  x = rng.normal(size=J.cols)
  y = rng.normal(size=J.rows)
  import torch
  xv = vector(J.cols, torch.from_numpy(x).cuda())
  yv = vector(J.rows, torch.from_numpy(y).cuda())
  assert np.abs(J.spmv(xv).get() - D_oracle @ x).max() <= 1e-12 * scale * np.abs(x).sum()
  assert np.abs(J.spmv(yv, transpose=True).get() - D_oracle.T @ y).max() <= 1e-12 * scale * np.abs(y).sum()


def cloth_obstacle_scene():
  from yasps_b200.energies import point_triangle
  from yasps_b200.scene import scene as make_scene
  cc = scenes.cloth_contact(10, 120, seed=5)
  sc = make_scene("rect")
  m = sc.addMesh("m")
  obst = m.addPrimitive("obstacle", numInstances=len(cc.obstacle))
  opos = obst.addAttribute("position", rows=3, cols=1)
  opos.updateValue(cc.obstacle)
  cloth = m.addPrimitive("cloth", numInstances=len(cc.cloth_position))
  pos = cloth.addAttribute("position", rows=3, cols=1)
  pos.updateValue(cc.cloth_position)
  allv = m.addPrimitiveUnion("all", [obst, cloth])
  apos = allv.addAttribute("position")
  pt = m.addPrimitive("pt", numInstances=len(cc.pt))
  c = pt.addConnectivity("to_vertices", allv, cc.pt, 4)
  e = pt.addAttribute("barrier", computed_attribute=point_triangle(
      pt.addAttribute("x", through=c, source=apos), cc.dhat, cc.kappa))
  return cc, e, pos, opos


def test_barrier_cloth_obstacle_coupling():
  cc, e, pos, opos = cloth_obstacle_scene()
  J = differentiator().diff2([e], [pos], [opos])
  assert isinstance(J, secondOrderJacobian)
  J.compute()
  no = len(cc.obstacle)
  allx = np.concatenate([cc.obstacle, cc.cloth_position])
  ids = cc.pt.astype(np.int64)
  _, _, h = ve.energy_grad_hess(3, allx[ids], None, (cc.dhat, cc.kappa))
  rc = np.where(ids >= no, 2 + 3 * (ids - no), 0)
  ccode = np.where(ids < no, 2 + 3 * ids, 0)
  check(J, orj.dense(h, rc, ccode, J.rows, J.cols), rc, ccode)
  # the transposed pair of target lists is the transposed matrix
  Jt = differentiator().diff2([e], [opos], [pos]).compute()
  assert np.abs(device_dense(Jt)[0] - device_dense(J)[0].T).max() == 0.0


@pytest.mark.parametrize("column", ["last_position", "velocity"])
def test_inertia_adjoint_blocks(column):
  cube = scenes.fem_cube(6, noise=0.01, seed=2)
  sc, h = scenes.fem_scene(cube)
  kin = next(r.energy for r in sc.minimizer.requests if r.energy.expr.kind == "inertia")
  J = differentiator().diff2([kin], [h["free_position"]], [h[column]]).compute()
  nf = cube.free_count
  dt = kin.expr.dt_p[1].scalar() if kin.expr.dt_p[0] == "scene" else float(kin.expr.dt_p[1])
  loc = orj.inertia_local(cube.mass, dt)
  arg = 1 if column == "last_position" else 2
  i = np.arange(nf)
  rc = np.stack([2 + 3 * i, np.zeros(nf, np.int64), np.zeros(nf, np.int64)], axis=1)
  ccode = np.zeros((nf, 3), dtype=np.int64)
  ccode[:, arg] = 2 + 3 * i
  check(J, orj.dense(loc, rc, ccode, J.rows, J.cols), rc, ccode)
  # sums of Jacobians over the same target lists
  both = (differentiator().diff2([kin], [h["free_position"]], [h[column]]) +
          differentiator().diff2([kin], [h["free_position"]], [h[column]])).compute()
  assert np.abs(device_dense(both)[0] - 2.0 * device_dense(J)[0]).max() <= 1e-15 * np.abs(loc).max()


def test_snh_free_pinned_coupling():
  cube = scenes.fem_cube(6, noise=0.01, seed=3)
  sc, h = scenes.fem_scene(cube)
  snh = next(r.energy for r in sc.minimizer.requests if r.energy.expr.kind == "snh")
  J = differentiator().diff2([snh], [h["free_position"]], [h["pinned_position"]]).compute()
  tets = cube.tets.astype(np.int64)
  _, _, hl = oe.snh_from_rest(cube.positions_all()[tets], cube.rest_all()[tets], cube.mu, cube.lam, cube.dt)
  npin = cube.pinned_count
  rc = np.where(tets >= npin, 2 + 3 * (tets - npin), 0)
  ccode = np.where(tets < npin, 2 + 3 * tets, 0)
  check(J, orj.dense(hl, rc, ccode, J.rows, J.cols), rc, ccode)


def test_square_and_gradient_forms():
  """diff2 with equal targets is the (projected) Hessian of the same terms;
  diff1 of scalar energies their gradient."""
  cube = scenes.fem_cube(5, noise=0.01, seed=4)
  sc, h = scenes.fem_scene(cube)
  energies = [r.energy for r in sc.minimizer.requests]
  H = sc.minimizer.computeNumericValue()
  g_scene = H.gradient.value.cpu().numpy()
  d = differentiator()
  H2 = d.diff2([energies[0]], [h["free_position"]], [h["free_position"]], projection_method=1) + \
      d.diff2([energies[1]], [h["free_position"]], [h["free_position"]], projection_method=-1)
  H2.compute()
  assert np.abs(H2.gradient.value.cpu().numpy() - g_scene).max() <= 1e-13 * np.abs(g_scene).max()
  p1, v1 = H.blocks3()
  p2, v2 = H2.blocks3()
  assert np.array_equal(p1.cpu().numpy(), p2.cpu().numpy())
  assert np.abs(v1.cpu().numpy() - v2.cpu().numpy()).max() <= 1e-13 * np.abs(v1.cpu().numpy()).max()
  g = d.diff1(energies, [h["free_position"]]).compute()
  assert np.abs(g.value.cpu().numpy() - g_scene).max() <= 1e-13 * np.abs(g_scene).max()


@pytest.mark.parametrize("kind", [8, 9, 10, 11])
def test_friction_position_against_step_start_positions(kind):
  """Lagged friction is a function of x - x_old: d2E/(dx dx_old) is minus the
  unprojected position Hessian, argument by argument (the oracle's local
  Hessian folded over the step-start leaves)."""
  from tests.vertex_scene import VertexScene
  from yasps_b200 import energies as E
  from yasps_b200.scene import scene as make_scene
  vs = VertexScene(m=6, seed=5)
  conn = {8: vs.pt, 9: vs.pe, 10: vs.ee, 11: vs.pp}[kind]
  lag = {8: vs.lagged, 9: vs.lagged_pe, 10: vs.lagged_ee, 11: vs.lagged_pp}[kind]
  sc = make_scene("friction_rect")
  m = sc.addMesh("m")
  verts = m.addPrimitive("vertices", numInstances=len(vs.x))
  pos = verts.addAttribute("position", rows=3, cols=1)
  pos.updateValue(vs.x)
  old = verts.addConstant("old_position", rows=3, cols=1)
  old.updateValue(vs.x_old)
  prim = m.addPrimitive("pairs", numInstances=len(conn))
  c = prim.addConnectivity("to_vertices", verts, conn.astype(np.uint32), conn.shape[1])
  lagged = prim.addConstant("lagged", rows=9, cols=1)
  lagged.updateValue(lag)
  fric = {8: E.friction_point_triangle, 9: E.friction_point_edge, 10: E.friction_edge_edge,
          11: E.friction_point_point}[kind]
  e = prim.addAttribute("friction", computed_attribute=fric(
      prim.addAttribute("x", through=c, source=pos), prim.addAttribute("x_old", through=c, source=old),
      *vs.fric_params, lagged))
  J = differentiator().diff2([e], [pos], [old]).compute()
  _, _, h = ve.energy_grad_hess(kind, vs.x[conn], vs.x_old[conn], vs.fric_params, lag)
  A = conn.shape[1]
  ext = np.block([[h, -h], [-h, h]])
  ids = conn.astype(np.int64)
  zero = np.zeros_like(ids)
  rc = np.concatenate([2 + 3 * ids, zero], axis=1)
  ccode = np.concatenate([zero, 2 + 3 * ids], axis=1)
  assert ext.shape[1] == 6 * A
  check(J, orj.dense(ext, rc, ccode, J.rows, J.cols), rc, ccode)


def test_snh_positions_against_rest_positions():
  """Shape derivatives d2E/(dx dX) of the SNH tetrahedra (free positions
  against free rest positions) against the oracle's autograd Hessian over
  (x, X); rest against rest is not built and raises."""
  from yasps_b200.graph import resolve_leaf_children
  cube = scenes.fem_cube(5, noise=0.01, seed=1)
  sc, h = scenes.fem_scene(cube)
  snh = next(r.energy for r in sc.minimizer.requests if r.energy.expr.kind == "snh")
  free_rest = resolve_leaf_children(snh.expr.rest.source)[0][-1]  # the free vertices' rest positions
  J = differentiator().diff2([snh], [h["free_position"]], [free_rest]).compute()
  tets = cube.tets.astype(np.int64)
  hl = oe.snh_hessian_with_rest(cube.positions_all()[tets], cube.rest_all()[tets], cube.mu, cube.lam, cube.dt)
  npin = cube.pinned_count
  free_code = np.where(tets >= npin, 2 + 3 * (tets - npin), 0)
  zero = np.zeros_like(free_code)
  rc = np.concatenate([free_code, zero], axis=1)
  ccode = np.concatenate([zero, free_code], axis=1)
  check(J, orj.dense(hl, rc, ccode, J.rows, J.cols), rc, ccode)
  with pytest.raises(NotImplementedError):
    differentiator().diff2([snh], [free_rest], [h["free_position"], free_rest]).compute()
