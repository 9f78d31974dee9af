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
  """Dense matrix from the block attributes (categories of (h, w) blocks)."""
  pos = J.block_positions.cpu().numpy().astype(np.int64).reshape(-1, 2)
  vals = J.blocks_flattened.cpu().numpy()
  D = np.zeros((J.rows, J.cols))
  b = 0
  for g, cnt in enumerate(J.block_counts):
    h, w = J.block_dimensions[2 * g:2 * g + 2]
    start = J.blocks_start_indices[g]
    for k in range(cnt):
      r, c = pos[b + k]
      D[r:r + h, c:c + w] += vals[start + k * h * w:start + (k + 1) * h * w].reshape(h, w)
    b += cnt
  return D, pos


def expected_positions(row_codes, col_codes):
  pairs = {(int(r) - 2, int(c) - 2) for rr, cc in zip(row_codes, col_codes) for r in rr if r >= 2 for c in cc if c >= 2}
  return np.array(sorted(pairs), dtype=np.int64).reshape(-1, 2)


def check(J, D_oracle, row_codes, col_codes):
  D, pos = device_dense(J)
  if row_codes is not None:
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
  against free rest positions), and rest positions against both (the
  rest-rest blocks d2E/dX2 among them), against the oracle's autograd
  Hessian over (x, X)."""
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
  # rows: rest positions; columns: positions, then rest positions
  J2 = differentiator().diff2([snh], [free_rest], [h["free_position"], free_rest]).compute()
  nfree = cube.free_count
  rest_code = np.where(tets >= npin, 2 + 3 * (tets - npin + nfree), 0)
  rc2 = np.concatenate([zero, free_code], axis=1)
  cc2 = np.concatenate([free_code, rest_code], axis=1)
  assert J2.rows == 3 * nfree and J2.cols == 6 * nfree
  check(J2, orj.dense(hl, rc2, cc2, J2.rows, J2.cols), rc2, cc2)


def material_scene(side=5):
  """A FEM cube whose tets carry their own Lame parameters (per-tet
  attributes), as the reference's material-optimization examples."""
  from yasps_b200.energies import inertia, stable_neo_hookean
  from yasps_b200.scene import scene as make_scene
  cube = scenes.fem_cube(side, noise=0.01, seed=6)
  rng = np.random.default_rng(1)
  sc = make_scene("material")
  body = sc.addMesh("body")
  pinned = body.addPrimitive("pinned", numInstances=cube.pinned_count)
  pp = pinned.addAttribute("position", rows=3, cols=1)
  pp.updateValue(cube.positions_all()[:cube.pinned_count])
  pr = pinned.addConstant("rest_position", rows=3, cols=1)
  pr.updateValue(cube.rest_all()[:cube.pinned_count])
  free = body.addPrimitive("free", numInstances=cube.free_count)
  fp = free.addAttribute("position", rows=3, cols=1)
  fp.updateValue(cube.free_position)
  fr = free.addConstant("rest_position", rows=3, cols=1)
  fr.updateValue(cube.rest_all()[cube.pinned_count:])
  last = free.addConstant("last_position", rows=3, cols=1)
  last.updateValue(cube.free_position + rng.uniform(-1e-3, 1e-3, size=cube.free_position.shape))
  vel = free.addConstant("velocity", rows=3, cols=1)
  vel.updateValue(rng.uniform(-0.1, 0.1, size=cube.free_position.shape))
  mass = free.addConstant("mass")
  mass.updateValue(cube.mass)
  verts = body.addPrimitiveUnion("vertices", [pinned, free])
  tets = body.addPrimitive("tetrahedra", numInstances=cube.tet_count)
  conn = tets.addConnectivity("to_vertices", verts, cube.tets.astype(np.uint32), 4)
  mu = tets.addConstant("mu")
  mu.updateValue(cube.mu * rng.uniform(0.5, 1.5, size=cube.tet_count))
  lam = tets.addConstant("lam")
  lam.updateValue(cube.lam * rng.uniform(0.5, 1.5, size=cube.tet_count))
  snh = tets.addAttribute("snh", computed_attribute=stable_neo_hookean(
      tets.addAttribute("rest", through=conn, source=verts.addAttribute("rest_position")),
      tets.addAttribute("x", through=conn, source=verts.addAttribute("position")), mu, lam, cube.dt))
  kin = free.addAttribute("inertia", computed_attribute=inertia(last, vel, cube.dt, fp, mass,
                                                                gravity=(0.0, 0.0, -9.8)))
  return cube, dict(snh=snh, inertia=kin, position=fp, mu=mu, lam=lam, mass=mass, last=last, vel=vel)


@pytest.mark.parametrize("which", ["mu", "lam"])
def test_snh_material_parameter_columns(which):
  """d2E/(dx d mu) and d2E/(dx d lambda) of SNH tets with per-tet Lame
  parameters (the reference's diff2(elastic, [position], [young]) of its
  material-optimization examples, here on the Lame arrays): (3 x 1) blocks
  against the oracle's autograd derivatives, and the products."""
  import torch
  cube, h = material_scene()
  J = differentiator().diff2([h["snh"]], [h["position"]], [h[which]]).compute()
  assert J.block_dimensions == [3, 1]
  tets = cube.tets.astype(np.int64)
  d = oe.snh_parameter_jacobian(cube.positions_all()[tets], cube.rest_all()[tets],
                                h["mu"].host_value.reshape(-1), h["lam"].host_value.reshape(-1), cube.dt,
                                0 if which == "mu" else 1)
  npin = cube.pinned_count
  D = np.zeros((J.rows, J.cols))
  for t in range(len(tets)):
    for a in range(4):
      if tets[t, a] >= npin:
        v = tets[t, a] - npin
        D[3 * v:3 * v + 3, t] += d[t, 3 * a:3 * a + 3]
  check(J, D, None, None)


def test_inertia_mass_column_beside_a_position_column():
  """d2E/(dx dm) of the inertia term (x - x~ per vertex, a (3 x 1) block)
  beside d2E/(dx dx_before) (-m I, 3 x 3) in one Jacobian: two block
  categories, the scalar columns first, products over both."""
  cube, h = material_scene()
  J = differentiator().diff2([h["inertia"]], [h["position"]], [h["mass"], h["last"]]).compute()
  assert J.block_dimensions == [3, 1, 3, 3]
  x = cube.free_position
  last = h["last"].host_value.reshape(-1, 3)
  vel = h["vel"].host_value.reshape(-1, 3)
  dt = cube.dt
  xt = last + vel * dt + np.array([0.0, 0.0, -9.8]) * dt * dt
  nf = cube.free_count
  D = np.zeros((J.rows, J.cols))
  for v in range(nf):
    D[3 * v:3 * v + 3, v] = x[v] - xt[v]
    D[3 * v:3 * v + 3, nf + 3 * v:nf + 3 * v + 3] = -cube.mass[v] * np.eye(3)
  check(J, D, None, None)


def test_first_order_jacobian_of_affine_vertex_positions():
  """diff1 of a vector-valued source: the affine-body vertex positions
  x_i = A_b xbar_i + t_b against the bodies' affine matrices (3 x 9 blocks,
  row r holding xbar_i) and translations (3 x 3 identities), as the
  reference's firstOrderJacobian; products in both directions."""
  from yasps_b200.jacobian import firstOrderJacobian
  from yasps_b200.scene import scene as make_scene
  bodies = scenes.affine_bodies(num_bodies=3, m=2, seed=3)
  sc = make_scene("abd_map")
  mesh = sc.addMesh("m")
  _, amat, trans, _, vpos = scenes._affine_body_attributes(mesh, bodies)
  J = differentiator().diff1(vpos, [amat, trans])
  assert isinstance(J, firstOrderJacobian)
  J.compute()
  assert J.block_dimensions == [3, 3, 3, 9]
  nv, nb = len(bodies.rest), bodies.num_bodies
  D = np.zeros((3 * nv, 12 * nb))
  for i in range(nv):
    b = int(bodies.vertex_body[i])
    for r in range(3):
      D[3 * i + r, 9 * b + 3 * r:9 * b + 3 * r + 3] = bodies.rest[i]
      D[3 * i + r, 9 * nb + 3 * b + r] = 1.0
  check(J, D, None, None)


def cloth_rest_local(kind, x, rest, conn, params):
  """Oracle local Hessians [n, 6A, 6A] of a cloth energy over (positions,
  rest positions) of each element, by autograd through the oracle's rest
  frame / rest dihedral."""
  import torch
  fn = {5: ve.bending, 6: ve.baraff_witkin, 7: ve.stvk_membrane}[kind]
  p = torch.tensor(params, dtype=torch.float64)
  out = []
  for q in conn:
    A = len(q)
    z0 = torch.tensor(np.concatenate([x[q], rest[q]]).ravel(), dtype=torch.float64)
    H = torch.autograd.functional.hessian(lambda z: fn(z[:3 * A].view(A, 3), z[3 * A:].view(A, 3), p), z0)
    out.append(H.numpy())
  return np.stack(out)


@pytest.mark.parametrize("membrane", ["baraff_witkin", "stvk"])
def test_cloth_energies_against_rest_positions(membrane):
  """Shape derivatives of the cloth energies through their rest quantities
  (rest frame and area of the membranes, rest dihedral and edge length of
  the bending): positions against rest positions per energy, and rest
  positions against both for the sum of the two, against autograd of the
  oracle formulas."""
  from tests.vertex_scene import VertexScene
  from yasps_b200.graph import resolve_leaf_children
  vs = VertexScene(m=5, seed=3, membrane=membrane)
  sc = vs.build()
  pos = sc.minimizer.wrt[0]
  es = {r.energy.expr.code: r.energy for r in sc.minimizer.requests
        if r.energy.expr.kind == "vertex" and r.energy.expr.code in (5, 6, 7)}
  rest = resolve_leaf_children(next(iter(es.values())).expr.rest.source)[0][-1]
  terms = {kind: (conn, params) for kind, conn, params, aux, _ in vs.terms() if kind in (5, 6, 7)}
  n3 = vs.n
  total = np.zeros((n3, 2 * n3))
  for kind, e in es.items():
    conn, params = terms[kind]
    hl = cloth_rest_local(kind, vs.x, vs.rest, conn, params)
    code = 2 + 3 * conn.astype(np.int64)
    zero = np.zeros_like(code)
    rc, cc = np.concatenate([code, zero], axis=1), np.concatenate([zero, code], axis=1)
    J = differentiator().diff2([e], [pos], [rest]).compute()
    check(J, orj.dense(hl, rc, cc, J.rows, J.cols), rc, cc)
    cc2 = np.concatenate([code, code + n3], axis=1)
    total += orj.dense(hl, np.concatenate([zero, code], axis=1), cc2, n3, 2 * n3)
  J2 = differentiator().diff2(list(es.values()), [rest], [pos, rest]).compute()
  assert J2.rows == n3 and J2.cols == 2 * n3
  check(J2, total, None, None)
