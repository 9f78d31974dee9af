"""Vertex-tuple energies (barriers, bending, membranes, friction) on the GPU
against the oracle, through the public scene API and the C ABI.

Tolerances: pattern and lookups bit-exact; FP64 gradient and projected
Hessian 1e-12 relative to the largest magnitude; solves at the stated true
relative residual.
"""

import numpy as np
import pytest

from oracle import solvers
from oracle import pattern as opattern
from tests.vertex_scene import VertexScene

pytestmark = pytest.mark.gpu


def rel(a, b):
  a, b = np.asarray(a), np.asarray(b)
  return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("membrane", ["baraff_witkin", "stvk"])
@pytest.mark.parametrize("method", [1, 2, 0])
def test_assembly_matches_oracle(membrane, method):
  vs = VertexScene(m=6, seed=3, membrane=membrane)
  sc = vs.build(projection_method=method)
  H = sc.minimizer.computeNumericValue()
  pat, values, grad = vs.oracle_assembly(projection_method=method)
  pos = H.block_positions.cpu().numpy().astype(np.int64).reshape(-1, 2)
  assert np.array_equal(pos, pat.positions)
  assert rel(H.gradient.value.cpu().numpy(), grad) <= 1e-12
  assert rel(H.blocks_flattened.cpu().numpy()[:values.size], values) <= 1e-12


def test_projection_changes_indefinite_terms():
  vs = VertexScene(m=6, seed=4)
  _, v_proj, _ = vs.oracle_assembly(projection_method=1)
  _, v_raw, _ = vs.oracle_assembly(projection_method=0)
  assert rel(v_proj, v_raw) > 1e-6, "the scene must exercise the projection"


def test_cloth_contact_solve():
  vs = VertexScene(m=8, seed=5)
  sc = vs.build(projection_method=1)
  sc.minimizer.setSolver("mas", stop_rule="residual")
  segs = sc.minimizeEnergy(tolerance=1e-8, maxIterations=2000)
  x = segs[0].cpu().numpy()
  pat, values, grad = vs.oracle_assembly(projection_method=1)
  matvec = lambda v: opattern.spmv(pat, values, v)
  assert solvers.relative_residual(matvec, grad, x) <= 1e-8


def test_cloth_over_obstacle_union_matches_oracle():
  """Contacts through a union [obstacle (DATA, not a target), cloth]: the
  obstacle slots carry code 1, take part in the projected local Hessians and
  are dropped at the scatter."""
  from oracle import pattern as op, projection
  from oracle import energies as oe
  from oracle import vertex_energies as ve
  from yasps_b200 import scenes
  cc = scenes.cloth_contact(side=7, pairs=40, seed=2)
  sc, _ = scenes.cloth_contact_scene(cc)
  H = sc.minimizer.computeNumericValue()
  no = len(cc.obstacle)
  allpos = np.concatenate([cc.obstacle, cc.cloth_position])
  n = 3 * len(cc.cloth_position)
  terms = [(7, no + cc.tris, (cc.mu, cc.lam, cc.thickness, cc.dt), np.concatenate([cc.obstacle, cc.cloth_rest]),
            None),
           (5, no + cc.bend, (cc.bend_stiff, cc.dt), np.concatenate([cc.obstacle, cc.cloth_rest]), None),
           (3, cc.pt.astype(np.int64), (cc.dhat, cc.kappa), None, None),
           (4, cc.ee.astype(np.int64), (cc.dhat, cc.kappa), None, None),
           (8, cc.pt.astype(np.int64), (cc.fdhat, cc.dt, cc.friction), allpos, cc.lagged)]
  coords, dims, per = [], [], []
  for kind, conn, params, aux, lag in terms:
    codes = np.where(conn >= no, 2 + 3 * (conn - no), 1)
    sizes = np.full_like(codes, 3)
    perm, _, _ = op.compress_slots(codes, sizes)
    c, d, o = op.coordinates(codes, sizes, perm)
    coords.append(c)
    dims.append(d)
    _, g, h = ve.energy_grad_hess(kind, allpos[conn], None if aux is None else aux[conn], params, lag)
    per.append((codes, sizes, perm, o, g, projection.project_spd(h, 1)))
  icodes = (2 + 3 * np.arange(len(cc.cloth_position), dtype=np.int64))[:, None]
  isizes = np.full_like(icodes, 3)
  iperm, _, _ = op.compress_slots(icodes, isizes)
  c, d, o = op.coordinates(icodes, isizes, iperm)
  coords.append(c)
  dims.append(d)
  xt = cc.cloth_position + np.array([0.0, -9.8, 0.0]) * cc.dt * cc.dt
  _, gi, hi = oe.inertia_local(cc.cloth_position, xt, cc.mass)
  per.append((icodes, isizes, iperm, o, gi, hi))
  pat = op.build_pattern(coords, dims)
  grad, values, diag = np.zeros(n), np.zeros(pat.total_values), np.zeros(3 * n)
  for k, (codes, sizes, perm, o, g, h) in enumerate(per):
    op.scatter_term(codes, sizes, perm, pat.lookups[k], o, g, h, grad, values, diag, [0, n], [0, 3 * n])
  pos = H.block_positions.cpu().numpy().astype(np.int64).reshape(-1, 2)
  assert np.array_equal(pos, pat.positions)
  assert rel(H.gradient.value.cpu().numpy(), grad) <= 1e-12
  assert rel(H.blocks_flattened.cpu().numpy()[:values.size], values) <= 1e-12
