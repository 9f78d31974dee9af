"""Dynamic contact terms: the pair set changes between computes (as the
reference's `updateNumInstances` / `updateConnectivity` test does,
tests/differentiator/test_hessian_sparsity_permutation_gpu.py:230-280);
the dynamic pattern is rebuilt every compute and the static + dynamic
assembly matches the oracle's dense matrix each time (1e-12)."""

import numpy as np
import pytest

from oracle import pattern as op, projection, solvers
from oracle import energies as oe
from oracle import vertex_energies as ve
from tests.vertex_scene import VertexScene

pytestmark = pytest.mark.gpu


def dense_of(H):
  n = H.rows
  out = np.zeros((n, n))
  for suffix in ("", "_dynamic"):
    counts = getattr(H, "block_counts" + suffix)
    if not counts:
      continue
    dims = getattr(H, "block_dimensions" + suffix)
    starts = getattr(H, "blocks_start_indices" + suffix)
    pos = getattr(H, "block_positions" + suffix).cpu().numpy().astype(np.int64)[:2 * sum(counts)].reshape(-1, 2)
    vals = getattr(H, "blocks_flattened" + suffix).cpu().numpy()
    c0 = 0
    for g, cnt in enumerate(counts):
      h, w = dims[2 * g:2 * g + 2]
      for b in range(cnt):
        r, c = pos[c0 + b]
        blk = vals[starts[g] + b * h * w:starts[g] + (b + 1) * h * w].reshape(h, w)
        out[r:r + h, c:c + w] += blk
        if r != c:
          out[c:c + w, r:r + h] += blk.T
      c0 += cnt
  return out


def oracle_dense(vs, pairs):
  n = vs.n
  H = np.zeros((n, n))
  g = np.zeros(n)

  def add(kind, conn, params, src, lag):
    if len(conn) == 0:
      return
    _, gl, hl = ve.energy_grad_hess(kind, vs.x[conn], None if src is None else src[conn], params, lag)
    hl = projection.project_spd(hl, 1)
    for t, c in enumerate(conn):
      idx = (3 * np.asarray(c)[:, None] + np.arange(3)).ravel()
      np.add.at(H, (idx[:, None], idx[None, :]), hl[t])
      np.add.at(g, idx, gl[t])

  add(6, vs.tris, vs.mem_params, vs.rest, None)
  add(3, pairs, (vs.dhat, vs.kappa), None, None)
  x_tilde = vs.x_old + vs.gravity[None] * vs.dt * vs.dt
  _, gi, hi = oe.inertia_local(vs.x, x_tilde, vs.mass)
  for v in range(len(vs.x)):
    H[3 * v:3 * v + 3, 3 * v:3 * v + 3] += hi[v]
    g[3 * v:3 * v + 3] += gi[v]
  return H, g


def test_dynamic_pairs_rebuild_their_pattern():
  from yasps_b200 import energies as E
  from yasps_b200.scene import scene as make_scene
  vs = VertexScene(m=6, seed=8)
  sc = make_scene("dynamic_contacts")
  mesh = sc.addMesh("cloth")
  verts = mesh.addPrimitive("vertices", numInstances=len(vs.x))
  pos = verts.addAttribute("position", rows=3, cols=1)
  pos.updateValue(vs.x)
  rest = verts.addConstant("rest_position", rows=3, cols=1)
  rest.updateValue(vs.rest)
  old = verts.addConstant("old_position", rows=3, cols=1)
  old.updateValue(vs.x_old)
  mass = verts.addConstant("mass")
  mass.updateValue(vs.mass)
  tri = mesh.addPrimitive("tris", numInstances=len(vs.tris))
  tc = tri.addConnectivity("to_vertices", verts, vs.tris.astype(np.uint32), 3)
  mem = tri.addAttribute("membrane", computed_attribute=E.baraff_witkin(
      tri.addAttribute("rest", through=tc, source=rest), tri.addAttribute("x", through=tc, source=pos),
      *vs.mem_params))
  pairs = mesh.addPrimitive("pairs", numInstances=len(vs.pt), isDynamic=True)
  pc = pairs.addConnectivity("to_vertices", verts, vs.pt.astype(np.uint32), 4)
  bar = pairs.addAttribute("barrier", computed_attribute=E.point_triangle(
      pairs.addAttribute("x", through=pc, source=pos), vs.dhat, vs.kappa))
  kin = verts.addAttribute("inertia", computed_attribute=E.inertia(old, None, vs.dt, pos, mass,
                                                                      gravity=tuple(vs.gravity)))
  sc.addEnergy(mem, projection_method=1)
  sc.addEnergy(bar, projection_method=1, dynamic_instances=True)
  sc.addEnergy(kin, projection_method=-1)
  sc.addMinimizeTarget([pos])
  sc.minimizer.setSolver("jacobian", stop_rule="residual")
  for active in (vs.pt, vs.pt[:3], vs.pt[:0], vs.pt[::-1][:4]):
    pairs.updateNumInstances(len(active))
    if len(active):
      pc.updateConnectivity(active.astype(np.uint32))
    H = sc.minimizer.computeNumericValue()
    exp_h, exp_g = oracle_dense(vs, active)
    assert np.abs(dense_of(H) - exp_h).max() <= 1e-12 * np.abs(exp_h).max()
    assert np.abs(H.gradient.value.cpu().numpy() - exp_g).max() <= 1e-12 * np.abs(exp_g).max()
    segs = sc.minimizeEnergy(tolerance=1e-10, maxIterations=5000)
    x = segs[0].cpu().numpy()
    assert np.linalg.norm(exp_h @ x - exp_g) <= 1e-10 * np.linalg.norm(exp_g)


def test_mas_with_a_dynamic_contact_set():
  """MAS over a static and a dynamic block set: the hierarchy is built on the
  static graph (the reference's default) and the dynamic blocks enter the
  domain matrices of every level, as the reference's numeric assembly over
  both sets does (mas/numeric_assembly.py:64-83).  The device MAS apply
  equals the oracle MAS on the same hierarchy with every block (FP32
  inverses: 2e-4; the fine-level weight raised as the reference's runtime
  does for dense contact sets), and the MAS PCG meets the oracle system's
  residual, as the pair set changes."""
  import torch
  from oracle import mas as omas
  from yasps_b200 import _lib as L
  from yasps_b200 import energies as E
  from yasps_b200.scene import scene as make_scene
  vs = VertexScene(m=6, seed=8)
  sc = make_scene("dynamic_contacts_mas")
  mesh = sc.addMesh("cloth")
  verts = mesh.addPrimitive("vertices", numInstances=len(vs.x))
  pos = verts.addAttribute("position", rows=3, cols=1)
  pos.updateValue(vs.x)
  rest = verts.addConstant("rest_position", rows=3, cols=1)
  rest.updateValue(vs.rest)
  old = verts.addConstant("old_position", rows=3, cols=1)
  old.updateValue(vs.x_old)
  mass = verts.addConstant("mass")
  mass.updateValue(vs.mass)
  tri = mesh.addPrimitive("tris", numInstances=len(vs.tris))
  tc = tri.addConnectivity("to_vertices", verts, vs.tris.astype(np.uint32), 3)
  mem = tri.addAttribute("membrane", computed_attribute=E.baraff_witkin(
      tri.addAttribute("rest", through=tc, source=rest), tri.addAttribute("x", through=tc, source=pos),
      *vs.mem_params))
  pairs = mesh.addPrimitive("pairs", numInstances=len(vs.pt), isDynamic=True)
  pc = pairs.addConnectivity("to_vertices", verts, vs.pt.astype(np.uint32), 4)
  bar = pairs.addAttribute("barrier", computed_attribute=E.point_triangle(
      pairs.addAttribute("x", through=pc, source=pos), vs.dhat, vs.kappa))
  kin = verts.addAttribute("inertia", computed_attribute=E.inertia(old, None, vs.dt, pos, mass,
                                                                      gravity=tuple(vs.gravity)))
  sc.addEnergy(mem, projection_method=1)
  sc.addEnergy(bar, projection_method=1, dynamic_instances=True)
  sc.addEnergy(kin, projection_method=-1)
  sc.addMinimizeTarget([pos])
  sc.minimizer.setSolver("mas", fine_level_weight=1.0, stop_rule="residual")
  nv = len(vs.x)
  for active in (vs.pt, vs.pt[:3], vs.pt[::-1][:4]):
    pairs.updateNumInstances(len(active))
    pc.updateConnectivity(active.astype(np.uint32))
    H = sc.minimizer.computeNumericValue()
    exp_h, exp_g = oracle_dense(vs, active)
    ms = sc.minimizer.linearSolver.implementation
    ms._ensure_hierarchy(H)
    assert len(H.block_sets) == 2 and ms._union is not None
    assert ms.numeric_update(H) == 0
    r = np.cos(np.arange(H.rows) * 0.37)
    rt = torch.from_numpy(r).cuda()
    z = torch.zeros_like(rt)
    L.call("ys_mas_apply", ms._mas, L.ptr(rt), L.ptr(z), L.stream_ptr())
    spos = H.block_sets[0].pattern
    sp = spos.positions[:2 * spos.num_unique].cpu().numpy().astype(np.int64).reshape(-1, 2)
    h = omas.build_hierarchy(np.full(nv, 3), [(a // 3, b // 3) for a, b in sp if a != b])
    blocks = [(a, b, exp_h[3 * a:3 * a + 3, 3 * b:3 * b + 3]) for a in range(nv) for b in range(a, nv)
              if np.any(exp_h[3 * a:3 * a + 3, 3 * b:3 * b + 3] != 0.0)]
    # the reference raises the fine-level weight for dense contact sets
    # (>= 0.1 dynamic blocks per fine variable: 3.0, mas/cuda_runtime.py:2716-2731)
    nl = len(h.levels)
    weights = list((1.0,) * (nl - 1) + (2.5,))
    if H.block_sets[1].pattern.num_unique / nv >= 0.1:
      weights[0] = max(weights[0], 3.0)
    assert ms.active_fine_level_weight == weights[0]
    pre = omas.MASPreconditioner(h, omas.level_local_matrices(h, blocks), level_weights=weights)
    ref = pre.apply(r)
    assert np.linalg.norm(z.cpu().numpy() - ref) <= 2e-4 * np.linalg.norm(ref)
    segs = sc.minimizeEnergy(tolerance=1e-10, maxIterations=5000)
    x = segs[0].cpu().numpy()
    assert np.linalg.norm(exp_h @ x - exp_g) <= 1e-10 * np.linalg.norm(exp_g)
