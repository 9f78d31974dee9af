"""A small cloth + contact scene for the vertex-tuple energies (test helper).

A sheet of ``m x m`` vertices in the xz plane (two triangles a quad) with a
membrane and dihedral bending, plus a cloud of free points hovering above it
at distances inside d-hat, coupled to the sheet by point-triangle,
edge-edge, point-edge and point-point barriers and by lagged friction of the
same four kinds.  Every vertex is a target (one primitive, no union).  ``build``
uses the public scene API; ``oracle_assembly`` assembles the same terms with
the oracle (same term order, same pattern rules).
"""

import numpy as np

from oracle import pattern, projection
from oracle import vertex_energies as ve


class VertexScene:
  def __init__(self, m=6, seed=0, membrane="baraff_witkin", dhat=1e-3, kappa=1e3, dt=0.01):
    rng = np.random.default_rng(seed)
    h = 0.1
    gi, gk = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    rest = np.stack([gi.ravel() * h, np.zeros(m * m), gk.ravel() * h], axis=1)
    x = rest + rng.uniform(-0.003, 0.003, size=rest.shape)
    x[:, 1] = rng.uniform(-0.002, 0.002, size=m * m)  # slight out-of-plane wrinkles
    tris = []
    for i in range(m - 1):
      for k in range(m - 1):
        a, b, c, d = i * m + k, (i + 1) * m + k, (i + 1) * m + k + 1, i * m + k + 1
        tris += [[a, c, b], [a, d, c]]  # normals along +y (the rest frame's singularity is -y)
    tris = np.asarray(tris)
    # interior edges: (e0, e1, opposite of tri 0, opposite of tri 1)
    edge_tris = {}
    for t, tri in enumerate(tris):
      for j in range(3):
        e = tuple(sorted((tri[j], tri[(j + 1) % 3])))
        edge_tris.setdefault(e, []).append((t, tri[(j + 2) % 3]))
    bend = [[e[0], e[1], v[0][1], v[1][1]] for e, v in edge_tris.items() if len(v) == 2]
    self.bend = np.asarray(bend)
    nsheet = m * m
    # hovering points: above random triangles at squared distance in (0.1, 0.9) dhat
    npts = 6
    cand = rng.choice(len(tris), size=npts, replace=False)
    pts, pts_rest = [], []
    for t in cand:
      c = x[tris[t]].mean(axis=0)
      n = np.cross(x[tris[t][1]] - x[tris[t][0]], x[tris[t][2]] - x[tris[t][0]])
      n /= np.linalg.norm(n)
      dist = np.sqrt(rng.uniform(0.1, 0.9) * dhat)
      pts.append(c + dist * n)
      pts_rest.append(rest[tris[t]].mean(axis=0) + dist * np.array([0.0, 1.0, 0.0]))
    self.x = np.concatenate([x, np.asarray(pts)])
    self.rest = np.concatenate([rest, np.asarray(pts_rest)])
    self.x_old = self.x + rng.uniform(-1e-4, 1e-4, size=self.x.shape)
    p_ids = nsheet + np.arange(npts)
    self.pt = np.stack([p_ids, *tris[cand].T], axis=1)
    # point-point / point-edge to the nearest sheet vertex / edge of the triangle
    self.pp = np.stack([p_ids, tris[cand][:, 0]], axis=1)
    self.pe = np.stack([p_ids, tris[cand][:, 0], tris[cand][:, 1]], axis=1)
    # edge-edge: point pairs as edges against a triangle edge below their midpoint
    self.ee = np.stack([p_ids[:-1:2], p_ids[1::2], tris[cand][:-1:2, 0], tris[cand][:-1:2, 2]], axis=1)
    self.tris = tris
    self.dhat, self.kappa, self.dt = dhat, kappa, dt
    self.membrane = membrane
    self.mem_params = (2000.0, 1000.0, 1e-3, dt) if membrane == "baraff_witkin" else (5e3, 2e3, 1e-3, dt)
    self.bend_params = (1e-3, dt)
    self.fric_params = (1e-6, dt, 0.3)
    self.lagged = np.stack([ve.lagged_friction_pt(self.x_old[q], dhat, kappa) for q in self.pt])
    self.lagged_pe = np.stack([ve.lagged_friction_pe(self.x_old[q], dhat, kappa) for q in self.pe])
    self.lagged_ee = np.stack([ve.lagged_friction_ee(self.x_old[q], dhat, kappa) for q in self.ee])
    self.lagged_pp = np.stack([ve.lagged_friction_pp(self.x_old[q], dhat, kappa) for q in self.pp])
    self.n = 3 * len(self.x)
    self.mass = np.full(len(self.x), 1e-3)
    self.gravity = np.array([0.0, -9.8, 0.0])

  # (kind, connectivity, params, uses rest/old positions, lagged)
  def terms(self):
    mem_kind = 6 if self.membrane == "baraff_witkin" else 7
    b = (self.dhat, self.kappa)
    return [(mem_kind, self.tris, self.mem_params, "rest", None),
            (5, self.bend, self.bend_params, "rest", None),
            (3, self.pt, b, None, None),
            (4, self.ee, b, None, None),
            (2, self.pe, b, None, None),
            (1, self.pp, b, None, None),
            (8, self.pt, self.fric_params, "old", self.lagged),
            (9, self.pe, self.fric_params, "old", self.lagged_pe),
            (10, self.ee, self.fric_params, "old", self.lagged_ee),
            (11, self.pp, self.fric_params, "old", self.lagged_pp)]

  def build(self, projection_method=1):
    from yasps_b200 import energies as E
    from yasps_b200.scene import scene as make_scene
    sc = make_scene("cloth_contact")
    mesh = sc.addMesh("cloth")
    verts = mesh.addPrimitive("vertices", numInstances=len(self.x))
    pos = verts.addAttribute("position", rows=3, cols=1)
    pos.updateValue(self.x)
    rest = verts.addConstant("rest_position", rows=3, cols=1)
    rest.updateValue(self.rest)
    old = verts.addConstant("old_position", rows=3, cols=1)
    old.updateValue(self.x_old)
    for idx, (kind, conn, params, aux, lag) in enumerate(self.terms()):
      prim = mesh.addPrimitive(f"t{idx}", numInstances=len(conn))
      c = prim.addConnectivity("to_vertices", verts, conn.astype(np.uint32), conn.shape[1])
      xj = prim.addAttribute("x", through=c, source=pos)
      aux_att = None
      if aux is not None:
        aux_att = prim.addAttribute("aux", through=c, source=rest if aux == "rest" else old)
      if kind == 1:
        e = E.point_point(xj, *params)
      elif kind == 2:
        e = E.point_edge(xj, *params)
      elif kind == 3:
        e = E.point_triangle(xj, *params)
      elif kind == 4:
        e = E.edge_edge(xj, *params)
      elif kind == 5:
        e = E.bending(xj, aux_att, *params)
      elif kind == 6:
        e = E.baraff_witkin(aux_att, xj, *params)
      elif kind == 7:
        e = E.stvk_membrane(aux_att, xj, *params)
      else:
        lagged = prim.addConstant("lagged", rows=9, cols=1)
        lagged.updateValue(lag)
        fric = {8: E.friction_point_triangle, 9: E.friction_point_edge, 10: E.friction_edge_edge,
                11: E.friction_point_point}[kind]
        e = fric(xj, aux_att, *params, lagged)
      att = prim.addAttribute("energy", computed_attribute=e)
      sc.addEnergy(att, projection_method=projection_method)
    mass = verts.addConstant("mass")
    mass.updateValue(self.mass)
    kin = verts.addAttribute("inertia", computed_attribute=E.inertia(old, None, self.dt, pos, mass,
                                                                        gravity=tuple(self.gravity)))
    sc.addEnergy(kin, projection_method=-1)
    sc.addMinimizeTarget([pos])
    return sc

  def oracle_assembly(self, projection_method=1):
    """Pattern, block values and gradient assembled by the oracle."""
    coords, dims, per_term = [], [], []
    for kind, conn, params, aux, lag in self.terms():
      codes = 2 + 3 * conn.astype(np.int64)
      sizes = np.full_like(codes, 3)
      perm, _, _ = pattern.compress_slots(codes, sizes)
      c, d, o = pattern.coordinates(codes, sizes, perm)
      coords.append(c)
      dims.append(d)
      src = None if aux is None else (self.rest if aux == "rest" else self.x_old)
      e, g, h = ve.energy_grad_hess(kind, self.x[conn], None if src is None else src[conn], params, lag)
      if projection_method >= 1:
        h = projection.project_spd(h, projection_method)
      per_term.append((codes, sizes, perm, o, g, h))
    from oracle import energies as oe
    icodes = (2 + 3 * np.arange(len(self.x), dtype=np.int64))[:, None]
    isizes = np.full_like(icodes, 3)
    iperm, _, _ = pattern.compress_slots(icodes, isizes)
    c, d, o = pattern.coordinates(icodes, isizes, iperm)
    coords.append(c)
    dims.append(d)
    x_tilde = self.x_old + self.gravity[None] * self.dt * self.dt
    _, gi, hi = oe.inertia_local(self.x, x_tilde, self.mass)
    per_term.append((icodes, isizes, iperm, o, gi, hi))
    pat = pattern.build_pattern(coords, dims)
    grad = np.zeros(self.n)
    values = np.zeros(pat.total_values)
    diag = np.zeros(3 * self.n)
    for k, (codes, sizes, perm, o, g, h) in enumerate(per_term):
      pattern.scatter_term(codes, sizes, perm, pat.lookups[k], o, g, h, grad, values, diag, [0, self.n],
                           [0, 3 * self.n])
    return pat, values, grad
