"""Small contact scene with affine bodies and its oracle assembly (test helper).

Cloth vertices (targets), the vertices of two affine bodies (``A xbar + t``)
and a container (DATA) in the union ``[cloth, abd, container]``; barrier
pairs of every kind mixing the three, with dHat above every pair's squared
distance so that all terms are active.  ``oracle_assembly`` differentiates
each pair in its leaves, merges repeated leaves and projects the merged
matrix whole (:mod:`oracle.coupled_contact`), then scatters with the oracle
pattern.
"""

import numpy as np

from oracle import coupled_contact as cc
from oracle import pattern

KIND = {"pp": 1, "pe": 2, "pt": 3, "ee": 4}


def make(seed=0):
  from yasps_b200 import scenes
  rng = np.random.default_rng(seed)
  g = np.stack(np.meshgrid(np.arange(3), np.arange(3), indexing="ij"), axis=-1).reshape(-1, 2)
  cloth = np.stack([g[:, 0] * 0.2, rng.uniform(-0.02, 0.02, 9), g[:, 1] * 0.2], axis=1)
  bodies = scenes.affine_bodies(num_bodies=2, m=2, seed=seed, deform=0.05)
  bodies.translation = np.array([[0.1, 0.3, 0.1], [0.3, -0.25, 0.2]]) + rng.uniform(-0.01, 0.01, (2, 3))
  container = np.array([[0.0, -0.5, 0.0], [0.5, -0.5, 0.0], [0.0, -0.5, 0.5], [0.5, -0.45, 0.5]])
  nc, nv = len(cloth), len(bodies.rest)
  C = lambda i: i
  B = lambda b, i: nc + 8 * b + i
  O = lambda i: nc + nv + i
  pairs = {
      "pp": [[C(0), B(0, 1)], [B(0, 2), B(1, 5)], [C(4), O(1)]],
      "pe": [[C(1), B(0, 0), B(0, 3)], [B(1, 2), C(3), C(4)], [O(2), B(1, 0), B(1, 7)]],
      "pt": [[C(4), B(0, 0), B(0, 1), B(0, 2)], [B(1, 6), C(0), C(1), C(4)], [O(0), B(1, 1), B(1, 2), B(1, 4)],
             [C(8), O(0), O(1), O(2)], [B(0, 7), B(1, 0), B(1, 3), B(1, 5)]],
      "ee": [[C(2), C(5), B(0, 4), B(0, 6)], [B(0, 1), B(0, 7), B(1, 0), B(1, 6)], [B(1, 3), B(1, 4), O(0), O(3)]],
  }
  pairs = {k: np.asarray(v, dtype=np.uint32) for k, v in pairs.items()}
  allpos = np.concatenate([cloth, bodies.positions(), container])
  d = max(_squared_distance(KIND[k], allpos[c]) for k, v in pairs.items() for c in v)
  mass = np.full(nc, 0.05)
  return dict(cloth=cloth, bodies=bodies, container=container, pairs=pairs, dhat=2.0 * d, kappa=1.0, mass=mass)


def _squared_distance(kind, x):
  if kind == 1:
    return float(np.dot(x[1] - x[0], x[1] - x[0]))
  if kind == 2:
    c = np.cross(x[1] - x[0], x[2] - x[0])
    return float(np.dot(c, c) / np.dot(x[2] - x[1], x[2] - x[1]))
  if kind == 3:
    b = np.cross(x[2] - x[1], x[3] - x[1])
    return float(np.dot(x[0] - x[1], b) ** 2 / np.dot(b, b))
  b = np.cross(x[1] - x[0], x[3] - x[2])
  return float(np.dot(x[2] - x[0], b) ** 2 / np.dot(b, b))


FRICTION = {"pp": 11, "pe": 9, "pt": 8, "ee": 10}


def add_friction(s, seed=0):
  """Lagged friction over the same pairs: union positions at the start of
  the step a small seeded move away, the lagged data of each pair from them
  (the oracle's restatement of the reference's friction helpers)."""
  from oracle import vertex_energies as ve
  rng = np.random.default_rng(100 + seed)
  allpos = union_positions(s)
  last = allpos + rng.uniform(-2e-3, 2e-3, allpos.shape)
  lagged = {}
  for key, conn in s["pairs"].items():
    lagged[key] = np.stack([ve.LAGGED[FRICTION[key]](last[c.astype(np.int64)], s["dhat"], s["kappa"])
                            for c in conn])
  s["friction"] = dict(last=last, fdhat=1e-6, rate=0.3, lagged=lagged)
  return s


def union_positions(s):
  return np.concatenate([s["cloth"], s["bodies"].positions(), s["container"]])


def scene(s, method, separate_hessian_jacobian=False):
  from yasps_b200 import scenes
  fr = None
  if "friction" in s:
    f = s["friction"]
    fr = dict(last=f["last"], fdhat=f["fdhat"], rate=f["rate"])
    fr.update({k: (s["pairs"][k], f["lagged"][k]) for k in s["pairs"]})
  return scenes.contact_with_bodies_scene(s["cloth"], s["bodies"], s["container"], s["pairs"], s["dhat"],
                                          s["kappa"], projection_method=method, friction=fr,
                                          separate_hessian_jacobian=separate_hessian_jacobian)


def oracle_assembly(s, method):
  """(dense H, gradient, energy total) of the barrier terms (and the friction
  terms when the scene has them), targets [cloth, A (three rows a body), t]."""
  cloth, bodies, container = s["cloth"], s["bodies"], s["container"]
  nc, nv, nb = len(cloth), len(bodies.rest), bodies.num_bodies
  start_a, start_t = 3 * nc, 3 * nc + 9 * nb
  n = start_t + 3 * nb
  A = bodies.affine
  terms = []
  energy = 0.0
  kinds = [(key, arity, KIND[key]) for key, arity in (("pp", 2), ("pe", 3), ("pt", 4), ("ee", 4))]
  if "friction" in s:
    kinds += [(key, arity, FRICTION[key]) for key, arity in (("pp", 2), ("pe", 3), ("pt", 4), ("ee", 4))]
  last = s["friction"]["last"] if "friction" in s else None
  for key, arity, ekind in kinds:
    conn = s["pairs"][key].astype(np.int64)
    fric = ekind in FRICTION.values()
    K = 4 * arity
    codes_t = np.zeros((len(conn), K), dtype=np.int64)
    sizes_t = np.zeros((len(conn), K), dtype=np.int64)
    g_t = np.zeros((len(conn), 3 * K))
    h_t = np.zeros((len(conn), 3 * K, 3 * K))
    for e, row in enumerate(conn):
      verts, desc = [], []
      for idx in row:
        if idx < nc:
          verts.append(("p", cloth[idx]))
          desc.append(("p", int(idx)))
        elif idx < nc + nv:
          i = idx - nc
          b = int(bodies.vertex_body[i])
          verts.append(("a", A[b], bodies.translation[b], bodies.rest[i], b))
          desc.append(("a", b))
        else:
          verts.append(("p", container[idx - nc - nv]))
          desc.append(("d", 0))
      codes = []
      for kind, i in desc:
        if kind == "p":
          codes.extend([2 + 3 * i, 0, 0, 0])
        elif kind == "d":
          codes.extend([1, 0, 0, 0])
        else:
          codes.extend([start_a + 3 * (3 * i + r) + 2 for r in range(3)] + [start_t + 3 * i + 2])
      if fric:
        f = s["friction"]
        en, codes_c, sizes_c, g_c, h_c = cc.local_compressed(ekind, verts, np.asarray(codes),
                                                             (f["fdhat"], 0.01, f["rate"]), method,
                                                             lagged=f["lagged"][key][e], rest=last[row])
      else:
        en, codes_c, sizes_c, g_c, h_c = cc.local_compressed(ekind, verts, np.asarray(codes),
                                                             (s["dhat"], s["kappa"]), method)
      energy += en
      codes_t[e], sizes_t[e] = codes_c, sizes_c
      g_t[e, :g_c.size] = g_c
      h_t[e, :g_c.size, :g_c.size] = h_c
    terms.append((codes_t, sizes_t, g_t, h_t))
  coords, dims, per = [], [], []
  for codes, sizes, g, h in terms:
    perm, _, _ = pattern.compress_slots(codes, sizes)
    c, d, o = pattern.coordinates(codes, sizes, perm)
    coords.append(c)
    dims.append(d)
    per.append((codes, sizes, perm, o, g, h))
  pat = pattern.build_pattern(coords, dims)
  seg = [0, start_a, start_t, n]
  dstart = [0, 9 * n, 18 * n, 27 * n]  # diagonal blocks are not compared here
  grad, values, diag = np.zeros(n), np.zeros(pat.total_values), np.zeros(27 * n + 1)
  for k, (codes, sizes, perm, o, g, h) in enumerate(per):
    pattern.scatter_term(codes, sizes, perm, pat.lookups[k], o, g, h, grad, values, diag, seg, dstart)
  return pattern.dense_from_blocks(pat, values, n), grad, energy
