"""Seeded synthetic workloads (FEM cubes) in the reference's scene idiom.

The cube follows the FEM workloads of this project: an ``n x n x n`` vertex
grid with spacing ``h``, every hexahedron split into six tetrahedra with the
reference's cube split (``tests/energy/test_stable_neo_hookean.py:28-30``,
``[[0,1,3,7],[1,2,3,7],[0,1,4,7],[1,5,4,7],[1,2,6,7],[1,5,6,7]]``, which is
conforming across hexahedra), tetrahedra oriented to a positive rest volume,
positions = rest + U(-noise, noise) from ``numpy.random.default_rng(seed)``.

The ``z = 0`` layer is a separate *non-target* DATA primitive stacked before
the free vertices in a primitive union ``[pinned, free]`` (the reference
idiom, ``examples/one_bunny_partial_abd``), so pinned vertices take part in
each element's 12x12 projection but are not unknowns.  Both primitives are
numbered in Morton (Z-order) of their grid coordinates, which makes chunks of
32 consecutive free vertices the 32-vertex Morton domains used by MAS, and
the tetrahedra are ordered by the Morton code of their hexahedron.
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import lru_cache

import numpy as np

# Reference cube corner numbering: 0 (0,0,0) 1 (1,0,0) 2 (1,1,0) 3 (0,1,0)
# 4 (0,0,1) 5 (1,0,1) 6 (1,1,1) 7 (0,1,1).
_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
_SPLIT = np.array([[0, 1, 3, 7], [1, 2, 3, 7], [0, 1, 4, 7], [1, 5, 4, 7], [1, 2, 6, 7], [1, 5, 6, 7]])


def morton3(i, j, k):
  """Interleave the bits of three non-negative integer arrays (x lowest)."""
  def spread(v):
    v = np.asarray(v, dtype=np.uint64) & np.uint64(0x1FFFFF)
    v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
    return v
  return spread(i) | (spread(j) << np.uint64(1)) | (spread(k) << np.uint64(2))


def lame(young, poisson):
  mu = young / (2.0 * (1.0 + poisson))
  lam = young * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson))
  return mu, lam


@dataclass
class FemCube:
  """Arrays of one FEM cube scene (union order: pinned first, then free)."""

  n: int
  spacing: float
  pinned_rest: np.ndarray      # (np, 3)
  free_rest: np.ndarray        # (nf, 3)
  pinned_position: np.ndarray  # (np, 3)
  free_position: np.ndarray    # (nf, 3)
  tets: np.ndarray             # (nt, 4) uint32 union indices
  mass: np.ndarray             # (nf,) lumped masses of the free vertices
  velocity: np.ndarray         # (nf, 3)
  mu: float
  lam: float
  density: float
  dt: float
  gravity: np.ndarray

  @property
  def pinned_count(self) -> int:
    return int(self.pinned_rest.shape[0])

  @property
  def free_count(self) -> int:
    return int(self.free_rest.shape[0])

  @property
  def tet_count(self) -> int:
    return int(self.tets.shape[0])

  @property
  def dofs(self) -> int:
    return 3 * self.free_count

  def positions_all(self) -> np.ndarray:
    return np.concatenate([self.pinned_position, self.free_position])

  def rest_all(self) -> np.ndarray:
    return np.concatenate([self.pinned_rest, self.free_rest])

  def free_positions(self) -> np.ndarray:
    return self.free_position

  def x_tilde(self) -> np.ndarray:
    """Inertia target ``x_before + v dt + g dt^2`` with ``x_before`` the current state."""
    return self.free_position + self.velocity * self.dt + self.gravity[None] * self.dt * self.dt

  def snh_slots(self):
    """Per-tet index slots ``[child, pad] x 4`` of the union path (codes, sizes)."""
    t = self.tets.astype(np.int64)
    codes = np.zeros((t.shape[0], 8), dtype=np.int64)
    sizes = np.zeros((t.shape[0], 8), dtype=np.int64)
    free = t >= self.pinned_count
    codes[:, 0::2] = np.where(free, 2 + 3 * (t - self.pinned_count), 1)
    sizes[:, 0::2] = 3
    return codes, sizes

  def inertia_slots(self):
    codes = (2 + 3 * np.arange(self.free_count, dtype=np.int64))[:, None]
    return codes, np.full_like(codes, 3)


def fem_scene(cube: "FemCube", name: str = "fem_cube", projection_method: int = 1):
  """Build the cube with the public scene API (the reference example idiom).

  Returns ``(scene, handles)`` where ``handles`` maps names to the attributes
  a Newton loop updates (``free_position``, ``pinned_position``, ...).
  """
  from .energies import inertia, stable_neo_hookean
  from .scene import scene as make_scene

  sc = make_scene(name)
  dt = sc.addConstant("dt")
  dt.updateValue(cube.dt)
  mu = sc.addConstant("mu")
  mu.updateValue(cube.mu)
  lam = sc.addConstant("lam")
  lam.updateValue(cube.lam)
  body = sc.addMesh("body")
  pinned = body.addPrimitive("pinned", numInstances=cube.pinned_count)
  pinned_position = pinned.addAttribute("position", rows=3, cols=1)
  pinned_position.updateValue(cube.pinned_position)
  pinned_rest = pinned.addConstant("rest_position", rows=3, cols=1)
  pinned_rest.updateValue(cube.pinned_rest)
  free = body.addPrimitive("free", numInstances=cube.free_count)
  free_position = free.addAttribute("position", rows=3, cols=1)
  free_position.updateValue(cube.free_position)
  free_rest = free.addConstant("rest_position", rows=3, cols=1)
  free_rest.updateValue(cube.free_rest)
  last = free.addConstant("last_position", rows=3, cols=1)
  last.updateValue(cube.free_position)
  vel = free.addConstant("velocity", rows=3, cols=1)
  vel.updateValue(cube.velocity)
  mass = free.addConstant("mass")
  mass.updateValue(cube.mass)
  verts = body.addPrimitiveUnion("vertices", [pinned, free])
  position = verts.addAttribute("position")
  rest = verts.addAttribute("rest_position")
  tets = body.addPrimitive("tetrahedra", numInstances=cube.tet_count)
  to_verts = tets.addConnectivity("to_vertices", verts, cube.tets, 4)
  tet_position = tets.addAttribute("position", through=to_verts, source=position)
  tet_rest = tets.addAttribute("rest_position", through=to_verts, source=rest)
  snh = tets.addAttribute("snh", computed_attribute=stable_neo_hookean(tet_rest, tet_position, mu, lam, dt))
  kin = free.addAttribute("inertia", computed_attribute=inertia(last, vel, dt, free_position, mass,
                                                                 gravity=tuple(cube.gravity)))
  sc.addEnergy(snh, projection_method=projection_method)
  sc.addEnergy(kin, projection_method=-1)
  sc.addMinimizeTarget([free_position])
  return sc, dict(free_position=free_position, pinned_position=pinned_position, last_position=last, velocity=vel,
                  snh=snh, inertia=kin, tets=tets)


@lru_cache(maxsize=64)
def _vertex_order(n: int):
  """Lexicographic grid coordinates and the pinned / free vertex orders of an
  ``n^3`` cube (Morton order within each primitive, as in ``fem_cube``)."""
  g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), axis=-1).reshape(-1, 3)
  codes = morton3(g[:, 0], g[:, 1], g[:, 2])
  pinned = g[:, 2] == 0
  pin_ids = np.flatnonzero(pinned)[np.argsort(codes[pinned], kind="stable")]
  free_ids = np.flatnonzero(~pinned)[np.argsort(codes[~pinned], kind="stable")]
  return g, pin_ids, free_ids


def fem_positions(n: int, spacing: float = 0.1, noise: float = 0.01, seed: int = 0):
  """``(pinned_position, free_position)`` of ``fem_cube(n, spacing=spacing,
  noise=noise, seed=seed)`` without rebuilding the mesh (same draws)."""
  g, pin_ids, free_ids = _vertex_order(n)
  rng = np.random.default_rng(seed)
  pos_lex = g.astype(np.float64) * spacing + rng.uniform(-noise, noise, size=g.shape)
  return pos_lex[pin_ids], pos_lex[free_ids]


def fem_cube(n: int, spacing: float = 0.1, young: float = 1e5, poisson: float = 0.4, noise: float = 0.01,
             seed: int = 0, density: float = 1000.0, dt: float = 0.01,
             gravity=(0.0, 0.0, -9.8)) -> FemCube:
  """Build the ``n^3`` FEM cube workload (see module docstring)."""
  if n < 2:
    raise ValueError("fem_cube needs at least 2 vertices per side")
  g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), axis=-1).reshape(-1, 3)
  lex = g[:, 0] * n * n + g[:, 1] * n + g[:, 2]
  rng = np.random.default_rng(seed)
  rest_lex = g.astype(np.float64) * spacing
  pos_lex = rest_lex + rng.uniform(-noise, noise, size=rest_lex.shape)
  codes = morton3(g[:, 0], g[:, 1], g[:, 2])
  pinned = g[:, 2] == 0
  pin_ids = np.flatnonzero(pinned)[np.argsort(codes[pinned], kind="stable")]
  free_ids = np.flatnonzero(~pinned)[np.argsort(codes[~pinned], kind="stable")]
  union_of_lex = np.empty(n ** 3, dtype=np.int64)
  union_of_lex[lex[pin_ids]] = np.arange(pin_ids.size)
  union_of_lex[lex[free_ids]] = pin_ids.size + np.arange(free_ids.size)
  h = np.stack(np.meshgrid(np.arange(n - 1), np.arange(n - 1), np.arange(n - 1), indexing="ij"), axis=-1).reshape(-1, 3)
  h = h[np.argsort(morton3(h[:, 0], h[:, 1], h[:, 2]), kind="stable")]
  corner = h[:, None, :] + _CORNERS[None]
  corner_lex = corner[..., 0] * n * n + corner[..., 1] * n + corner[..., 2]
  tets_lex = corner_lex[:, _SPLIT].reshape(-1, 4)
  r = rest_lex[tets_lex]
  det = np.linalg.det(np.stack([r[:, 1] - r[:, 0], r[:, 2] - r[:, 0], r[:, 3] - r[:, 0]], axis=2))
  flip = det < 0
  tets_lex[flip, 2], tets_lex[flip, 3] = tets_lex[flip, 3].copy(), tets_lex[flip, 2].copy()
  vol = np.abs(det) / 6.0
  vmass = np.zeros(n ** 3)
  np.add.at(vmass, tets_lex.ravel(), np.repeat(density * vol / 4.0, 4))
  mu, lam = lame(young, poisson)
  return FemCube(
      n=n, spacing=spacing,
      pinned_rest=rest_lex[pin_ids], free_rest=rest_lex[free_ids],
      pinned_position=pos_lex[pin_ids], free_position=pos_lex[free_ids],
      tets=union_of_lex[tets_lex].astype(np.uint32), mass=vmass[free_ids],
      velocity=np.zeros((free_ids.size, 3)), mu=mu, lam=lam, density=density, dt=dt,
      gravity=np.asarray(gravity, dtype=np.float64))


# ---- affine (ABD) bodies beside a soft cube ---------------------------------------------

@dataclass
class AffineBodies:
  """Arrays of ``num_bodies`` affine bodies: each an ``m^3`` lattice of tets
  (the cube split above) in its body frame, placed by ``A xbar + t``."""

  rest: np.ndarray          # (nv, 3) body-frame rest positions xbar
  vertex_body: np.ndarray   # (nv,) body of each vertex
  tets: np.ndarray          # (nt, 4) uint32 vertex indices (one body each)
  affine: np.ndarray        # (nb, 9) A per body, row-major
  translation: np.ndarray   # (nb, 3)
  mass: np.ndarray          # (nv,) lumped masses
  velocity: np.ndarray      # (nv, 3)
  mu: float
  lam: float
  stiffness: float          # orthogonality scale
  dt: float
  gravity: np.ndarray

  @property
  def num_bodies(self) -> int:
    return int(self.affine.shape[0])

  def positions(self) -> np.ndarray:
    a = self.affine.reshape(-1, 3, 3)[self.vertex_body]
    return np.einsum("vrc,vc->vr", a, self.rest) + self.translation[self.vertex_body]


def affine_bodies(num_bodies: int = 4, m: int = 3, spacing: float = 0.1, young: float = 1e7, poisson: float = 0.3,
                  stiffness: float = 1e5, deform: float = 0.02, seed: int = 0, density: float = 1000.0,
                  dt: float = 0.01, gravity=(0.0, 0.0, -9.8)) -> AffineBodies:
  """Seeded affine bodies: A = R (I + S), R a random rotation, S symmetric with
  entries U(-deform, deform); t spaced along x above the soft cube."""
  rng = np.random.default_rng(seed)
  g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), axis=-1).reshape(-1, 3)
  xbar = (g - (m - 1) / 2.0) * spacing
  h = np.stack(np.meshgrid(np.arange(m - 1), np.arange(m - 1), np.arange(m - 1), indexing="ij"), axis=-1).reshape(-1, 3)
  corner = h[:, None, :] + _CORNERS[None]
  lex = corner[..., 0] * m * m + corner[..., 1] * m + corner[..., 2]
  tl = lex[:, _SPLIT].reshape(-1, 4)
  r = xbar[tl]
  det = np.linalg.det(np.stack([r[:, 1] - r[:, 0], r[:, 2] - r[:, 0], r[:, 3] - r[:, 0]], axis=2))
  flip = det < 0
  tl[flip, 2], tl[flip, 3] = tl[flip, 3].copy(), tl[flip, 2].copy()
  vmass = np.zeros(m ** 3)
  np.add.at(vmass, tl.ravel(), np.repeat(density * np.abs(det) / 24.0, 4))
  nv = m ** 3
  affine, trans = [], []
  for b in range(num_bodies):
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if np.linalg.det(q) < 0:
      q[:, 0] = -q[:, 0]
    sym = rng.uniform(-deform, deform, size=(3, 3))
    affine.append((q @ (np.eye(3) + 0.5 * (sym + sym.T))).ravel())
    trans.append([0.4 * b, 0.0, 1.0] + rng.uniform(-0.01, 0.01, size=3))
  mu, lam = lame(young, poisson)
  return AffineBodies(
      rest=np.tile(xbar, (num_bodies, 1)), vertex_body=np.repeat(np.arange(num_bodies), nv),
      tets=(tl[None] + nv * np.arange(num_bodies)[:, None, None]).reshape(-1, 4).astype(np.uint32),
      affine=np.asarray(affine), translation=np.asarray(trans), mass=np.tile(vmass, num_bodies),
      velocity=rng.uniform(-0.01, 0.01, size=(num_bodies * nv, 3)), mu=mu, lam=lam, stiffness=stiffness, dt=dt,
      gravity=np.asarray(gravity, dtype=np.float64))


def affine_scene(cube: "FemCube", bodies: AffineBodies, name: str = "soft_and_affine", projection_method: int = 1):
  """The soft cube of :func:`fem_scene` plus affine bodies, built the way
  ``examples/dropping_in_container_mixed/dropping_in_container.py:235-405``
  builds its ABD bunnies: body attributes ``affine_matrices`` (3x3) and
  ``translations``, vertex positions ``A xbar + t`` through a vertex-to-body
  connectivity, inertia of the body vertices, Stable Neo-Hookean of the body
  tets, the orthogonality energy of the bodies, and the targets
  ``[soft positions, affine_matrices, translations]``.
  """
  from .energies import affine_energy, affine_position, inertia, stable_neo_hookean
  sc, hd = fem_scene(cube, name, projection_method)
  dt = sc["dt"]
  abd = sc.addMesh("bodies_abd")
  prims = abd.addPrimitive("affine_bodies", numInstances=bodies.num_bodies)
  affine_matrices = prims.addAttribute("affine_matrices", rows=3, cols=3)
  affine_matrices.updateValue(bodies.affine)
  translations = prims.addAttribute("translations", rows=3, cols=1)
  translations.updateValue(bodies.translation)
  nv = bodies.rest.shape[0]
  verts = abd.addPrimitive("vertices_abd", numInstances=nv)
  rest = verts.addConstant("rest_position", rows=3, cols=1)
  rest.updateValue(bodies.rest)
  last = verts.addConstant("last_position", rows=3, cols=1)
  last.updateValue(bodies.positions())
  vel = verts.addConstant("velocity", rows=3, cols=1)
  vel.updateValue(bodies.velocity)
  mass = verts.addConstant("mass")
  mass.updateValue(bodies.mass)
  v2b = verts.addConnectivity("v_abd2_abd", prims, bodies.vertex_body[:, None].astype(np.uint32), 1)
  va = verts.addAttribute("affine_matrix", through=v2b, source=affine_matrices).resize(3, 3)
  vt = verts.addAttribute("translation", through=v2b, source=translations).resize(3, 1)
  vpos = verts.addAttribute("position", computed_attribute=affine_position(va, rest, vt))
  tets = abd.addPrimitive("tets_abd", numInstances=bodies.tets.shape[0])
  t2v = tets.addConnectivity("tets_abds2_vertices", verts, bodies.tets, 4)
  tpos = tets.addAttribute("positions", through=t2v, source=vpos)
  trest = tets.addAttribute("rest_positions", through=t2v, source=rest)
  snh = tets.addAttribute("snh_abds", computed_attribute=stable_neo_hookean(trest, tpos, bodies.mu, bodies.lam, dt))
  kin = verts.addAttribute("inertia_abds", computed_attribute=inertia(last, vel, dt, vpos, mass,
                                                                       gravity=tuple(bodies.gravity)))
  ortho = prims.addAttribute("affine_energy", computed_attribute=affine_energy(affine_matrices, bodies.stiffness))
  sc.addEnergy(snh, projection_method=projection_method)
  sc.addEnergy(kin, projection_method=-1)
  sc.addEnergy(ortho, projection_method=2)
  sc.addMinimizeTarget([hd["free_position"], affine_matrices, translations])
  hd.update(affine_matrices=affine_matrices, translations=translations, vertices_abd=verts)
  return sc, hd


# ---- cloth over a static obstacle with synthetic contacts ------------------------------

def lagged_friction_pt(x_old, dhat, kappa):
  """Lagged point-triangle friction data for pairs ``x_old`` [n, 4, 3] (point,
  triangle) at the start of the step, vectorised: the closest-point
  coordinates, the tangent basis and the contact force magnitude
  (``friction_helpers.py:12-27, 73-141``); returns [n, 9]
  (beta1, beta2, tangent0, tangent1, lambda_last_h)."""
  x = np.asarray(x_old, dtype=np.float64)
  p, t0, t1, t2 = x[:, 0], x[:, 1], x[:, 2], x[:, 3]
  e01, e02 = t1 - t0, t2 - t0
  B = np.stack([e01, e02], axis=2)                       # [n, 3, 2]
  btb = np.einsum("nki,nkj->nij", B, B)
  beta = np.einsum("nij,nj->ni", np.linalg.inv(btb), np.einsum("nki,nk->ni", B, p - t0))
  tan0 = e01 / np.linalg.norm(e01, axis=1, keepdims=True)
  c = np.cross(np.cross(e01, e02), e01)
  tan1 = c / np.linalg.norm(c, axis=1, keepdims=True)
  q = t0 + beta[:, :1] * e01 + beta[:, 1:] * e02
  d2 = np.einsum("ni,ni->n", p - q, p - q)
  lg = np.log(d2 / dhat)
  lenE = d2 - dhat
  inner = lg * lg * (2.0 * d2 - 2.0 * dhat) + 2.0 * lg * lenE * lenE / d2
  lam = -kappa * 2.0 * np.sqrt(d2) * inner
  return np.concatenate([beta, tan0, tan1, lam[:, None]], axis=1)


@dataclass
class ClothContact:
  """Arrays of the cloth-over-obstacle scene (union order: obstacle, cloth)."""

  side: int
  cloth_rest: np.ndarray      # (nc, 3)
  cloth_position: np.ndarray  # (nc, 3)
  obstacle: np.ndarray        # (no, 3) static, non-target
  tris: np.ndarray            # (nt, 3) cloth triangles (cloth-local ids)
  bend: np.ndarray            # (nb, 4) interior edges + opposite vertices (cloth-local)
  pt: np.ndarray              # (npt, 4) union ids: cloth point, obstacle triangle
  ee: np.ndarray              # (nee, 4) union ids: cloth edge, obstacle edge
  lagged: np.ndarray          # (npt, 9) friction data of the PT pairs
  mass: np.ndarray            # (nc,)
  mu: float
  lam: float
  thickness: float
  bend_stiff: float
  dhat: float
  kappa: float
  friction: float
  fdhat: float
  dt: float
  bodies: "AffineBodies" = None   # affine bodies over the cloth (icospheres), or None
  body_pt: np.ndarray = None      # (nbp, 4) PT pairs in the union [cloth, abd, obstacle]


def icosphere(subdivisions: int):
  """Unit icosphere: vertices (10 * 4^s + 2, 3) and triangles (20 * 4^s, 3),
  each face split into four with the edge midpoints pushed to the sphere."""
  t = (1.0 + 5.0 ** 0.5) / 2.0
  v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
  f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
                [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
  v /= np.linalg.norm(v, axis=1, keepdims=True)
  for _ in range(subdivisions):
    e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
    key = np.sort(e, axis=1)
    uniq, inv = np.unique(key, axis=0, return_inverse=True)
    mid = v[uniq[:, 0]] + v[uniq[:, 1]]
    mid /= np.linalg.norm(mid, axis=1, keepdims=True)
    m = len(v) + inv.reshape(3, -1)  # midpoint of edges (0,1), (1,2), (2,0) per face
    a, b, c = f[:, 0], f[:, 1], f[:, 2]
    f = np.concatenate([np.stack([a, m[0], m[2]], 1), np.stack([b, m[1], m[0]], 1), np.stack([c, m[2], m[1]], 1),
                        np.stack([m[0], m[1], m[2]], 1)])
    v = np.concatenate([v, mid])
  return v, f


def _bodies_over_cloth(rng, side, spacing, dhat, num_bodies, subdivisions, radius, stiffness, dt):
  """Icosphere affine bodies on a grid over the cloth, each lowered until its
  lowest vertex is just above sqrt(0.1 d-hat) (the cloth lies at y = 0)."""
  unit, faces = icosphere(subdivisions)
  xbar = unit * radius
  nv = len(xbar)
  g = int(np.ceil(np.sqrt(num_bodies)))
  extent = (side - 1) * spacing
  affine, trans = [], []
  for b in range(num_bodies):
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if np.linalg.det(q) < 0:
      q[:, 0] = -q[:, 0]
    sym = rng.uniform(-1e-3, 1e-3, size=(3, 3))
    a = q @ (np.eye(3) + 0.5 * (sym + sym.T))
    low = float((xbar @ a.T)[:, 1].min())
    cx, cz = ((b % g) + 0.5) * extent / g, ((b // g) + 0.5) * extent / g
    affine.append(a.ravel())
    trans.append([cx, 1.02 * np.sqrt(0.1 * dhat) - low, cz])
  return AffineBodies(
      rest=np.tile(xbar, (num_bodies, 1)), vertex_body=np.repeat(np.arange(num_bodies), nv),
      tets=np.zeros((0, 4), dtype=np.uint32), affine=np.asarray(affine), translation=np.asarray(trans),
      mass=np.full(num_bodies * nv, 2.0 / nv), velocity=np.zeros((num_bodies * nv, 3)), mu=0.0, lam=0.0,
      stiffness=stiffness, dt=dt, gravity=np.array([0.0, -9.8, 0.0])), faces


def _body_cloth_pairs(bodies, faces, cloth_pos, side, spacing, dhat):
  """PT pairs between the bodies and the flat cloth (y = 0), in the union
  [cloth, abd, obstacle]: (a) a body vertex over the cloth triangle below
  it, (b) a cloth vertex below a body triangle; kept when the squared
  plane distance lies in (0.1, 1) d-hat."""
  n, nc = side, len(cloth_pos)
  x = bodies.positions()
  lo, hi = 0.1 * dhat, dhat
  out = []
  # (a) body vertex -> cloth triangle (plane y = 0: squared distance y^2)
  y2 = x[:, 1] ** 2
  i = np.floor(x[:, 0] / spacing).astype(np.int64)
  k = np.floor(x[:, 2] / spacing).astype(np.int64)
  ok = (y2 > lo) & (y2 < hi) & (i >= 0) & (i < n - 1) & (k >= 0) & (k < n - 1)
  for v in np.flatnonzero(ok):
    a = i[v] * n + k[v]
    u, w = x[v, 0] / spacing - i[v], x[v, 2] / spacing - k[v]
    tri = (a, a + n + 1, a + n) if u > w else (a, a + 1, a + n + 1)
    out.append((nc + v, *tri))
  # (b) cloth vertex nearest below a body triangle's centroid
  nv = bodies.rest.shape[0] // bodies.num_bodies
  for b in range(bodies.num_bodies):
    f = faces + b * nv
    p = x[f]
    low = np.all(p[:, :, 1] < np.sqrt(hi) * 1.5, axis=1)
    for tri, q in zip(f[low], p[low]):
      c = q.mean(axis=0)
      ci, ck = int(round(c[0] / spacing)), int(round(c[2] / spacing))
      if not (0 <= ci < n and 0 <= ck < n):
        continue
      cv = ci * n + ck
      nrm = np.cross(q[1] - q[0], q[2] - q[0])
      d = float(np.dot(cloth_pos[cv] - q[0], nrm) ** 2 / np.dot(nrm, nrm))
      if lo < d < hi:
        out.append((cv, nc + tri[0], nc + tri[1], nc + tri[2]))
  return np.asarray(out, dtype=np.uint32).reshape(-1, 4)


def cloth_contact(side: int = 256, pairs: int = 200_000, spacing: float = 0.05, young: float = 1e4,
                  poisson: float = 0.3, thickness: float = 1e-3, bend_stiff: float = 1e-3, dhat: float = 1e-3,
                  kappa: float = 1e3, friction: float = 0.3, eps_v: float = 1e-3, density: float = 200.0,
                  dt: float = 0.01, seed: int = 0, num_bodies: int = 0, body_subdivisions: int = 4,
                  body_radius: float = 0.5, body_stiffness: float = 1e5) -> ClothContact:
  """A ``side x side`` cloth sheet (xz plane, triangles wound to +y normals)
  over a static obstacle grid offset by half a cell, with ``pairs`` synthetic
  contacts split between point-triangle and edge-edge pairs whose squared
  distances spread over (0.1, 1.0) d-hat (obstacle heights drawn per vertex).
  With ``num_bodies``, icosphere affine bodies (10 * 4^s + 2 vertices each)
  rest on the cloth, coupled to it by point-triangle pairs in the same
  distance window; they take their share of the point-triangle pairs."""
  rng = np.random.default_rng(seed)
  n = side
  gi, gk = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
  rest = np.stack([gi.ravel() * spacing, np.zeros(n * n), gk.ravel() * spacing], axis=1)
  pos = rest + rng.uniform(-0.01, 0.01, size=rest.shape) * spacing
  pos[:, 1] = 0.0
  a = (gi[:-1, :-1] * n + gk[:-1, :-1]).ravel()
  b, c, d = a + n, a + n + 1, a + 1
  tris = np.concatenate([np.stack([a, c, b], axis=1), np.stack([a, d, c], axis=1)])
  # interior edges with their two opposite vertices
  e = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]])
  opp = np.concatenate([tris[:, 2], tris[:, 0], tris[:, 1]])
  key = np.sort(e, axis=1)
  order = np.lexsort((key[:, 1], key[:, 0]))
  key, e, opp = key[order], e[order], opp[order]
  same = np.all(key[1:] == key[:-1], axis=1)
  i = np.flatnonzero(same)
  bend = np.stack([e[i, 0], e[i, 1], opp[i], opp[i + 1]], axis=1)
  # obstacle: (n-1) x (n-1) grid at the cell centres, below the cloth
  m = n - 1
  oi, ok = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
  obstacle = np.stack([(oi.ravel() + 0.5) * spacing, np.zeros(m * m), (ok.ravel() + 0.5) * spacing], axis=1)
  obstacle[:, 1] = -np.sqrt(rng.uniform(0.1, 1.0, size=m * m) * dhat)
  no = m * m
  oa = (oi[:-1, :-1] * m + ok[:-1, :-1]).ravel()
  otris = np.stack([oa, oa + m + 1, oa + m], axis=1)
  bodies, body_pt = None, None
  if num_bodies:
    bodies, faces = _bodies_over_cloth(rng, n, spacing, dhat, num_bodies, body_subdivisions, body_radius,
                                       body_stiffness, dt)
    body_pt = _body_cloth_pairs(bodies, faces, pos, n, spacing, dhat)
  npt = max(0, pairs // 2 - (0 if body_pt is None else len(body_pt)))
  nee = pairs - pairs // 2
  # PT: a cloth vertex above an obstacle triangle (cloth vertex (i+1, k+1) lies over cell (i, k))
  tri_pick = rng.integers(0, len(otris), size=npt)
  ti, tk = tri_pick // (m - 1), tri_pick % (m - 1)
  cloth_v = (ti + 1) * n + (tk + 1)
  pt = np.stack([no + cloth_v, otris[tri_pick, 0], otris[tri_pick, 1], otris[tri_pick, 2]], axis=1)
  # EE: a cloth x-edge crossing an obstacle z-edge below it
  ei = rng.integers(0, m - 1, size=nee)
  ek = rng.integers(1, m, size=nee)
  c0 = ei * n + ek
  c1 = (ei + 1) * n + ek
  o0 = ei * m + (ek - 1)
  o1 = ei * m + ek
  ee = np.stack([no + c0, no + c1, o0, o1], axis=1)
  allpos = np.concatenate([obstacle, pos])
  lagged = lagged_friction_pt(allpos[pt], dhat, kappa)
  areas = np.zeros(n * n)
  cr = np.cross(rest[tris[:, 1]] - rest[tris[:, 0]], rest[tris[:, 2]] - rest[tris[:, 0]])
  tri_area = 0.5 * np.linalg.norm(cr, axis=1)
  np.add.at(areas, tris.ravel(), np.repeat(tri_area / 3.0, 3))
  mu, lam = lame(young, poisson)
  return ClothContact(side=n, cloth_rest=rest, cloth_position=pos, obstacle=obstacle, tris=tris, bend=bend,
                      pt=pt.astype(np.uint32), ee=ee.astype(np.uint32), lagged=lagged,
                      mass=density * thickness * areas, mu=mu, lam=lam, thickness=thickness,
                      bend_stiff=bend_stiff, dhat=dhat, kappa=kappa, friction=friction, fdhat=eps_v * eps_v,
                      dt=dt, bodies=bodies, body_pt=body_pt)


def cloth_contact_scene(cc: ClothContact, projection_method: int = 1):
  """The cloth scene with the public API: StVK membrane and bending on the
  cloth, PT/EE barriers and PT friction through a union [obstacle, cloth]
  (the obstacle is DATA but not a minimisation target), inertia."""
  from .energies import (edge_edge, friction_point_triangle, inertia, point_triangle, bending as bend_energy,
                         stvk_membrane)
  from .scene import scene as make_scene
  sc = make_scene("cloth_contact")
  body = sc.addMesh("cloth")
  obst = body.addPrimitive("obstacle", numInstances=len(cc.obstacle))
  opos = obst.addAttribute("position", rows=3, cols=1)
  opos.updateValue(cc.obstacle)
  orest = obst.addConstant("old_position", rows=3, cols=1)
  orest.updateValue(cc.obstacle)
  cloth = body.addPrimitive("cloth", numInstances=len(cc.cloth_position))
  pos = cloth.addAttribute("position", rows=3, cols=1)
  pos.updateValue(cc.cloth_position)
  rest = cloth.addConstant("rest_position", rows=3, cols=1)
  rest.updateValue(cc.cloth_rest)
  old = cloth.addConstant("old_position", rows=3, cols=1)
  old.updateValue(cc.cloth_position)
  mass = cloth.addConstant("mass")
  mass.updateValue(cc.mass)
  tri = body.addPrimitive("triangles", numInstances=len(cc.tris))
  tc = tri.addConnectivity("to_cloth", cloth, cc.tris.astype(np.uint32), 3)
  mem = tri.addAttribute("stvk", computed_attribute=stvk_membrane(
      tri.addAttribute("rest", through=tc, source=rest), tri.addAttribute("x", through=tc, source=pos),
      cc.mu, cc.lam, cc.thickness, cc.dt))
  be = body.addPrimitive("bending_edges", numInstances=len(cc.bend))
  bc = be.addConnectivity("to_cloth", cloth, cc.bend.astype(np.uint32), 4)
  ben = be.addAttribute("bending", computed_attribute=bend_energy(
      be.addAttribute("x", through=bc, source=pos), be.addAttribute("rest", through=bc, source=rest),
      cc.bend_stiff, cc.dt))
  allv = body.addPrimitiveUnion("all_vertices", [obst, cloth])
  apos = allv.addAttribute("position")
  aold = allv.addAttribute("old_position")
  contact = []
  if len(cc.pt):
    ptp = body.addPrimitive("pt_pairs", numInstances=len(cc.pt))
    ptc = ptp.addConnectivity("to_vertices", allv, cc.pt, 4)
    ptx = ptp.addAttribute("x", through=ptc, source=apos)
    lag = ptp.addConstant("lagged", rows=9, cols=1)
    lag.updateValue(cc.lagged)
    contact += [ptp.addAttribute("barrier", computed_attribute=point_triangle(ptx, cc.dhat, cc.kappa)),
                ptp.addAttribute("friction", computed_attribute=friction_point_triangle(
                    ptx, ptp.addAttribute("x_old", through=ptc, source=aold), cc.fdhat, cc.dt, cc.friction, lag))]
  if len(cc.ee):
    eep = body.addPrimitive("ee_pairs", numInstances=len(cc.ee))
    eec = eep.addConnectivity("to_vertices", allv, cc.ee, 4)
    contact.append(eep.addAttribute("barrier", computed_attribute=edge_edge(
        eep.addAttribute("x", through=eec, source=apos), cc.dhat, cc.kappa)))
  kin = cloth.addAttribute("inertia", computed_attribute=inertia(old, None, cc.dt, pos, mass,
                                                                 gravity=(0.0, -9.8, 0.0)))
  for e in [mem, ben] + contact:
    sc.addEnergy(e, projection_method=projection_method)
  sc.addEnergy(kin, projection_method=-1)
  if cc.bodies is None:
    sc.addMinimizeTarget([pos])
    return sc, dict(position=pos, old_position=old)
  # affine bodies on the cloth: the collision union [cloth, abd, obstacle]
  # (dropping_in_container.py:344) carries the body-cloth point-triangle pairs
  prims, amat, trans, verts, vpos = _affine_body_attributes(body, cc.bodies)
  if len(cc.body_pt):
    coll = body.addPrimitiveUnion("collision_vertices", [cloth, verts, obst])
    cpos = coll.addAttribute("position")
    bpp = body.addPrimitive("body_pt_pairs", numInstances=len(cc.body_pt))
    bpc = bpp.addConnectivity("to_collision_vertices", coll, cc.body_pt, 4)
    sc.addEnergy(bpp.addAttribute("barrier", computed_attribute=point_triangle(
        bpp.addAttribute("x", through=bpc, source=cpos), cc.dhat, cc.kappa)), projection_method=projection_method)
  _affine_body_energies(sc, cc.bodies, prims, amat, verts, vpos, cc.dt)
  sc.addMinimizeTarget([pos, amat, trans])
  return sc, dict(position=pos, old_position=old, affine_matrices=amat, translations=trans)


# ---- contact between cloth, affine bodies and a container ------------------------------

def _affine_body_attributes(m, bodies: AffineBodies):
  """Bodies (``affine_matrices``, ``translations``) and their vertices at
  ``A xbar + t`` on mesh ``m``, as ``dropping_in_container.py:241-270``."""
  from .energies import affine_position
  prims = m.addPrimitive("affine_bodies", numInstances=bodies.num_bodies)
  amat = prims.addAttribute("affine_matrices", rows=3, cols=3)
  amat.updateValue(bodies.affine)
  trans = prims.addAttribute("translations", rows=3, cols=1)
  trans.updateValue(bodies.translation)
  verts = m.addPrimitive("vertices_abd", numInstances=len(bodies.rest))
  rest = verts.addConstant("rest_position", rows=3, cols=1)
  rest.updateValue(bodies.rest)
  v2b = verts.addConnectivity("v_abd2_abd", prims, bodies.vertex_body[:, None].astype(np.uint32), 1)
  va = verts.addAttribute("affine_matrix", through=v2b, source=amat).resize(3, 3)
  vt = verts.addAttribute("translation", through=v2b, source=trans).resize(3, 1)
  vpos = verts.addAttribute("position", computed_attribute=affine_position(va, rest, vt))
  return prims, amat, trans, verts, vpos


def _affine_body_energies(sc, bodies: AffineBodies, prims, amat, verts, vpos, dt):
  """Inertia of the body vertices (no projection) and the bodies'
  orthogonality energy (projection 2), as ``dropping_in_container.py:377-395``."""
  from .energies import affine_energy, inertia
  last = verts.addConstant("last_position", rows=3, cols=1)
  last.updateValue(bodies.positions())
  vel = verts.addConstant("velocity", rows=3, cols=1)
  vel.updateValue(bodies.velocity)
  vm = verts.addConstant("mass")
  vm.updateValue(bodies.mass)
  sc.addEnergy(verts.addAttribute("inertia_abds", computed_attribute=inertia(last, vel, dt, vpos, vm,
                                                                              gravity=tuple(bodies.gravity))),
               projection_method=-1)
  sc.addEnergy(prims.addAttribute("affine_energy", computed_attribute=affine_energy(amat, bodies.stiffness)),
               projection_method=2)


BARRIER_PAIRS = (("pp", 2), ("pe", 3), ("pt", 4), ("ee", 4))


def contact_with_bodies_scene(cloth_position, bodies: AffineBodies, container, pairs, dhat: float, kappa: float,
                              projection_method: int = 2, cloth_mass=None, dt: float = 0.01,
                              name: str = "contact_with_bodies", friction=None,
                              separate_hessian_jacobian: bool = False):
  """Barrier pairs over the collision union ``[cloth, abd vertices, container]``
  (``examples/dropping_in_container_mixed/dropping_in_container.py:344-405``):
  the abd vertices sit at ``A xbar + t`` of their bodies, the container is
  DATA, the targets are ``[cloth position, affine_matrices, translations]``.
  ``pairs`` maps ``pp/pe/pt/ee`` to union-index connectivities.  With
  ``cloth_mass`` the scene also carries the inertia of the cloth and body
  vertices and the bodies' orthogonality energy (a solvable system).
  ``friction`` (optional) adds lagged friction over the same union
  (``examples/dropping_in_container/dropping_in_container.py:248-290``): a dict
  with ``last`` (the union's positions at the start of the step, one row a
  union vertex), ``fdhat``, ``rate``, and per kind ``pp/pe/pt/ee`` a pair of
  (union connectivity, lagged [n, 9])."""
  from .energies import (edge_edge, friction_edge_edge, friction_point_edge, friction_point_point,
                         friction_point_triangle, inertia, point_edge, point_point, point_triangle)
  from .scene import scene as make_scene
  sc = make_scene(name)
  m = sc.addMesh("collision_mesh")
  cloth = m.addPrimitive("cloth", numInstances=len(cloth_position))
  cpos = cloth.addAttribute("position", rows=3, cols=1)
  cpos.updateValue(cloth_position)
  prims, amat, trans, verts, vpos = _affine_body_attributes(m, bodies)
  cont = m.addPrimitive("container", numInstances=len(container))
  opos = cont.addAttribute("position", rows=3, cols=1)
  opos.updateValue(container)
  allv = m.addPrimitiveUnion("vertices", [cloth, verts, cont])
  apos = allv.addAttribute("position")
  makers = {"pp": point_point, "pe": point_edge, "pt": point_triangle, "ee": edge_edge}
  for key, arity in BARRIER_PAIRS:
    conn = pairs.get(key)
    if conn is None or len(conn) == 0:
      continue
    p = m.addPrimitive(key, numInstances=len(conn))
    c = p.addConnectivity(key + "2v", allv, np.asarray(conn, dtype=np.uint32), arity)
    x = p.addAttribute("positions", through=c, source=apos)
    sc.addEnergy(p.addAttribute("barrier", computed_attribute=makers[key](x, dhat, kappa)),
                 projection_method=projection_method, separate_hessian_jacobian=separate_hessian_jacobian)
  if friction is not None:
    last = np.asarray(friction["last"], dtype=np.float64).reshape(-1, 3)
    nc, nv = len(cloth_position), len(bodies.rest)
    for prim, part in ((cloth, last[:nc]), (verts, last[nc:nc + nv]), (cont, last[nc + nv:])):
      a = prim.addConstant("contact_last_position", rows=3, cols=1)
      a.updateValue(part)
    alast = allv.addAttribute("contact_last_position")
    fmakers = {"pp": friction_point_point, "pe": friction_point_edge, "pt": friction_point_triangle,
               "ee": friction_edge_edge}
    for key, arity in BARRIER_PAIRS:
      if key not in friction:
        continue
      conn, lagged = friction[key]
      p = m.addPrimitive("friction_" + key, numInstances=len(conn))
      c = p.addConnectivity(key + "f2v", allv, np.asarray(conn, dtype=np.uint32), arity)
      x = p.addAttribute("positions", through=c, source=apos)
      xl = p.addAttribute("last_positions", through=c, source=alast)
      lag = p.addConstant("lagged", rows=9, cols=1)
      lag.updateValue(np.asarray(lagged, dtype=np.float64))
      sc.addEnergy(p.addAttribute("friction", computed_attribute=fmakers[key](x, xl, friction["fdhat"], dt,
                                                                              friction["rate"], lag)),
                   projection_method=projection_method, separate_hessian_jacobian=separate_hessian_jacobian)
  if cloth_mass is not None:
    old = cloth.addConstant("old_position", rows=3, cols=1)
    old.updateValue(cloth_position)
    cm = cloth.addConstant("mass")
    cm.updateValue(cloth_mass)
    sc.addEnergy(cloth.addAttribute("inertia", computed_attribute=inertia(old, None, dt, cpos, cm,
                                                                         gravity=tuple(bodies.gravity))),
                 projection_method=-1)
    _affine_body_energies(sc, bodies, prims, amat, verts, vpos, dt)
  sc.addMinimizeTarget([cpos, amat, trans])
  return sc, dict(position=cpos, affine_matrices=amat, translations=trans, vertices=allv)
