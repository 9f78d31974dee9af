"""Host-side logic (no GPU): workloads, the MAS hierarchy builder, the API graph."""

import numpy as np
import pytest

from oracle import mas as omas
from oracle import pattern
from yasps_b200 import mas_hierarchy, scenes


def _cube_edges(n):
  c = scenes.fem_cube(n)
  codes, sizes = c.snh_slots()
  perm, _, _ = pattern.compress_slots(codes, sizes)
  coords, dims, _ = pattern.coordinates(codes, sizes, perm)
  pat = pattern.build_pattern([coords], [dims])
  pos = pat.positions
  return c, pos, (pos[pos[:, 0] != pos[:, 1]] // 3)


def test_fem_cube_counts():
  c = scenes.fem_cube(10)
  assert (c.pinned_count, c.free_count, c.tet_count) == (100, 900, 4374)
  r = c.rest_all()[c.tets.astype(np.int64)]
  det = np.linalg.det(np.stack([r[:, 1] - r[:, 0], r[:, 2] - r[:, 0], r[:, 3] - r[:, 0]], axis=2))
  assert np.all(det > 0)
  assert np.isclose(c.mass.sum() + 0.0, c.mass.sum())
  # Lame parameters from E, nu
  mu, lam = scenes.lame(1e5, 0.4)
  assert np.isclose(mu, 35714.285714285714) and np.isclose(lam, 142857.14285714287)


def test_cube_edge_count_matches_grid_formula():
  # all vertices free: axis + face-diagonal + body-diagonal edges + diagonal blocks
  n = 6
  c = scenes.fem_cube(n)
  t = c.tets.astype(np.int64)
  e = set()
  for a in range(4):
    for b in range(a + 1, 4):
      e |= {(min(x, y), max(x, y)) for x, y in zip(t[:, a], t[:, b])}
  axis = 3 * (n - 1) * n * n
  face = 3 * (n - 1) ** 2 * n
  body = (n - 1) ** 3
  assert len(e) == axis + face + body


@pytest.mark.parametrize("n", [4, 6, 9])
def test_product_hierarchy_matches_oracle(n):
  c, pos, edges = _cube_edges(n)
  nv = c.free_count
  hp = mas_hierarchy.build_hierarchy(np.full(nv, 3), edges)
  ho = omas.build_hierarchy(np.full(nv, 3), [tuple(e) for e in edges])
  assert hp.domains_per_level == [len(l.domains) for l in ho.levels]
  assert hp.nodes_per_level == [l.dims.size for l in ho.levels]
  for lp, lo in zip(hp.levels, ho.levels):
    assert [sorted(np.asarray(d).tolist()) for d in lp.domains] == [sorted(d) for d in lo.domains]
  for cp, co in zip(hp.composed, ho.composed):
    assert np.array_equal(cp, co)


def test_hierarchy_tables_are_consistent():
  c, pos, edges = _cube_edges(6)
  nv = c.free_count
  h = mas_hierarchy.build_hierarchy(np.full(nv, 3), edges)
  t = mas_hierarchy.build_tables(h, pos)
  L = len(h.levels)
  assert t.cmap.size == L * nv
  assert t.dom_node_ptr[-1] == t.level_node_offset[-1]
  # every packed node belongs to exactly one domain
  assert np.array_equal(np.sort(t.dom_nodes), np.arange(t.level_node_offset[-1]))
  # coarse block sources reference earlier blocks only
  idx = t.cb_src & 0x3FFFFFFF
  assert idx.size == 0 or idx.max() < t.fine_blocks + t.cb_level_begin[-1]
  assert t.max_domain_dofs <= 96
  # the children of the level-1 nodes are every fine variable exactly once
  # (the PCG update writes the level-1 residuals from this partition)
  ptr = np.asarray(t.child_ptr, dtype=np.int64)
  lo, hi = int(t.level_node_offset[1]) - nv, int(t.level_node_offset[2]) - nv
  kids = np.asarray(t.child_fine, dtype=np.int64)[ptr[lo]:ptr[hi]]
  assert np.array_equal(np.sort(kids), np.arange(nv))


def test_scene_api_validation():
  from yasps_b200 import scene, stable_neo_hookean
  sc = scene("s")
  m = sc.addMesh("m")
  v = m.addPrimitive("v", numInstances=4)
  x = v.addAttribute("x", rows=3, cols=1)
  t = m.addPrimitive("t", numInstances=1)
  con = t.addConnectivity("c", v, [[0, 1, 2, 3]], 4)
  tx = t.addAttribute("x", through=con, source=x)
  with pytest.raises(ValueError):
    stable_neo_hookean(x, tx, 1.0, 1.0, 0.01)  # rest must be a JOIN
  with pytest.raises(ValueError):
    t.addConnectivity("bad", v, [[0, 1, 2, 9]], 4)
  with pytest.raises(ValueError):
    sc.addMinimizeTarget([x, x])


def test_fem_positions_match_fem_cube():
  from yasps_b200 import scenes
  c = scenes.fem_cube(6, young=3e4, poisson=0.33, noise=0.02, seed=11)
  pinned, free = scenes.fem_positions(6, noise=0.02, seed=11)
  assert np.array_equal(pinned, c.pinned_position) and np.array_equal(free, c.free_position)


def test_poisson_stream_shapes_and_ranges():
  from yasps_b200 import serving
  reqs = serving.poisson_fem_stream(count=40, mean_spacing=2e-3, side_range=(4, 9), seed=3)
  arr = np.array([r.arrival for r in reqs])
  assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
  assert all(4 <= r.side <= 9 for r in reqs)
  for r in reqs:
    assert r.free_position.numel() == 3 * r.side ** 2 * (r.side - 1)
    assert r.pinned_position.numel() == 3 * r.side ** 2
  mu = np.array([r.mu for r in reqs])
  assert np.all(mu > 0)


def test_serve_entry_points_validate_without_gpu():
  import ctypes
  from yasps_b200 import _lib as L
  lib = L.load()
  h = ctypes.c_void_p()
  assert lib.ys_serve_create(0, 4, ctypes.byref(h)) == L.YS_ERR_INVALID
  assert lib.ys_serve_create(8, 0, ctypes.byref(h)) == L.YS_ERR_INVALID
  assert lib.ys_serve_attach(None, 0, None) == L.YS_ERR_INVALID
  assert lib.ys_serve_workspace_doubles(1000) >= 15 * 1000


def test_mas_tile_layout_host_math():
  """The tiled FP32 inverse layout: the Python size formula equals the
  library's, the folded tile order is a bijection onto [0, T(T+1)/2) that the
  GEMV inverts with its float quotient, and its partial grid rows are read
  without shared-memory bank conflicts."""
  from yasps_b200 import _lib
  from yasps_b200.mas_hierarchy import inverse_floats
  lib = _lib.load()
  for n in range(3, 129, 3):
    t = (n + 3) // 4
    t += t & 1
    assert inverse_floats(n) == lib.ys_mas_inverse_floats(n) == 16 * t * (t + 1) // 2
    assert 4 * t <= (96 if n <= 96 else 128)  # inside the inverse kernel's register tile

    def slot(a, b):
      if a < t // 2:
        return a * (t + 1) + (b - a)
      q = t - 1 - a
      return q * (t + 1) + (t - q) + (b - a)

    slots = sorted(slot(a, b) for a in range(t) for b in range(a, t))
    assert slots == list(range(t * (t + 1) // 2))
    inv_w = np.float32(1.0) / np.float32(t + 1)
    for a in range(t):
      for b in range(a, t):
        s = slot(a, b)
        q = int((np.float32(s) + np.float32(0.5)) * inv_w)
        c = s - q * (t + 1)
        first = c < t - q
        assert (q if first else t - 1 - q) == a
        assert ((q + c) if first else a + (c - (t - q))) == b
    ld = (t + 6) // 8 * 8 + 1
    assert ld >= t and ld % 8 == 1
    banks = {((i // 4) * ld * 4 + i % 4) % 32 for i in range(32)}
    assert len(banks) == 32


def _tiled_sweep(s, tiles=6):
  """Model of the domain-inverse kernel's symmetric 2-pivot sweep on a
  16-row tile grid: only upper tiles are updated, lower tiles hold NaN, the
  pivot column is read from column K for rows up to the pivot's tile and
  from row K beyond it (the kernel's publish / read rule)."""
  n = s.shape[0]
  size = 16 * tiles
  x = np.zeros((size, size))
  x[:n, :n] = s
  x[np.arange(n, size), np.arange(n, size)] = 1.0
  tile = np.arange(size) // 16
  upper = tile[:, None] <= tile[None, :]
  x[~upper] = np.nan
  for k in range(0, n, 2):
    kb = k // 16
    kk = [k, k + 1]
    colb, rowb = x[:, kk].copy(), x[kk, :].copy()
    for m in range(2):
      colb[kk[m], m] -= 1.0
      rowb[m, kk[m]] -= 1.0
    pinv = np.linalg.inv(colb[kk, :] + np.eye(2))
    vi = np.where((tile <= kb)[:, None], colb, rowb.T)
    vj = np.where((tile >= kb)[:, None], rowb.T, colb)
    x = np.where(upper, x - (vi @ pinv) @ vj.T, x)
    x[k, k] -= 2.0
    x[k + 1, k + 1] -= 2.0
  return x


def test_symmetric_sweep_model_reads_upper_tiles_only():
  """The upper-tile sweep gives -S^-1 on every upper tile and never reads a
  lower one (NaN there would spread)."""
  rng = np.random.default_rng(3)
  for n in (2, 18, 48, 96):
    b = rng.normal(size=(n, n))
    a = b @ b.T + n * np.eye(n)
    d = 1.0 / np.sqrt(np.diag(a))
    s = a * d[:, None] * d[None, :]
    x = _tiled_sweep(s)
    tile = np.arange(n) // 16
    up = tile[:, None] <= tile[None, :]
    got = -x[:n, :n]
    assert not np.isnan(got[up]).any()
    inv = np.linalg.inv(s)
    assert np.abs(np.where(up, got - inv, 0.0)).max() <= 1e-12 * np.abs(inv).max()
