"""GPU parity of the Newton inner loop against the oracle (CUDA path via the C ABI).

Tolerances (relative to the largest magnitude of the compared quantity):
pattern, lookups and assembly plan bit-exact; FP64 gradient / Hessian 1e-12;
FP32 SpMV 1e-5; solutions at the stated relative residual.
"""

import numpy as np
import pytest

from oracle import solvers
from tests.oracle_scene import OracleCube
from yasps_b200 import scenes

pytestmark = pytest.mark.gpu


def rel(a, b):
  a, b = np.asarray(a), np.asarray(b)
  return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def c0():
  cube = scenes.fem_cube(10, spacing=0.1, young=1e5, poisson=0.4, noise=0.01, seed=0)
  return cube, OracleCube(cube)


def build(cube, solver=None, **opts):
  sc, h = scenes.fem_scene(cube)
  if solver:
    sc.minimizer.setSolver(solver, **opts)
  return sc, h


def test_pattern_and_lookups_bit_exact(c0):
  cube, ora = c0
  sc, _ = build(cube)
  H = sc.minimizer.computeNumericValue()
  pos = H.block_positions.cpu().numpy().astype(np.int64).reshape(-1, 2)
  assert np.array_equal(pos, ora.pattern.positions)
  assert H.block_counts == ora.pattern.category_counts.tolist()
  assert H.block_dimensions == [3, 3]
  assert H.blocks_start_indices == ora.pattern.category_starts.tolist()
  lk = H._static.pattern.lookup.cpu().numpy().astype(np.int64)
  assert np.array_equal(lk, np.concatenate(ora.pattern.lookups))


def test_gradient_and_hessian_fp64(c0):
  cube, ora = c0
  sc, _ = build(cube)
  H = sc.minimizer.computeNumericValue()
  assert rel(H.gradient.value.cpu().numpy(), ora.gradient) <= 1e-12
  assert rel(H.blocks_flattened.cpu().numpy()[:ora.values.size], ora.values) <= 1e-12
  assert rel(H.diagonal_blocks.cpu().numpy(), ora.diag_blocks) <= 1e-12


def test_projection_path_with_many_indefinite_elements():
  cube = scenes.fem_cube(6, noise=0.04, seed=5)
  ora = OracleCube(cube)
  assert (~ora.psd).sum() > 10, "the case must exercise the eigen-projection"
  sc, _ = build(cube)
  H = sc.minimizer.computeNumericValue()
  assert rel(H.blocks_flattened.cpu().numpy()[:ora.values.size], ora.values) <= 1e-12


@pytest.mark.parametrize("method", [0, 2])
def test_projection_methods(method):
  cube = scenes.fem_cube(5, noise=0.04, seed=7)
  ora = OracleCube(cube, projection_method=method)
  sc, _ = scenes.fem_scene(cube, projection_method=method)
  H = sc.minimizer.computeNumericValue()
  assert rel(H.blocks_flattened.cpu().numpy()[:ora.values.size], ora.values) <= 1e-12


def test_assembly_is_bit_reproducible(c0):
  cube, _ = c0
  sc, _ = build(cube)
  H = sc.minimizer.computeNumericValue()
  v1 = H.blocks_flattened.clone()
  g1 = H.gradient.value.clone()
  H.compute()
  assert bool((v1 == H.blocks_flattened).all()) and bool((g1 == H.gradient.value).all())


def test_spmv_fp64_and_fp32(c0):
  import torch
  from yasps_b200 import vector
  cube, ora = c0
  sc, _ = build(cube)
  H = sc.minimizer.computeNumericValue()
  x = np.linspace(-0.8, 0.9, H.cols)
  xv = vector(H.cols)
  xv.updateValue(x)
  ref = ora.matvec(x)
  for transpose in (False, True):
    assert rel(H.spmv(xv, transpose=transpose).get(), ref) <= 1e-12
  H.ensure_fp32()
  y32 = H.spmv(xv, fp32=True).get()
  assert rel(y32, ref) <= 1e-5
  # the float4 copy of x gives the same products in the same order: bit-exact
  from yasps_b200 import _lib as L
  nv = H.rows // 3
  xd = torch.from_numpy(x).cuda()
  x32 = torch.empty(4 * nv, dtype=torch.float32, device="cuda")
  y = torch.empty(H.rows, dtype=torch.float64, device="cuda")
  L.call("ys_pack_x32", L.ptr(xd), nv, L.ptr(x32), L.stream_ptr())
  assert torch.equal(x32.view(nv, 4)[:, :3], xd.view(nv, 3).float())
  for k, bs in enumerate(H.block_sets):
    row_ptr, eb, ec = H.spmv_plan(bs)
    L.call("ys_spmv3_x32", L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), nv, L.ptr(x32), L.ptr(y),
           1 if k else 0, L.stream_ptr())
  assert np.array_equal(y.cpu().numpy(), y32)
  # the tiled SpMV (shared-memory stages by bulk copies) gives the same bits
  check_tiled_spmv(H, x32, y.cpu().numpy())
  check_streamed_spmv(H, x32, y.cpu().numpy())


def check_tiled_spmv(H, x32, expected):
  import torch
  from yasps_b200 import _lib as L
  nv = H.rows // 3
  (bs,) = H.block_sets
  row_ptr, eb, ec = H.spmv_plan(bs)
  row_block, cap, ecap = H.tile_plan(bs)
  assert cap > 0 and ecap > 0 and ecap % 4 == 0
  rb = row_block.cpu().numpy().astype(np.int64)[:nv + 1]
  pos = bs.pattern.positions[:2 * bs.pattern.num_unique].cpu().numpy().astype(np.int64).reshape(-1, 2)
  assert np.array_equal(rb, np.searchsorted(pos[:, 0], 3 * np.arange(nv + 1), side="left"))
  tiles = np.arange(0, nv, L.YS_SPMV_TILE_ROWS)
  ends = np.minimum(tiles + L.YS_SPMV_TILE_ROWS, nv)
  assert cap == int((rb[ends] - rb[tiles]).max())
  rp = row_ptr.cpu().numpy().astype(np.int64)[:nv + 1]
  assert ecap == int((((rp[ends] + 3) & ~3) - (rp[tiles] & ~3)).max())
  status = torch.zeros(1, dtype=torch.int32, device="cuda")
  y = torch.full((H.rows,), np.nan, dtype=torch.float64, device="cuda")
  for stages in (0, 2, 3, 4, 0):  # 0: as many stages as let two CTAs share an SM
    L.call("ys_spmv3_x32_tiled", L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), L.ptr(row_block), cap,
           ecap, stages, nv, L.ptr(x32), L.ptr(y), 0, L.ptr(status), L.stream_ptr())
    assert np.array_equal(y.cpu().numpy(), expected)
  assert int(status.item()) == 0


def check_streamed_spmv(H, x32, expected):
  """The streamed-tile plan against the row plan (every entry word decodes
  to its entry's neighbour, block and orientation; the distinct columns of
  each tile are its entries' columns, ascending) and the streamed SpMV
  against ``expected`` bit for bit, with the grid capped so that CTAs loop
  over several tiles."""
  import torch
  from yasps_b200 import _lib as L
  nv = H.rows // 3
  (bs,) = H.block_sets
  row_ptr, eb, ec = H.spmv_plan(bs)
  sp = H.stream_plan(bs)
  assert sp is not None
  rp = row_ptr.cpu().numpy().astype(np.int64)[:nv + 1]
  ebn = eb.cpu().numpy().view(np.uint32).astype(np.int64)
  ecn = ec.cpu().numpy().astype(np.int64)
  desc = sp.desc.cpu().numpy().view(np.uint32).astype(np.int64).reshape(-1, 4)
  rows = sp.rows.cpu().numpy().view(np.uint32).astype(np.int64).reshape(-1, 68)
  words = sp.words.cpu().numpy().view(np.uint32).astype(np.int64)
  halo = sp.halo.cpu().numpy().view(np.uint32).astype(np.int64)
  src = sp.src.cpu().numpy().view(np.uint32).astype(np.int64)
  R = L.YS_SPMV_TILE_ROWS
  ntiles = (nv + R - 1) // R
  for t in range(ntiles):
    r0, r1 = t * R, min(t * R + R, nv)
    base, nslots, ne, nh = desc[t]
    assert base % 4 == 0 and base == (rp[r0] + 4 * t + 3) & ~3 and ne == rp[r1] - rp[r0]
    assert np.array_equal(rows[t, :r1 - r0 + 1], rp[r0:r1 + 1] - rp[r0]) and rows[t, 65] == nh
    cols = ecn[rp[r0]:rp[r1]]
    assert np.array_equal(halo[base:base + nh], np.unique(cols))
    w = words[base:base + ne]
    assert np.array_equal(halo[base + (w & 0xffff)], cols)
    slot = (w >> 16) & 0x7fff
    assert slot.max() < nslots
    assert np.array_equal(src[base + slot], ebn[rp[r0]:rp[r1]] & 0x7fffffff)
    assert np.array_equal(w >> 31, ebn[rp[r0]:rp[r1]] >> 31)
  assert sp.block_cap == max(((int(d[1]) + 3) & ~3) for d in desc[:ntiles])
  status = torch.zeros(1, dtype=torch.int32, device="cuda")
  y = torch.full((H.rows,), np.nan, dtype=torch.float64, device="cuda")
  st = sp.struct()
  for stages, max_ctas in ((0, 0), (2, 1), (3, 1), (2, 3), (3, 3), (0, 0)):
    L.call("ys_spmv3_x32_streamed", st, L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), nv, L.ptr(x32),
           L.ptr(y), 0, stages, max_ctas, L.ptr(status), L.stream_ptr())
    assert np.array_equal(y.cpu().numpy(), expected)
  # beta = 1 adds to y
  L.call("ys_spmv3_x32_streamed", st, L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), nv, L.ptr(x32),
         L.ptr(y), 1, 0, 0, L.ptr(status), L.stream_ptr())
  assert np.array_equal(y.cpu().numpy(), expected + expected)
  assert int(status.item()) == 0


def test_streamed_pcg_matches_tiled_pcg_bit_for_bit():
  """The FP32 MAS-PCG loop over the streamed-tile SpMV and over the tiled
  SpMV (same products; one tile a CTA in both grids here, so the curvature
  sums group alike): the same iterations and the same solution bits; the
  packed blocks follow new FP32 values."""
  import torch
  from yasps_b200 import _lib as L
  cube = scenes.fem_cube(16, spacing=0.1, young=1e6, poisson=0.45, noise=0.005, seed=3)
  sc, _ = build(cube, "mas", mixed_spmv=True, stop_rule="residual")
  solver = sc.minimizer.linearSolver
  mas = solver.implementation
  H = sc.minimizer.computeNumericValue()
  H.ensure_fp32()
  (bs,) = H.block_sets
  solver.computeSolution(H, H.gradient, None, tolerance=1e-6, maxIterations=2000, zero_initial_guess=True)
  runs = []
  for use_stream in (True, False, True):
    if use_stream:
      bs.stream = None  # rebuilt
    else:
      bs.stream = False  # no streamed plan: the tiled SpMV
    z = torch.zeros(H.rows, dtype=torch.float64, device="cuda")
    res = mas._run_pcg(H, H.gradient.value, z, True, L.YS_PREC_MAS, None, mas._mas, 1e-30, 30, True, "residual")
    runs.append((int(res.iterations), z.cpu().numpy().copy()))
  assert runs[0][0] == runs[1][0] == 30
  assert np.array_equal(runs[0][1], runs[1][1]) and np.array_equal(runs[0][1], runs[2][1])
  # a new assembly writes the packed blocks itself: the same as a fill
  assert sc.minimizer.computeNumericValue() is H
  sp = H.stream_plan(bs)
  assert sp.filled == (H.values32_version, bs.values32.data_ptr())
  want = torch.zeros_like(sp.blocks32)
  L.call("ys_spmv_stream_fill", L.ptr(bs.values32), L.ptr(sp.src), sp.slots, L.ptr(want), L.stream_ptr())
  used = (sp.src != -1).repeat_interleave(9)
  assert torch.equal(sp.blocks32[used], want[used])
  # new FP32 values (a new version) refresh the packed blocks before use
  before = sp.blocks32.clone()
  bs.values32.mul_(2.0)
  H.values32_version += 1
  assert H.stream_plan(bs) is sp
  assert torch.equal(sp.blocks32, before * 2.0)


def test_tiled_spmv_many_tiles_bit_identical():
  """A 24^3 cube (13,248 free variables, 207 tiles of 64 rows) through the
  tiled SpMV against the row-plan SpMV, bit for bit, and the FP32 loop that
  uses it against the oracle."""
  import torch
  from yasps_b200 import _lib as L
  cube = scenes.fem_cube(24, spacing=0.1, young=1e6, poisson=0.45, noise=0.005, seed=1)
  sc, _ = build(cube, "mas", mixed_spmv=True, stop_rule="residual")
  H = sc.minimizer.computeNumericValue()
  H.ensure_fp32()
  nv = H.rows // 3
  (bs,) = H.block_sets
  row_ptr, eb, ec = H.spmv_plan(bs)
  x = torch.sin(torch.arange(H.rows, dtype=torch.float64, device="cuda") * 0.37)
  x32 = torch.empty(4 * nv, dtype=torch.float32, device="cuda")
  L.call("ys_pack_x32", L.ptr(x), nv, L.ptr(x32), L.stream_ptr())
  y = torch.empty(H.rows, dtype=torch.float64, device="cuda")
  L.call("ys_spmv3_x32", L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), nv, L.ptr(x32), L.ptr(y), 0,
         L.stream_ptr())
  check_tiled_spmv(H, x32, y.cpu().numpy())
  check_streamed_spmv(H, x32, y.cpu().numpy())
  ora = OracleCube(cube)
  segs = sc.minimizeEnergy(tolerance=1e-6, maxIterations=2000)
  assert solvers.relative_residual(ora.matvec, ora.gradient, segs[0].cpu().numpy()) <= 1e-6


def test_block_jacobi_pcg_matches_oracle(c0):
  cube, ora = c0
  sc, _ = build(cube, "jacobian")
  H = sc.minimizer.computeNumericValue()
  n = H.rows
  inv = solvers.diagonal_inverse(ora.diag_blocks, [n // 3], [3])
  ref = solvers.jacobi_pcg(ora.matvec, ora.gradient, inv, [n // 3], [3], 1e-16, 2000)
  code = sc.minimizer.linearSolver.computeSolution(H, H.gradient, None, tolerance=1e-16, maxIterations=2000,
                                                   zero_initial_guess=True)
  assert ref.status > 0 and abs(code - ref.status) <= 1
  x = sc.minimizer.linearSolver.solution.cpu().numpy()
  assert solvers.relative_residual(ora.matvec, ora.gradient, x) <= 1e-7
  assert rel(x, ref.solution) <= 1e-6


def test_jacobi_status_codes(c0):
  cube, _ = c0
  sc, _ = build(cube, "jacobian")
  H = sc.minimizer.computeNumericValue()
  code = sc.minimizer.linearSolver.computeSolution(H, H.gradient, None, tolerance=1e-30, maxIterations=3,
                                                   zero_initial_guess=True)
  assert code == -4
  code = sc.minimizer.linearSolver.computeSolution(H, H.gradient, None, tolerance=1.0, maxIterations=3,
                                                   zero_initial_guess=True)
  assert code == 0


def test_mas_pcg_matches_oracle(c0):
  from oracle import mas as omas
  cube, ora = c0
  sc, _ = build(cube, "mas", fine_level_weight=1.0)  # the CPU reference's level weights
  H = sc.minimizer.computeNumericValue()
  p = ora.pattern
  edges = [(r // 3, c // 3) for r, c in p.positions if r != c]
  h = omas.build_hierarchy(np.full(ora.n // 3, 3), edges)
  blocks = [(r // 3, c // 3, ora.values[o:o + 9].reshape(3, 3)) for (r, c), o in zip(p.positions, p.value_offsets)]
  pre = omas.MASPreconditioner(h, omas.level_local_matrices(h, blocks))
  ref = solvers.mas_pcg(ora.matvec, ora.gradient, pre.apply, 1e-12, 500)
  code = sc.minimizer.linearSolver.computeSolution(H, H.gradient, None, tolerance=1e-12, maxIterations=500,
                                                   zero_initial_guess=True)
  st = sc.minimizer.linearSolver.statistics
  assert code == 0 and ref.converged
  assert abs(st["iterations"] - ref.iterations) <= 2
  x = sc.minimizer.linearSolver.solution.cpu().numpy()
  assert solvers.relative_residual(ora.matvec, ora.gradient, x) <= 10 * ref.relative_residual + 1e-9


@pytest.mark.parametrize("mixed", [False, True])
def test_mas_true_residual_target(c0, mixed):
  cube, ora = c0
  sc, _ = build(cube, "mas", mixed_spmv=mixed, stop_rule="residual")
  segs = sc.minimizeEnergy(tolerance=1e-6, maxIterations=1000)
  x = segs[0].cpu().numpy()
  assert solvers.relative_residual(ora.matvec, ora.gradient, x) <= 1e-6


def test_mas_apply_matches_oracle(c0):
  import torch
  from oracle import mas as omas
  from yasps_b200 import _lib as L
  cube, ora = c0
  sc, _ = build(cube, "mas", fine_level_weight=1.0)  # the CPU reference's level weights
  H = sc.minimizer.computeNumericValue()
  ms = sc.minimizer.linearSolver.implementation
  ms._ensure_hierarchy(H)
  assert ms.numeric_update(H) == 0
  r = np.cos(np.arange(H.rows) * 0.37)
  rt = torch.from_numpy(r).cuda()
  z = torch.zeros_like(rt)
  L.call("ys_mas_apply", ms._mas, L.ptr(rt), L.ptr(z), L.stream_ptr())
  p = ora.pattern
  edges = [(a // 3, b // 3) for a, b in p.positions if a != b]
  h = omas.build_hierarchy(np.full(ora.n // 3, 3), edges)
  blocks = [(a // 3, b // 3, ora.values[o:o + 9].reshape(3, 3)) for (a, b), o in zip(p.positions, p.value_offsets)]
  pre = omas.MASPreconditioner(h, omas.level_local_matrices(h, blocks))
  # FP32 inverses and level vectors: single-precision agreement
  assert rel(z.cpu().numpy(), pre.apply(r)) <= 2e-4


def test_mas_singular_domain_is_reported(c0):
  """A domain whose scaled diagonal is not positive voids the solve: the
  check runs after the solve (no extra synchronisation before it) and
  raises, as the reference's pivot test does (mas/local_inverse.py:43-65)."""
  import torch
  cube, _ = c0
  sc, _ = build(cube, "mas", mixed_spmv=True, stop_rule="residual")
  H = sc.minimizer.computeNumericValue()
  bs = H.block_sets[0]
  pos = bs.pattern.positions[:2 * bs.pattern.num_unique].cpu().numpy().reshape(-1, 2)
  k = int(np.nonzero((pos[:, 0] == 0) & (pos[:, 1] == 0))[0][0])
  off = int(bs.pattern.value_offset[k].item())
  bs.values[off:off + 9] = torch.tensor([-1.0, 0, 0, 0, -1.0, 0, 0, 0, -1.0], dtype=torch.float64, device="cuda")
  solver = sc.minimizer.linearSolver
  with pytest.raises(np.linalg.LinAlgError):
    solver.computeSolution(H, H.gradient, None, tolerance=1e-6, maxIterations=50, zero_initial_guess=True)
