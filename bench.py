#!/usr/bin/env python
"""Newton solves/sec of the YASPS inner loop on B200.

Workload (one step = one Newton step): Stable Neo-Hookean + implicit-Euler
inertia on a 64x64x64 vertex cube (262,144 vertices, 1,500,282 tets, z=0
layer pinned: 774,144 DoF), E=1e6, nu=0.45, noise +-0.005, dt=1/100,
gravity -9.8 z.  A step evaluates every element gradient and SPD-projected
Hessian, assembles the 3x3 block matrix, rebuilds the MAS preconditioner
(32-vertex Morton domains) and solves H x = g to a true relative residual of
1e-6 in the precision form (FP32 SpMV/MAS, FP64 dots and FP64 refinement).
The plain FP64 path (FP64 SpMV) is timed beside it (``fp64``).

``value``: whole-job solves/s with the scene resident on the device.
``e2e``: the same through ``scene.minimizeEnergy`` with host positions copied
in and the solution copied out every step.
``serving``: the serving form on a seeded stream of 512 FEM Newton steps
(Poisson arrivals, sides 8..48): continuous batching in the precision form
beside the serial plain FP64 path, solves/s and p50/p99 latency (rank 0, N=1).
``cloth_contact``: Newton steps of the mixed cloth + affine bodies + contact
scene (StVK, bending, 16 icosphere bodies, 200k barrier pairs, friction) in
both precision forms (rank 0, N=1).
``error_vs_oracle``: the device gradient, assembled Hessian and solutions
against one whole FP64 CPU Newton step of the same workload (oracle), which
is also ``cpu_baseline`` (rank 0, N=1).
``--impl reference``: whole CPU Newton steps of the same workload (the oracle
restatement of the reference path), rank 0 only.

Launch: ``python bench.py --gpus N --steps K --warmup W``; for N>1 under
torchrun every rank solves its own independent scene (replicas, weak scaling).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Newton solves/sec at 1e-6 rel. residual, FP32+refine vs FP64; p50/p99 latency"


def parse():
  p = argparse.ArgumentParser()
  p.add_argument("--gpus", type=int, default=1)
  p.add_argument("--steps", type=int, default=30)
  p.add_argument("--warmup", type=int, default=3)
  p.add_argument("--impl", default="b200", choices=["b200", "reference"])
  p.add_argument("--side", type=int, default=64, help="cube side in vertices")
  p.add_argument("--no-cpu-baseline", action="store_true")
  p.add_argument("--tol", type=float, default=1e-6)
  p.add_argument("--no-cloth", action="store_true", help="skip the cloth + contact leg")
  p.add_argument("--serving-requests", type=int, default=512,
                 help="requests of the serving stream (0: skip the serving leg)")
  p.add_argument("--workload", default="fem64", choices=["fem64", "mixed-serving"],
                 help="fem64: the headline line; mixed-serving: only the mixed serving stream (64 cloth + "
                      "affine-body + contact scenes beside 8 FEM cubes of 126^3 vertices, 150 GB budget)")
  return p.parse_args()


def workload(side, seed):
  from yasps_b200 import scenes
  return scenes.fem_cube(side, spacing=0.1, young=1e6, poisson=0.45, noise=0.005, seed=seed)


def config(cube, extra=None):
  c = {"workload": f"SNH+inertia FEM cube {cube.n}^3 verts, {cube.tet_count} tets, {cube.dofs} DoF, "
                   "MAS 32-vertex Morton domains, solve to 1e-6 true relative residual",
       "vertices": cube.n ** 3, "tets": cube.tet_count, "dof": cube.dofs, "young": 1e6, "poisson": 0.45,
       "l2": "working set > L2 (element records ~1.1 GB, MAS inverses ~0.3 GB, blocks 0.15 GB)"}
  if extra:
    c.update(extra)
  return c


class Clocks:
  """nvidia-smi samples during the timed region."""

  FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
            "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
            "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

  def __init__(self, device):
    self.device = device
    self.proc = None
    self.file = None

  def start(self):
    try:
      self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
      self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                    "-lms", "50", "-i", str(self.device)], stdout=self.file,
                                   stderr=subprocess.DEVNULL)
    except Exception:
      self.proc = None
      return
    # nvidia-smi takes a moment to start: hold the timed region until the
    # first sample is written (at most 5 s)
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
      if os.path.getsize(self.file.name) > 0:
        break
      time.sleep(0.02)

  def stop(self):
    if self.proc is None:
      return None
    time.sleep(0.06)
    self.proc.terminate()
    try:
      self.proc.wait(timeout=5)
    except Exception:
      self.proc.kill()
    self.file.flush()
    self.file.seek(0)
    rows = [l.split(",") for l in self.file.read().strip().splitlines() if l.strip()]
    os.unlink(self.file.name)
    sm, mx, reasons = [], 0.0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for r in rows:
      try:
        sm.append(float(r[1]))
        mx = max(mx, float(r[2]))
        for name, v in zip(names, r[5:9]):
          if v.strip().lower() == "active":
            reasons.add(name)
      except (ValueError, IndexError):
        continue
    if not sm:
      return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
  try:
    with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
      d = json.load(f)
    return float(d["hbm_gbs"]), "measured"
  except Exception:
    return 6650.0, "fallback"


def dist_setup(args):
  import torch
  rank = int(os.environ.get("RANK", "0"))
  world = int(os.environ.get("WORLD_SIZE", "1"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  if torch.cuda.is_available():
    torch.cuda.set_device(local)
  pg = None
  if world > 1:
    import datetime
    import torch.distributed as dist
    if torch.cuda.is_available():
      dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                              device_id=torch.device("cuda", local))
    else:  # host-only ranks (the multi-rank logic tested on CPU)
      dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    pg = dist
  return rank, world, local, pg


def max_over_ranks(x, pg):
  if pg is None:
    return x
  import torch
  dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
  t = torch.tensor([x], dtype=torch.float64, device=dev)
  pg.all_reduce(t, op=pg.ReduceOp.MAX)
  return float(t.item())


def replica_value(world, steps, ms):
  """Whole-job solves/s of `world` replicas that each ran `steps` Newton
  steps, the slowest in `ms` milliseconds (max over ranks)."""
  return world * steps / (ms / 1e3)


def barrier(pg):
  if pg is not None:
    pg.barrier()


def time_steps(fn, steps, pg):
  import torch
  lat = []
  torch.cuda.synchronize()
  barrier(pg)
  torch.cuda.synchronize()
  start = torch.cuda.Event(enable_timing=True)
  end = torch.cuda.Event(enable_timing=True)
  start.record()
  for _ in range(steps):
    t0 = time.perf_counter()
    fn()
    lat.append(time.perf_counter() - t0)
  end.record()
  torch.cuda.synchronize()
  barrier(pg)
  ms = start.elapsed_time(end)
  return max_over_ranks(ms, pg), lat


def gpu_arm(args):
  import torch
  from yasps_b200 import _lib as L
  from yasps_b200 import scenes
  rank, world, local, pg = dist_setup(args)
  L.load()
  cube = workload(args.side, seed=rank)
  sc, h = scenes.fem_scene(cube)
  mz = sc.minimizer
  solver = mz.setSolver("mas", mixed_spmv=True, stop_rule="residual")
  step = lambda: mz.computeHessianAndGradient(tolerance=args.tol, maxIterations=2000)
  for _ in range(max(args.warmup, 3)):
    step()
  stats = dict(solver.statistics)
  clocks = Clocks(local)
  clocks.start()
  ms, lat = time_steps(step, args.steps, pg)
  clk = clocks.stop()
  stats = dict(solver.statistics)
  impl = solver.implementation
  rel_res = float(getattr(impl, "final_relative_residual", float("nan")))
  Hs = mz.activeHessian()
  device_out = {"g": Hs.gradient.value.cpu().numpy(), "pos": Hs.block_positions.cpu().numpy(),
                "val": Hs.blocks_flattened.cpu().numpy(), "x": {"fp32_refine": impl.solution.cpu().numpy()}}
  value = replica_value(world, args.steps, ms)
  lat_ms = sorted(1e3 * x for x in lat)
  levels = len(impl.hierarchy.levels)
  its, refs = int(stats["iterations"]), int(stats.get("refinements", 1))
  launches_per_step = launches_per_newton_step(impl, its, refs)
  # plain FP64 path on the same scene
  solver64 = mz.setSolver("mas", mixed_spmv=False, stop_rule="residual")
  for _ in range(2):
    step()
  ms64, _ = time_steps(step, max(3, args.steps // 3), pg)
  fp64_value = replica_value(world, max(3, args.steps // 3), ms64)
  stats64 = dict(solver64.statistics)
  device_out["x"]["fp64"] = solver64.implementation.solution.cpu().numpy()
  # end to end through the public API with host buffers
  mz.setSolver("mas", mixed_spmv=True, stop_rule="residual")
  host_pos = torch.from_numpy(np.ascontiguousarray(cube.free_position.reshape(-1))).pin_memory()
  out_host = torch.empty(cube.dofs, dtype=torch.float64).pin_memory()
  fp = h["free_position"]

  def e2e_step():
    fp.updateValue(host_pos)
    segs = sc.minimizeEnergy(tolerance=args.tol, maxIterations=2000)
    out_host.copy_(segs[0])
  fp.updateValue(host_pos.cuda())
  for _ in range(2):
    e2e_step()
  ms_e2e, _ = time_steps(e2e_step, max(3, args.steps // 3), pg)
  e2e_value = replica_value(world, max(3, args.steps // 3), ms_e2e)
  # roofline of the MAS domain GEMV, timed on its own stream
  ms_solver = mz.linearSolver.implementation
  H = mz.activeHessian()
  import ctypes
  nbytes = ctypes.c_uint64(0)
  s = torch.cuda.current_stream()
  L.call("ys_mas_gemv", ms_solver._mas, s.cuda_stream, ctypes.byref(nbytes))
  reps = 50
  torch.cuda.synchronize()
  e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
  e0.record(s)
  for _ in range(reps):
    L.call("ys_mas_gemv", ms_solver._mas, s.cuda_stream, None)
  e1.record(s)
  torch.cuda.synchronize()
  gemv_ms = e0.elapsed_time(e1) / reps
  hbm, peak_kind = peaks()
  achieved = nbytes.value / (gemv_ms / 1e3) / 1e9
  # DRAM traffic per launch from an ncu capture of the 56^3 cube (109.60 MB
  # read + 7.08 MB written; its tiled layout holds GEMV_LAYOUT_56 bytes),
  # scaled by this launch's layout bytes (traffic grows with the domains)
  from yasps_b200.kernelbench import gemv_layout_bytes
  traffic = (109.60e6 + 7.08e6) / GEMV_LAYOUT_56 * gemv_layout_bytes(ms_solver._tables)
  roofline_gemv = {"kernel": "mas_gemv (MAS domain-inverse apply, FP32)", "bound": "hbm", "achieved": achieved,
                   "peak": hbm, "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                   "traffic": traffic, "bytes_per_launch": int(nbytes.value), "ms_per_launch": gemv_ms}
  # the headline roofline is the step's dominant kernel: the SpMV of the PCG
  # loop (one launch an iteration)
  roofline = spmv_roofline(mz.activeHessian(), hbm, peak_kind, args.side)
  # the host-bound serving loop runs before the CPU baseline, whose worker
  # threads would otherwise compete with it for the host cores
  serve = None
  if rank == 0 and world == 1 and args.serving_requests > 0:
    serve = serving_leg(args)
  cloth = None
  if rank == 0 and world == 1 and not args.no_cloth:
    cloth = cloth_leg(args)
  cpu, err = None, None
  if rank == 0 and world == 1 and not args.no_cpu_baseline:
    cpu, err = cpu_step_leg(cube, args.tol, (device_out["g"], device_out["pos"], device_out["val"],
                                             device_out["x"]))
  line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
          "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
          "vs_baseline": None, "dtype": "f32+f64 refine (f64 element Hessians and projection)",
          "data": "synthetic (seeded FEM cube, no external data)",
          "config": config(cube, {"parallelism": f"replicas x{world}", "path": "fp32+refine",
                                  "iterations": its, "refinements": refs, "levels": levels,
                                  "true_rel_residual": rel_res}),
          "p50_ms": lat_ms[len(lat_ms) // 2], "p99_ms": lat_ms[min(len(lat_ms) - 1, int(0.99 * len(lat_ms)))],
          "fp64": {"value": fp64_value, "unit": "solves/s", "iterations": int(stats64["iterations"])},
          "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": 8 * cube.dofs,
                  "d2h_bytes_per_step": 8 * cube.dofs},
          "gpu_launches": int(launches_per_step * args.steps), "roofline": roofline,
          "roofline_gemv": roofline_gemv, "clocks": clk,
          "cpu_baseline": cpu, "error_vs_oracle": err, "serving": serve, "cloth_contact": cloth}
  if rank == 0:
    print(json.dumps(line), flush=True)
  if pg is not None:
    pg.destroy_process_group()


GEMV_LAYOUT_56 = 111_651_744  # tiled-layout bytes of one domain-GEMV launch on the 56^3 cube


# DRAM bytes (read + write) of one streamed-tile SpMV launch on this 64^3
# workload, from an ncu capture of the same launch (dram__bytes.sum.per_second
# x gpu__time_duration.sum = 3.2909 TB/s x 37.984 us); None on other sizes
SPMV_STREAM_TRAFFIC_64 = 125.00e6


def spmv_roofline(H, hbm, peak_kind, side, reps=50):
  """The SpMV of the FP32 PCG loop timed alone with CUDA events over `reps`
  launches on its stream: the streamed-tile kernel (each tile's packed FP32
  blocks, entry words and row offsets staged in shared memory by bulk
  copies, its distinct neighbour vectors gathered once), or the tiled one
  for a block set without a streamed plan.  Algorithmic bytes per launch
  (the symmetric storage's own count): nb (9 * 4 + 8) for the stored FP32
  blocks and two 32-bit indices each, plus the vector read and the product
  written once in FP64, 2 * 8 * n."""
  import torch
  from yasps_b200 import _lib as L
  bs = H.block_sets[0]
  row_ptr, eb, ec = H.spmv_plan(bs)
  row_block, cap, ecap = H.tile_plan(bs)
  sp = H.stream_plan(bs)
  nv = H.rows // 3
  entries = int(row_ptr[nv].item())
  x = torch.cos(torch.arange(H.rows, dtype=torch.float64, device="cuda") * 0.37)
  x32 = torch.empty(4 * nv, dtype=torch.float32, device="cuda")
  y = torch.empty_like(x)
  s = torch.cuda.current_stream()
  L.call("ys_pack_x32", L.ptr(x), nv, L.ptr(x32), s.cuda_stream)
  if sp is not None:
    st = sp.struct()
    name = "spmv3_x32_stream (streamed-tile symmetric 3x3 block SpMV of the FP32 PCG loop)"
    call = lambda: L.call("ys_spmv3_x32_streamed", st, L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), nv,
                          L.ptr(x32), L.ptr(y), 0, 0, 0, None, s.cuda_stream)
  else:
    name = "spmv3_x32_tiled (tiled symmetric 3x3 block SpMV of the FP32 PCG loop)"
    call = lambda: L.call("ys_spmv3_x32_tiled", L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec),
                          L.ptr(row_block), cap, ecap, 0, nv, L.ptr(x32), L.ptr(y), 0, None, s.cuda_stream)
  for _ in range(3):
    call()
  torch.cuda.synchronize()
  e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
  e0.record(s)
  for _ in range(reps):
    call()
  e1.record(s)
  torch.cuda.synchronize()
  ms = e0.elapsed_time(e1) / reps
  nb = bs.pattern.num_unique
  nbytes = nb * (9 * 4 + 8) + 2 * 8 * H.rows
  achieved = nbytes / (ms / 1e3) / 1e9
  out = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": hbm, "peak_source": peak_kind, "unit": "GB/s",
         "frac": achieved / hbm,
         "traffic": SPMV_STREAM_TRAFFIC_64 if (side == 64 and sp is not None) else None,
         "bytes_per_launch": nbytes, "ms_per_launch": ms, "stored_blocks": nb, "entries": entries}
  if sp is not None:
    out.update({"stream_block_cap": sp.block_cap, "stream_entry_cap": sp.entry_cap, "stream_halo_cap": sp.halo_cap})
  else:
    out.update({"tile_cap": cap, "entry_cap": ecap})
  return out


def served_oracle_check(done, seed, count=8, max_side=30):
  """True relative residual ||g - H x|| / ||g|| of a sample of served
  solutions under g and H assembled by the FP64 oracle from the same request
  (cube side, material, seeded positions): the `count` requests of smallest
  side up to `max_side` (the oracle assembles serially)."""
  import dataclasses
  from oracle import solvers
  from tests.oracle_scene import OracleCube
  from yasps_b200 import scenes
  pick = sorted((r for r in done if r.side <= max_side), key=lambda r: (r.side, r.tag))[:count]
  res = []
  for r in pick:
    cube = scenes.fem_cube(r.side, noise=0.01, seed=seed * 1000003 + int(r.tag))
    cube = dataclasses.replace(cube, mu=r.mu, lam=r.lam)
    ora = OracleCube(cube)
    res.append(solvers.relative_residual(ora.matvec, ora.gradient, r.solution))
  return {"oracle": "FP64 CPU assembly of each sampled request", "requests": [int(r.tag) for r in pick],
          "sides": [int(r.side) for r in pick], "rel_residuals": res, "max_rel_residual": max(res) if res else None}


def launches_per_newton_step(impl, its, refs):
  """Kernels of this library launched in one Newton step of the precision form.

  Element stage: SNH eval + projection, inertia, block and gradient assembly,
  diagonal extraction (6).  MAS numeric update: one Galerkin sum per coarse
  level and the domain inverses.  Refinement: the initial residual (1) and per
  refinement x += d and r = g - H x (2).  Each PCG solve: init = residual,
  the grid restrictions of the levels above 64 nodes, the one-CTA tail of the
  rest, the level-0 and the coarse domain GEMVs, collect; every iteration =
  SpMV+dot, update (+ level-1 restriction), grid restrictions from level 2,
  tail, the two GEMVs, collect + direction (one cooperative kernel).
  """
  t = impl._tables
  offs = [int(v) for v in t.level_node_offset]
  levels = len(offs) - 1
  first = levels
  while first > 1 and offs[first] - offs[first - 1] <= 64:
    first -= 1
  coarse = 1 if levels > 1 else 0
  tail_init = 1 if first < levels else 0
  init = 1 + (first - 1) + tail_init + 1 + coarse + 1
  if levels > 1:
    f_it = max(first, 2)
    per_it = 2 + (first - 2 if first > 2 else 0) + (1 if f_it < levels else 0) + 1 + coarse + 1
  else:
    per_it = 2 + 1 + 2
  return 6 + (levels - 1) + 1 + 1 + 2 * refs + refs * init + its * per_it


def cloth_leg(args):
  """Mixed cloth + contact Newton steps (StVK membrane, bending, 100k PT + 100k
  EE barriers, PT friction, inertia; 256^2 cloth over a static obstacle, 16
  icosphere affine bodies resting on it through body-cloth PT pairs):
  precision form and plain FP64, CUDA-event timed."""
  import torch
  from yasps_b200 import scenes
  cc = scenes.cloth_contact(256, 200_000, num_bodies=16)
  sc, _ = scenes.cloth_contact_scene(cc)
  mz = sc.minimizer
  nbp = len(cc.body_pt)
  out = {"workload": ("256x256 cloth (65,536 verts, 130,050 tris) StVK E=1e4 nu=0.3 h=1e-3, bending kb=1e-3, "
                      "16 affine bodies (icospheres of 2,562 verts, 12 DoF each, orthogonality 1e5, inertia), "
                      f"{nbp} body-cloth + {100_000 - nbp} cloth-obstacle point-triangle and 100k edge-edge "
                      "log-barrier pairs (d-hat 1e-3, squared distances in (0.1, 1) d-hat), lagged PT friction "
                      "mu=0.3, cloth inertia; solve to 1e-6 true relative residual"),
         "body_cloth_pairs": nbp}
  for name, mixed in (("fp32_refine", True), ("fp64", False)):
    solver = mz.setSolver("mas", mixed_spmv=mixed, stop_rule="residual")
    step = lambda: mz.computeHessianAndGradient(tolerance=args.tol, maxIterations=5000)
    for _ in range(2):
      step()
    ms, _ = time_steps(step, 5, None)
    st = solver.statistics
    out[name] = {"solves_per_s": 5 / (ms / 1e3), "ms_per_step": ms / 5, "iterations": int(st["iterations"]),
                 "refinements": int(st.get("refinements", 0))}
    # the solution checked on the host in FP64 against the FP64 system the
    # device assembled (each element kind of it matches the oracle in the
    # tests): an independent residual, not the solver's own
    Hc = mz.activeHessian()
    pos3, val3 = Hc.blocks3()
    A = blocks_to_csr(pos3.cpu().numpy(), val3.cpu().numpy(), Hc.rows)
    g = Hc.gradient.value.cpu().numpy()
    x = solver.implementation.solution.cpu().numpy()
    out[name]["host_fp64_rel_residual"] = float(np.linalg.norm(g - A @ x) / np.linalg.norm(g))
  impl = mz.linearSolver.implementation
  out["dof"] = mz.activeHessian().rows
  out["blocks"] = int(mz.activeHessian()._static.pattern.num_unique)
  return out


def mixed_serving_leg(args):
  """The mixed serving stream: 64 cloth + affine-body + contact scenes (cloth
  side U{64..256}, 2..16 icosphere bodies, 10k..200k barrier pairs, each its
  own topology) interleaved with 8 FEM cubes of 126^3 vertices (E=1e6,
  nu=0.45, noise +-0.005), Poisson arrivals (mean gap 2 ms) and all at once,
  a 150 GB admission budget; the precision form served beside the serial
  plain FP64 path.  Errors: every solution's true relative residual under the
  device FP64 system, and under the FP64 oracle's system for a sample (the
  three smallest and the largest cloth scene, one FEM cube)."""
  import torch
  from oracle import baseline, cloth_scene
  from yasps_b200 import scenes, serving
  wl = serving.mixed_workload(seed=0)
  srv = serving.NewtonServer(max_slots=len(wl.order), passes=8, memory_budget=150e9, tolerance=args.tol,
                             max_iterations=5000)
  t0 = time.perf_counter()
  for spec in wl.scenes:
    srv.add_topology(serving.cloth_scene_topology(spec))
  srv.register([sp.key for sp in wl.scenes], slots_per_side=1)
  srv.register([wl.fem_side], slots_per_side=len(wl.fem))
  t_register = time.perf_counter() - t0
  hbm, peak_kind = peaks()
  fem_topo = srv.topology(wl.fem_side)
  big = max(wl.scenes, key=lambda sp: sp.side)
  spmv = {"fem_126": spmv_roofline(fem_topo.H, hbm, peak_kind, wl.fem_side),
          "cloth_largest": spmv_roofline(srv.topology(big.key).H, hbm, peak_kind, big.side)}
  for v in spmv.values():
    v["traffic"] = None
  # warm-up: the stream once each way (CUDA graphs of the size buckets, the
  # FP64 solver state of every topology)
  srv.run(wl.requests(srv))
  srv.solve_serial_fp64(wl.requests(srv))
  clocks = Clocks(torch.cuda.current_device())
  clocks.start()
  created = srv.slots_created
  done = srv.run(wl.requests(srv))
  out = {"workload": (f"{len(wl.scenes)} cloth + affine-body + contact scenes (cloth side U{{64..256}}, 2..16 "
                      f"icosphere bodies of 2,562 vertices, 10k..200k barrier pairs, lagged PT friction; each "
                      f"its own topology) interleaved with {len(wl.fem)} SNH FEM cubes of {wl.fem_side}^3 vertices "
                      f"({(wl.fem_side - 1) ** 3 * 6:,} tets, E=1e6, nu=0.45, noise +-0.005); Poisson arrivals "
                      "(mean gap 2 ms) and all at once; 150 GB admission budget; solve to 1e-6 true relative "
                      "residual"),
         "register_topologies_s": t_register,
         "cloth_vertices": int(sum(sp.side ** 2 for sp in wl.scenes)),
         "fem_dof_each": int(fem_topo.n)}
  out["served"] = serving.stream_stats(done)
  out["served_saturated"] = serving.stream_stats(srv.run(wl.requests(srv, all_at_once=True)))
  out["serial_fp64"] = serving.stream_stats(srv.solve_serial_fp64(wl.requests(srv)))
  out["serial_fp64_saturated"] = serving.stream_stats(srv.solve_serial_fp64(wl.requests(srv, all_at_once=True)))
  out["clocks"] = clocks.stop()
  out["slots_created_while_timed"] = srv.slots_created - created
  out["resident_slot_gb"] = srv.resident_bytes / 1e9
  out["max_allocated_gb"] = torch.cuda.max_memory_allocated() / 1e9
  out["spmv_roofline"] = spmv
  # errors: device FP64 residual of every solution, oracle residual of a sample
  out["served"]["max_rel_residual"] = max(r.relative_residual for r in done)
  by_tag = {r.tag: r for r in done}
  cloth_tags = sorted((k for k, (kind, _) in enumerate(wl.order) if kind == "cloth"),
                      key=lambda k: wl.scenes[wl.order[k][1]].side)
  sample = cloth_tags[:3] + cloth_tags[-1:]
  oracle = {"oracle": "FP64 CPU restatement (matrix-free g and H x of each sampled request)", "cloth": {}}
  for k in sample:
    sp = wl.scenes[wl.order[k][1]]
    cc = srv.topology(sp.key).cloth
    oracle["cloth"][f"side{sp.side}_bodies{sp.bodies}_pairs{sp.pairs}"] = cloth_scene.relative_residual(
        cc, by_tag[k].solution)
  fem_tag = next(k for k, (kind, _) in enumerate(wl.order) if kind == "fem")
  f = wl.fem[wl.order[fem_tag][1]]
  cube = scenes.fem_cube(wl.fem_side, young=f["young"], poisson=f["poisson"], noise=f["noise"], seed=f["seed"])
  oracle[f"fem_{wl.fem_side}"] = baseline.relative_residual_pooled(cube, by_tag[fem_tag].solution)
  oracle["max_rel_residual"] = max(list(oracle["cloth"].values()) + [oracle[f"fem_{wl.fem_side}"]])
  out["served"]["error_vs_oracle"] = oracle
  srv.close()
  return out


def serving_leg(args):
  """Serving form on a seeded Poisson stream of FEM Newton steps (one GPU):
  continuous batching (FP32+refine) beside the serial plain FP64 path."""
  import torch
  from yasps_b200 import serving
  n = args.serving_requests
  srv = serving.NewtonServer(max_slots=64, passes=8, memory_budget=40e9, tolerance=args.tol)
  t0 = time.perf_counter()
  srv.register(range(8, 49), slots_per_side=3)
  t_register = time.perf_counter() - t0
  srv.run(serving.poisson_fem_stream(count=82, mean_spacing=0.0, seed=99))
  # steady state: pools sized for the timed streams (no slot, a device
  # allocation that synchronises, is created inside them) and an untimed
  # pass of the two timed streams (the CUDA graphs of their size buckets)
  srv.reserve(serving.poisson_fem_stream(count=n, mean_spacing=2e-3, seed=0))
  srv.run(serving.poisson_fem_stream(count=n, mean_spacing=2e-3, seed=0))
  srv.run(serving.poisson_fem_stream(count=n, mean_spacing=0.0, seed=0))
  srv.solve_serial_fp64(serving.poisson_fem_stream(count=41, mean_spacing=0.0, seed=98))
  out = {"workload": (f"{n} FEM Newton-step requests, Poisson arrivals (mean gap 2 ms), cube side U{{8..48}}, "
                      "E log-uniform [1e4, 1e6], nu U[0.3, 0.45], noise +-0.01, 40 GB admission budget, "
                      "solve to 1e-6 true relative residual"),
         "register_topologies_s": t_register}
  clocks = Clocks(torch.cuda.current_device())
  clocks.start()
  created = srv.slots_created
  done = srv.run(serving.poisson_fem_stream(count=n, mean_spacing=2e-3, seed=0))
  out["served"] = serving.stream_stats(done)
  out["served"]["max_rel_residual"] = max(r.relative_residual for r in done)
  out["served"]["error_vs_oracle"] = served_oracle_check(done, seed=0)
  out["served_saturated"] = serving.stream_stats(
      srv.run(serving.poisson_fem_stream(count=n, mean_spacing=0.0, seed=0)))
  out["serial_fp64"] = serving.stream_stats(
      srv.solve_serial_fp64(serving.poisson_fem_stream(count=n, mean_spacing=2e-3, seed=0)))
  out["serial_fp64_saturated"] = serving.stream_stats(
      srv.solve_serial_fp64(serving.poisson_fem_stream(count=n, mean_spacing=0.0, seed=0)))
  out["clocks"] = clocks.stop()
  out["resident_gb"] = srv.resident_bytes / 1e9
  out["slots_created_while_timed"] = srv.slots_created - created
  srv.close()
  return out


def blocks_to_csr(positions, values, n):
  """Symmetric CSR of upper 3x3 block storage (scalar block offsets)."""
  import scipy.sparse as sp
  pos = np.asarray(positions, dtype=np.int64).reshape(-1, 2)
  vals = np.asarray(values, dtype=np.float64)[:9 * len(pos)].reshape(-1, 3, 3)
  k = np.arange(3)
  rows = (pos[:, 0, None, None] + k[None, :, None]).repeat(3, axis=2)
  cols = (pos[:, 1, None, None] + k[None, None, :]).repeat(3, axis=1)
  up = sp.coo_matrix((vals.ravel(), (rows.ravel(), cols.ravel())), shape=(n, n)).tocsr()
  off = pos[:, 0] != pos[:, 1]
  lo = sp.coo_matrix((vals[off].ravel(), (rows[off].ravel(), cols[off].ravel())), shape=(n, n)).tocsr().T
  return (up + lo).tocsr()


def cpu_step_leg(cube, tol, gpu=None):
  """One whole, unsampled CPU Newton step of the workload (the oracle's
  restatement of the reference's CPU path: every element, the full MAS
  update, MAS-PCG to the target), timed; and, with ``gpu`` = (g, positions,
  values, {name: x}) from the device, the device's error against this FP64
  oracle: gradient and assembled Hessian (largest entry difference relative
  to the largest entry) and the true relative residual ``||g - H x|| / ||g||``
  of each device solution under the oracle's g and H."""
  from oracle import baseline
  t0 = time.perf_counter()
  pool = baseline.ElementPool(cube)
  threads = pool.workers
  try:
    g0, H0 = pool.assemble()
    mas = baseline.CpuMas(H0, cube.free_count)
    setup_s = time.perf_counter() - t0
    g, H, x, its, phases = baseline.cpu_newton_step(cube, mas, tol=tol, pool=pool)
  finally:
    pool.close()
  cpu = {"value": 1.0 / phases["total_s"], "unit": "solves/s", "cores": threads, "kind": "port",
         "sample": (f"one whole Newton step of the same workload, unsampled (oracle NumPy/SciPy restatement "
                    f"of the reference CPU path; elements on {threads} worker processes, BLAS threads for the "
                    f"rest): all {cube.tet_count} tets' SNH + projection + assembly, the MAS update of every "
                    f"domain, {its} MAS-PCG iterations to the target residual; hierarchy built once beforehand "
                    f"({setup_s:.1f} s with the first assembly, cached per structure as in the reference)"),
         "steps_timed": 1, "breakdown_s": phases}
  err = None
  if gpu is not None:
    g_dev, pos_dev, val_dev, xs = gpu
    Hd = blocks_to_csr(pos_dev, val_dev, cube.dofs)
    gn = float(np.linalg.norm(g))
    err = {"oracle": "FP64 CPU restatement, same seeded inputs",
           "gradient_rel_max": float(np.abs(g_dev - g).max() / np.abs(g).max()),
           "hessian_rel_max": float(abs(Hd - H).max() / abs(H).max()),
           "cpu_solution_rel_residual": float(np.linalg.norm(g - H @ x) / gn)}
    for name, xd in xs.items():
      err[f"{name}_rel_residual"] = float(np.linalg.norm(g - H @ xd) / gn)
  return cpu, err


def reference_arm(args):
  """Whole, unsampled CPU Newton steps of the workload (the oracle port of
  the reference's CPU path; the reference itself is Python and does not
  travel to the GPU box).  Steps are timed whole, after one untimed
  assembly: the requested count, or fewer when the next step would take the
  timed region past two minutes (at least one); the line says how many ran."""
  rank = int(os.environ.get("RANK", "0"))
  if rank != 0:
    return
  from oracle import baseline
  cube = workload(args.side, seed=0)
  pool = baseline.ElementPool(cube)
  threads = pool.workers
  try:
    g0, H0 = pool.assemble()  # warm-up: the first assembly
    mas = baseline.CpuMas(H0, cube.free_count)
    totals, its = [], 0
    t0 = time.perf_counter()
    while len(totals) < args.steps:
      _, _, _, its, ph = baseline.cpu_newton_step(cube, mas, tol=args.tol, pool=pool)
      totals.append(ph["total_s"])
      if time.perf_counter() - t0 + ph["total_s"] > 120.0:
        break
    wall = time.perf_counter() - t0
  finally:
    pool.close()
  steps = len(totals)
  value = steps / wall
  cpu = {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
         "sample": (f"{steps} whole Newton steps timed (of {args.steps} requested; the timed region stops before "
                    f"it would pass 120 s), unsampled: every tet, the full MAS update, {its} MAS-PCG iterations to "
                    f"1e-6 true relative residual; oracle NumPy/SciPy restatement of the reference CPU path, "
                    f"elements on {threads} worker processes"),
         "steps_timed": steps}
  lat = sorted(1e3 * t for t in totals)
  line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1,
          "steps": steps, "steps_requested": args.steps, "warmup": args.warmup, "warmup_done": 1,
          "ms_per_step": 1e3 * wall / steps,
          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
          "data": "synthetic (seeded FEM cube)",
          "config": config(cube, {"parallelism": "cpu", "path": "fp64", "iterations": its}),
          "p50_ms": lat[len(lat) // 2], "p99_ms": lat[-1],
          "cpu_baseline": cpu, "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                                       "d2h_bytes_per_step": 0}}
  print(json.dumps(line), flush=True)


def mixed_arm(args):
  """``--workload mixed-serving``: the mixed serving stream alone (rank 0 of
  one GPU), one JSON line whose value is the served stream's solves/s."""
  import torch
  if int(os.environ.get("WORLD_SIZE", "1")) > 1 and int(os.environ.get("RANK", "0")) != 0:
    return
  torch.cuda.set_device(0)
  out = mixed_serving_leg(args)
  line = {"metric": METRIC, "value": out["served"]["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
          "dtype": "f32+f64 refine (f64 element Hessians, projection and barrier terms)",
          "data": "synthetic (seeded cloth, body and FEM scenes, no external data)",
          "config": {"workload": out["workload"], "parallelism": "one GPU, continuous batching"},
          "p50_ms": out["served"]["p50_ms"], "p99_ms": out["served"]["p99_ms"], "mixed_serving": out}
  print(json.dumps(line), flush=True)


def main():
  args = parse()
  if args.impl == "reference":
    reference_arm(args)
  elif args.workload == "mixed-serving":
    mixed_arm(args)
  else:
    gpu_arm(args)


if __name__ == "__main__":
  main()
