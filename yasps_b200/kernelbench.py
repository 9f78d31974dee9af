"""Per-kernel timing of the Newton inner loop on one FEM cube.

``python -m yasps_b200.kernelbench --side 64 [--kernel all|gemv|spmv|...] [--reps 20]``

Builds the cube workload, runs one Newton step (``masSolver(mixed_spmv=True)``)
and then launches each kernel stage again ``--reps`` times, timing it with
CUDA events on the launching stream.  Also the case driver for ncu captures
(``--kernel gemv --reps 3`` launches the GEMV stage three times).
"""

from __future__ import annotations

import argparse
import ctypes
import json

import numpy as np

import torch

from . import _lib as L
from . import scenes


def _time(fn, reps):
  s = torch.cuda.current_stream()
  fn()
  torch.cuda.synchronize()
  e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
  e0.record(s)
  for _ in range(reps):
    fn()
  e1.record(s)
  torch.cuda.synchronize()
  return e0.elapsed_time(e1) / reps


def cloth_main(args):
  """Cloth + contact scene (StVK, bending, PT/EE barriers, PT friction)."""
  cc = scenes.cloth_contact(args.side, args.pairs)
  sc, _ = scenes.cloth_contact_scene(cc)
  mz = sc.minimizer
  mz.setSolver("mas", mixed_spmv=True, stop_rule="residual")
  mz.computeHessianAndGradient(tolerance=1e-6, maxIterations=2000)
  torch.cuda.synchronize()
  H = mz.activeHessian()
  bs = H._static
  out = {"scene": "cloth_contact", "side": args.side, "pairs": args.pairs, "dof": H.rows,
         "blocks": bs.pattern.num_unique, "pcg": mz.linearSolver.statistics}
  for d in bs.infos:
    t = d["term"]
    plan = H._term_plan(d, bs)
    name = type(t.expr).__name__
    out[name + "_ms"] = _time(lambda: t.evaluate(plan, bs.records, H._grad_records), args.reps)
    out[name + "_elements"] = t.n
  out["compute_ms"] = _time(lambda: H.compute(), max(2, args.reps // 4))
  out["newton_step_ms"] = _time(lambda: mz.computeHessianAndGradient(tolerance=1e-6, maxIterations=2000),
                                max(2, args.reps // 5))
  print(json.dumps(out))


def gemv_layout_bytes(tables) -> int:
  """Bytes one domain-GEMV launch reads and writes in the tiled inverse
  layout: every tile of every inverse, the gathered residual, node ids and
  the correction."""
  from yasps_b200.mas_hierarchy import inverse_floats
  sizes = np.diff(np.asarray(tables.dom_node_ptr, dtype=np.int64))
  return int(sum(4 * inverse_floats(3 * int(k)) + 28 * int(k) for k in sizes))


def trace_pcg(run):
  """Kernels of one PCG graph launch with their device durations, from the
  CUDA activity torch.profiler records (the kernels of the conditional loop
  body are reported for one iteration)."""
  from torch.profiler import ProfilerActivity, profile
  run()
  torch.cuda.synchronize()
  with profile(activities=[ProfilerActivity.CUDA]) as prof:
    run()
    torch.cuda.synchronize()
  events = [e for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA]
  events.sort(key=lambda e: e.time_range.start)
  rows = [{"kernel": e.name, "start_us": e.time_range.start, "us": e.time_range.elapsed_us()} for e in events]
  t0 = rows[0]["start_us"] if rows else 0
  for r in rows:
    r["start_us"] = round(r["start_us"] - t0, 1)
    r["us"] = round(r["us"], 1)
  print(json.dumps(rows, indent=1))


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument("--side", type=int, default=64)
  ap.add_argument("--kernel", default="all")
  ap.add_argument("--reps", type=int, default=20)
  ap.add_argument("--scene", default="fem", choices=["fem", "cloth"])
  ap.add_argument("--pairs", type=int, default=200_000)
  ap.add_argument("--trace-pcg", action="store_true",
                  help="print the kernels of one MAS-PCG launch (torch.profiler CUDA activity)")
  args = ap.parse_args()
  if args.scene == "cloth":
    return cloth_main(args)
  cube = scenes.fem_cube(args.side, young=1e6, poisson=0.45, noise=0.005)
  sc, _ = scenes.fem_scene(cube)
  mz = sc.minimizer
  mz.setSolver("mas", mixed_spmv=True, stop_rule="residual")
  mz.computeHessianAndGradient(tolerance=1e-6, maxIterations=2000)
  torch.cuda.synchronize()
  H = mz.activeHessian()
  mas = mz.linearSolver.implementation
  bs = H._static
  d = bs.infos[0]
  snh = d["term"]
  plan = H._term_plan(d, bs)
  p = bs.pattern
  st = L.stream_ptr()
  row_ptr, eb, ec = H.spmv_plan(bs)
  row_block, tile_cap, entry_cap = H.tile_plan(bs)
  x = torch.cos(torch.arange(H.rows, dtype=torch.float64, device="cuda") * 0.37)
  y = torch.zeros_like(x)
  z = torch.zeros_like(x)
  nv = H.rows // 3
  x32 = torch.empty(4 * nv, dtype=torch.float32, device="cuda")
  L.call("ys_pack_x32", L.ptr(x), nv, L.ptr(x32), st)

  def snh_eval(method):
    snh.projection_method = method
    snh.evaluate(plan, bs.records, H._grad_records)
    snh.projection_method = 1

  def tiled(stages):
    L.call("ys_spmv3_x32_tiled", L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), L.ptr(row_block),
           tile_cap, entry_cap, stages, nv, L.ptr(x32), L.ptr(y), 0, None, st)

  sp = H.stream_plan(bs)
  sps = sp.struct() if sp is not None else None

  def streamed(stages):
    L.call("ys_spmv3_x32_streamed", sps, L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), nv, L.ptr(x32),
           L.ptr(y), 0, stages, 0, None, st)

  def pcg_without_stream():
    keep = bs.stream
    bs.stream = False
    try:
      mas._run_pcg(H, H.gradient.value, z, True, L.YS_PREC_MAS, None, mas._mas, 1e-30, 50, True, "residual")
    finally:
      bs.stream = keep

  cases = {
      "snh_eval_only": lambda: snh_eval(0),
      "snh_eval_project": lambda: snh_eval(1),
      "assemble3": lambda: L.call("ys_assemble3", L.ptr(bs.records), L.ptr(p.record_begin), L.ptr(p.record_count),
                                  L.ptr(p.value_offset), p.num_unique, L.ptr(bs.values), L.ptr(bs.values32), st),
      "mas_numeric": lambda: mas.numeric_update(H, check=False),
      "spmv_fp64": lambda: L.call("ys_spmv3", L.ptr(bs.values), None, L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), nv,
                                  L.ptr(x), L.ptr(y), 0, st),
      "spmv_fp32": lambda: L.call("ys_spmv3", None, L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), nv,
                                  L.ptr(x), L.ptr(y), 0, st),
      "spmv_fp32_x32": lambda: L.call("ys_spmv3_x32", L.ptr(bs.values32), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), nv,
                                      L.ptr(x32), L.ptr(y), 0, st),
      "spmv_fp32_tiled": lambda: tiled(0),
      "spmv_fp32_tiled_s2": lambda: tiled(2),
      "spmv_fp32_tiled_s3": lambda: tiled(3),
      "spmv_fp32_tiled_s4": lambda: tiled(4),
      "spmv_fp32_stream": lambda: streamed(0),
      "spmv_fp32_stream_s2": lambda: streamed(2),
      "spmv_fp32_stream_s3": lambda: streamed(3),
      "stream_fill": lambda: L.call("ys_spmv_stream_fill", L.ptr(bs.values32), L.ptr(sp.src), sp.slots,
                                    L.ptr(sp.blocks32), st),
      "mas_apply": lambda: L.call("ys_mas_apply", mas._mas, L.ptr(x), L.ptr(z), st),
      "gemv": lambda: L.call("ys_mas_gemv", mas._mas, st, None),
      "newton_step": lambda: mz.computeHessianAndGradient(tolerance=1e-6, maxIterations=2000),
      # 50 MAS-PCG iterations (unreachable tolerance) from one graph launch
      "pcg50_fp32": lambda: mas._run_pcg(H, H.gradient.value, z, True, L.YS_PREC_MAS, None, mas._mas, 1e-30, 50,
                                         True, "residual"),
      # the same loop over the tiled SpMV (no streamed-tile plan)
      "pcg50_fp32_tiled": lambda: pcg_without_stream(),
      "pcg50_fp64": lambda: mas._run_pcg(H, H.gradient.value, z, False, L.YS_PREC_MAS, None, mas._mas, 1e-30, 50,
                                         True, "residual"),
  }
  nbytes = ctypes.c_uint64(0)
  L.call("ys_mas_gemv", mas._mas, st, ctypes.byref(nbytes))
  if args.trace_pcg:
    return trace_pcg(cases["pcg50_fp32"])
  out = {"side": args.side, "tets": cube.tet_count, "dof": cube.dofs, "blocks": p.num_unique,
         "plan_entries": int(row_ptr[nv].item()), "tile_cap": tile_cap, "entry_cap": entry_cap,
         "gemv_alg_bytes": int(nbytes.value), "gemv_layout_bytes": gemv_layout_bytes(mas._tables),
         "non_psd": int(snh._const_cache[("work", snh.n)][1].item()), "pcg": mz.linearSolver.statistics}
  for name, fn in cases.items():
    if args.kernel == "all" or name in args.kernel.split(","):
      out[name + "_ms"] = _time(fn, args.reps if name != "newton_step" else max(2, args.reps // 5))
  print(json.dumps(out))


if __name__ == "__main__":
  main()
