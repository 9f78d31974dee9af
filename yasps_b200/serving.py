"""Serving form: continuous batching of Newton-step solves on one GPU.

A request is one Newton step of a resident scene (gradient and SPD-projected
Hessian, then ``H x = g`` to a true relative residual, the step
``scene.minimizeEnergy`` takes; ``PKG/scene/scene.pyx:155-200``).  Its
topology key selects a resident topology: the scene, the BSR pattern, the
SpMV plan and the MAS hierarchy are built once per topology and stay on the
device.  Two kinds of topology exist: a Stable Neo-Hookean FEM cube keyed by
its side (its requests bring their material and positions), and any scene
with one static 3x3 block set and a MAS hierarchy (the mixed cloth + affine
body + contact scenes among them), whose requests bring the values of named
input attributes.  The server

* admits queued requests as slots and HBM free up (a byte budget over every
  resident per-request buffer);
* runs each admitted request's element evaluation, assembly and MAS numeric
  update on an admission stream, overlapping the solves in flight;
* attaches a request to the batched PCG (``ys_serve_*``) once that admission
  work has finished, so solves of different sizes advance together (one PCG
  iteration of every live solve per pass, ``passes`` passes per launch of the
  CUDA graph of the current size bucket);
* retires converged solves after every launch and copies their solutions to
  host memory.

The solve of a request is bit-identical whatever else shares the GPU with
it.  The reference has no serving form; ``solve_serial_fp64`` is its plain
path (FP64 MAS PCG, one request at a time) on the same topologies.
"""

from __future__ import annotations

import collections
import ctypes
import math
import time
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

from . import _lib as L
from . import scenes
from .hessian import _torch
from .solver import create_mas_handle, mas_numeric_buffers


@dataclass
class NewtonRequest:
  """One Newton-step solve: inputs in pinned host memory, results filled in.

  A FEM-cube request carries ``side``, its Lame parameters and positions; a
  scene request carries ``key`` (its topology) and ``inputs`` (attribute
  name -> pinned float64 tensor)."""

  side: int
  mu: float
  lam: float
  free_position: object      # pinned float64 tensor [3 * free vertices]
  pinned_position: object    # pinned float64 tensor [3 * pinned vertices]
  arrival: float = 0.0       # seconds after the start of the stream
  tag: object = None
  key: object = None         # topology key (the cube side when None)
  inputs: Optional[dict] = None
  solution: Optional[np.ndarray] = None
  phase: int = L.YS_SERVE_EMPTY
  iterations: int = 0
  refinements: int = 0
  relative_residual: float = math.nan
  t_admit: float = math.nan
  t_done: float = math.nan

  @property
  def latency(self) -> float:
    return self.t_done - self.arrival

  @property
  def topology_key(self):
    return self.side if self.key is None else self.key

  @property
  def converged(self) -> bool:
    return self.phase == L.YS_SERVE_DONE


def fem_request(side: int, young: float, poisson: float, noise: float, seed: int, arrival: float = 0.0,
                tag=None, spacing: float = 0.1) -> NewtonRequest:
  """A request for ``scenes.fem_cube(side, spacing, young, poisson, noise, seed)``."""
  torch = _torch()
  pinned, free = scenes.fem_positions(side, spacing=spacing, noise=noise, seed=seed)
  mu, lam = scenes.lame(young, poisson)
  pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).reshape(-1)).pin_memory()
  return NewtonRequest(side, mu, lam, pin(free), pin(pinned), arrival, tag)


def scene_request(key, inputs: dict, arrival: float = 0.0, tag=None) -> NewtonRequest:
  """A request for the resident scene topology ``key``: ``inputs`` maps
  input-attribute names to arrays, copied here into pinned host memory."""
  torch = _torch()
  pinned = {}
  for name, v in inputs.items():
    t = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64).reshape(-1))
    pinned[name] = t.pin_memory() if torch.cuda.is_available() else t
  return NewtonRequest(0, math.nan, math.nan, None, None, arrival, tag, key=key, inputs=pinned)


class SceneTopology:
  """Resident structure of one scene: its Hessian pattern (one static 3x3
  block set), SpMV plan and MAS hierarchy, reused by every request of this
  topology.  ``inputs`` names the attributes a request sets (name ->
  attribute); the scene's other values stay as built."""

  def __init__(self, key, scene, inputs: Optional[dict] = None, solver_options: Optional[dict] = None):
    self.key = key
    self.scene = scene
    self.input_attributes = dict(inputs or {})
    self._setup(solver_options)

  def _setup(self, solver_options: Optional[dict]) -> None:
    opts = dict(solver_options or {})
    opts["mixed_spmv"] = True
    self.scene.minimizer.setSolver("mas", **opts)
    self.mas_solver = self.scene.minimizer.linearSolver.implementation
    H = self.scene.minimizer.computeNumericValue()
    H.want_diagonal = False  # the MAS path reads no diagonal blocks
    self.mas_solver._ensure_hierarchy(H)
    self.H = H
    self.tables = self.mas_solver._tables
    self.weights = self.mas_solver.weights_for(len(self.tables.level_node_offset) - 1)
    dev, _ = self.mas_solver._dev_tables
    self.dev_tables = {k: v for k, v in dev.items() if k not in mas_numeric_keys()}
    if len(H.block_sets) != 1:
      raise ValueError("SceneTopology: the serving form takes scenes with one static block set")
    bs = H.block_sets[0]
    self.plan = H.spmv_plan(bs)
    self.nvalues = int(bs.values.numel())
    self.nvalues32 = int(bs.values32.numel())
    self.n = int(H.rows)
    self.nv = self.n // 3

  def load_inputs(self, req: NewtonRequest) -> None:
    """Input attributes of ``req`` into the template (current stream)."""
    missing = set(self.input_attributes) - set(req.inputs or {})
    if missing or set(req.inputs or {}) - set(self.input_attributes):
      raise ValueError(f"SceneTopology {self.key!r}: request inputs {sorted(req.inputs or {})} "
                       f"differ from {sorted(self.input_attributes)}")
    for name, value in req.inputs.items():
      self.input_attributes[name].copyValueFrom(value)


class FemTopology(SceneTopology):
  """Resident structure of one cube side: a template scene whose Hessian
  pattern, SpMV plan and MAS hierarchy every request of this side reuses."""

  def __init__(self, side: int, spacing: float = 0.1, solver_options: Optional[dict] = None):
    self.side = int(side)
    self.key = self.side
    cube = scenes.fem_cube(self.side, spacing=spacing, noise=0.0)
    self.scene, self.handles = scenes.fem_scene(cube)
    self.input_attributes = {}
    self._setup(solver_options)
    self.mu_att = self.scene["mu"]
    self.lam_att = self.scene["lam"]

  def load_inputs(self, req: NewtonRequest) -> None:
    """Material and positions of ``req`` into the template (current stream)."""
    self.mu_att.setScalar(req.mu)
    self.lam_att.setScalar(req.lam)
    h = self.handles
    h["free_position"].copyValueFrom(req.free_position)
    h["last_position"].copyValueFrom(req.free_position)
    h["pinned_position"].copyValueFrom(req.pinned_position)


def mas_numeric_keys():
  return ("coarse_values", "inverse", "rl", "zl", "rl64", "status")


class _Slot:
  """Per-request device buffers of one topology (pooled and reused)."""

  def __init__(self, topo: FemTopology):
    torch = _torch()
    dev = torch.device("cuda")
    self.topo = topo
    self.values = torch.zeros(topo.nvalues, dtype=torch.float64, device=dev)
    self.values32 = torch.zeros(topo.nvalues32, dtype=torch.float32, device=dev)
    self.g = torch.zeros(topo.n, dtype=torch.float64, device=dev)
    self.x = torch.zeros(topo.n, dtype=torch.float64, device=dev)
    self.work = torch.zeros(int(L.load().ys_serve_workspace_doubles(topo.nv)), dtype=torch.float64, device=dev)
    self.numeric = mas_numeric_buffers(topo.tables)
    tables = dict(topo.dev_tables)
    tables.update(self.numeric)
    self.mas, self._keep = create_mas_handle(topo.tables, topo.nv, topo.weights, tables)
    self.ready = torch.cuda.Event()
    owned = [self.values, self.values32, self.g, self.x, self.work, *self.numeric.values()]
    self.nbytes = int(sum(t.numel() * t.element_size() for t in owned))

  def release(self) -> None:
    if self.mas is not None:
      L.call("ys_mas_destroy", self.mas)
      self.mas = None

  def admit(self, req: NewtonRequest) -> None:
    """Element evaluation, assembly and MAS numeric update of ``req`` on the
    current stream; ``ready`` is recorded behind them."""
    topo = self.topo
    topo.load_inputs(req)
    H = topo.scene.minimizer.computeNumericValue()
    bs = H.block_sets[0]
    self.values.copy_(bs.values, non_blocking=True)
    self.values32.copy_(bs.values32, non_blocking=True)
    self.g.copy_(H.gradient.value, non_blocking=True)
    L.call("ys_mas_numeric_update", self.mas, L.ptr(self.values), L.stream_ptr(), None)
    self.ready.record()

  def desc(self, tolerance: float, refinement_tolerance: float, max_iterations: int) -> L.ServeSlotDesc:
    row_ptr, eb, ec = self.topo.plan
    m = L.Matrix3()
    m.num_sets = 1
    m.values[0], m.values32[0] = L.ptr(self.values), L.ptr(self.values32)
    m.row_ptr[0], m.entry_block[0], m.entry_col[0] = L.ptr(row_ptr), L.ptr(eb), L.ptr(ec)
    m.num_vars = self.topo.nv
    d = L.ServeSlotDesc()
    d.mas = self.mas
    d.matrix = m
    d.rhs, d.solution, d.workspace = L.ptr(self.g), L.ptr(self.x), L.ptr(self.work)
    d.tolerance = float(tolerance)
    d.refinement_tolerance = float(refinement_tolerance)
    d.max_iterations = int(max_iterations)
    return d


class NewtonServer:
  """Continuous-batching Newton-step server over ``ys_serve_*`` (one GPU).

  ``max_slots`` solves are in flight at most; ``memory_budget`` bounds the
  bytes of the pooled per-request buffers (admission by HBM footprint);
  ``passes`` PCG passes run per launch between two host checks;
  ``admission_streams`` streams carry the admission work of different
  topologies.  FEM-cube topologies are built on first use; scene topologies
  are added with ``add_topology``.
  """

  def __init__(self, max_slots: int = 64, passes: int = 8, memory_budget: float = 40e9, tolerance: float = 1e-6,
               refinement_tolerance: float = 1e-3, max_iterations: int = 2000, spacing: float = 0.1,
               solver_options: Optional[dict] = None, admission_streams: int = 4):
    torch = _torch()
    self.max_slots = int(max_slots)
    self.passes = int(passes)
    self.memory_budget = float(memory_budget)
    self.tolerance = float(tolerance)
    self.refinement_tolerance = float(refinement_tolerance)
    self.max_iterations = int(max_iterations)
    self.spacing = float(spacing)
    self.solver_options = dict(solver_options or {})
    h = ctypes.c_void_p()
    L.call("ys_serve_create", self.max_slots, self.passes, ctypes.byref(h))
    self.handle = h
    self._status = (L.ServeSlotStatus * self.max_slots)()
    # admission work of different topologies overlaps on several streams; one
    # topology always uses the same stream (its requests share the template
    # buffers)
    self.admit_streams = [torch.cuda.Stream() for _ in range(int(admission_streams))]
    self._stream_of = {}                          # topology key -> admission stream
    self.solve_stream = torch.cuda.Stream()
    self.topologies: Dict[object, SceneTopology] = {}
    self._idle = collections.defaultdict(list)   # topology key -> idle slots
    self.resident_bytes = 0
    self._free_ids = list(range(self.max_slots - 1, -1, -1))
    self._pending = collections.deque()           # (req, slot, id) admitted, admission work in flight
    self._active = {}                             # id -> (req, slot)
    self.launches = 0
    self.passes_run = 0
    self.slots_created = 0
    self.host_seconds = collections.Counter()    # admit / attach / launch / wait (host time per phase)
    self.gpu_ms = collections.Counter()          # device time of the PCG launches (CUDA events)
    self._launch_events = []

  # -- resources ------------------------------------------------------------------
  def topology(self, key) -> SceneTopology:
    """The topology of ``key``; an integer key not yet resident builds the
    FEM cube of that side."""
    topo = self.topologies.get(key)
    if topo is None:
      if not isinstance(key, (int, np.integer)):
        raise KeyError(f"NewtonServer: no topology {key!r} (add scene topologies with add_topology)")
      topo = FemTopology(int(key), self.spacing, self.solver_options)
      self.topologies[topo.key] = topo
    return topo

  def add_topology(self, topo: SceneTopology) -> SceneTopology:
    """Make a prebuilt scene topology resident under ``topo.key``."""
    if topo.key in self.topologies:
      raise ValueError(f"NewtonServer.add_topology: topology {topo.key!r} exists")
    self.topologies[topo.key] = topo
    return topo

  def register(self, keys, slots_per_side: int = 1) -> None:
    """Build (FEM sides) or look up the topologies of ``keys`` and pool
    ``slots_per_side`` slots each."""
    for key in keys:
      topo = self.topology(key)
      while len(self._idle[topo.key]) < slots_per_side:
        slot = self._new_slot(topo)
        if slot is None:
          break
        self._idle[topo.key].append(slot)
    _torch().cuda.synchronize()

  def reserve(self, requests) -> None:
    """Pool enough slots for ``requests`` (their count per topology, at most
    ``max_slots`` each) within the memory budget, so serving that stream
    creates no slot (a device allocation synchronises the device)."""
    need = collections.Counter(r.topology_key for r in requests)
    for key, count in need.items():
      topo = self.topology(key)
      while len(self._idle[key]) < min(count, self.max_slots):
        slot = self._new_slot(topo, evict=False)
        if slot is None:
          break
        self._idle[key].append(slot)
    _torch().cuda.synchronize()

  def _new_slot(self, topo: SceneTopology, evict: bool = True) -> Optional[_Slot]:
    need = getattr(topo, "slot_bytes", None)
    if need is not None and self.resident_bytes + need > self.memory_budget:
      if evict:
        self._evict_idle(need)
      if self.resident_bytes + need > self.memory_budget:
        return None
    self.slots_created += 1
    slot = _Slot(topo)
    topo.slot_bytes = slot.nbytes
    if self.resident_bytes + slot.nbytes > self.memory_budget:
      if evict:
        self._evict_idle(slot.nbytes)
      if self.resident_bytes + slot.nbytes > self.memory_budget:
        slot.release()
        return None
    self.resident_bytes += slot.nbytes
    return slot

  def _evict_idle(self, need: int) -> None:
    """Release idle pooled slots (of any topology) until ``need`` more bytes fit."""
    for key in list(self._idle):
      while self._idle[key] and self.resident_bytes + need > self.memory_budget:
        old = self._idle[key].pop()
        self.resident_bytes -= old.nbytes
        old.release()

  def _take_slot(self, key) -> Optional[_Slot]:
    if self._idle[key]:
      return self._idle[key].pop()
    return self._new_slot(self.topology(key))

  def _admit_stream(self, key):
    stream = self._stream_of.get(key)
    if stream is None:
      stream = self.admit_streams[len(self._stream_of) % len(self.admit_streams)]
      self._stream_of[key] = stream
    return stream

  def close(self) -> None:
    if self.handle is not None:
      _torch().cuda.synchronize()
      L.call("ys_serve_destroy", self.handle)
      self.handle = None
    for slots in self._idle.values():
      for s in slots:
        s.release()
    self._idle.clear()

  def __del__(self):
    try:
      self.close()
    except Exception:
      pass

  # -- request loop ---------------------------------------------------------------
  def _admit_arrivals(self, queue, now):
    torch = _torch()
    while queue and self._free_ids:
      slot = self._take_slot(queue[0].topology_key)
      if slot is None:
        break
      req = queue.popleft()
      t = time.perf_counter()
      with torch.cuda.stream(self._admit_stream(req.topology_key)):
        slot.admit(req)
      self.host_seconds["admit"] += time.perf_counter() - t
      req.t_admit = now
      self._pending.append((req, slot, self._free_ids.pop()))

  def _attach_ready(self) -> None:
    keep = collections.deque()
    while self._pending:
      req, slot, sid = self._pending.popleft()
      if slot.ready.query():
        d = slot.desc(self.tolerance, self.refinement_tolerance, self.max_iterations)
        L.call("ys_serve_attach", self.handle, sid, ctypes.byref(d))
        self._active[sid] = (req, slot)
      else:
        keep.append((req, slot, sid))
    self._pending = keep

  def _retire(self, clock, t0) -> List[NewtonRequest]:
    torch = _torch()
    t = time.perf_counter()
    L.call("ys_serve_status", self.handle, self.solve_stream.cuda_stream, self._status)
    self.host_seconds["wait"] += time.perf_counter() - t
    for e0, e1 in self._launch_events:
      self.gpu_ms["launch"] += e0.elapsed_time(e1)
    self._launch_events.clear()
    done = [sid for sid in self._active
            if self._status[sid].phase in (L.YS_SERVE_DONE, L.YS_SERVE_FAILED)]
    if not done:
      return []
    # the status read synchronised the solve stream: plain copies of the
    # solutions (no pinned buffers, whose allocation would synchronise the
    # device while other solves are in flight)
    sols = {}
    with torch.cuda.stream(self.solve_stream):
      for sid in done:
        sols[sid] = self._active[sid][1].x.cpu().numpy()
    t = clock() - t0
    out = []
    for sid in done:
      req, slot = self._active.pop(sid)
      st = self._status[sid]
      req.phase, req.iterations, req.refinements = int(st.phase), int(st.iterations), int(st.refinements)
      req.relative_residual = float(st.relative_residual)
      req.solution = sols[sid]
      req.t_done = t
      L.call("ys_serve_detach", self.handle, sid)
      self._free_ids.append(sid)
      self._idle[slot.topo.key].append(slot)
      out.append(req)
    return out

  def run(self, requests, clock=time.perf_counter) -> List[NewtonRequest]:
    """Serve ``requests`` as they arrive (``arrival`` seconds after the call);
    returns them in completion order with results and times filled in."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    total, i = len(reqs), 0
    queue = collections.deque()
    finished: List[NewtonRequest] = []
    t0 = clock()
    while len(finished) < total:
      now = clock() - t0
      while i < total and reqs[i].arrival <= now:
        queue.append(reqs[i])
        i += 1
      self._attach_ready()
      if self._active:
        t = time.perf_counter()
        e0, e1 = _torch().cuda.Event(enable_timing=True), _torch().cuda.Event(enable_timing=True)
        e0.record(self.solve_stream)
        L.call("ys_serve_launch", self.handle, self.solve_stream.cuda_stream)
        e1.record(self.solve_stream)
        self._launch_events.append((e0, e1))
        self.host_seconds["launch"] += time.perf_counter() - t
        self.launches += 1
        self.passes_run += self.passes
        # admission work of new arrivals overlaps the launch in flight
        now = clock() - t0
        while i < total and reqs[i].arrival <= now:
          queue.append(reqs[i])
          i += 1
        self._admit_arrivals(queue, now)
        finished += self._retire(clock, t0)
        continue
      self._admit_arrivals(queue, now)
      if self._pending:
        t = time.perf_counter()
        self._pending[0][1].ready.synchronize()
        self.host_seconds["wait_admission"] += time.perf_counter() - t
      elif queue:
        raise RuntimeError(f"a request of topology {queue[0].topology_key!r} does not fit the memory budget")
      elif i < total:
        wait = reqs[i].arrival - (clock() - t0)
        if wait > 0:
          time.sleep(min(wait, 2e-4))
    return finished

  def solve_serial_fp64(self, requests, clock=time.perf_counter) -> List[NewtonRequest]:
    """The plain drop-in path on the same topologies: one request at a time in
    arrival order (each waits for the one before), FP64 blocks, MAS PCG to the
    same true relative residual, solution copied to the host."""
    torch = _torch()
    reqs = sorted(requests, key=lambda r: r.arrival)
    t0 = clock()
    for req in reqs:
      while clock() - t0 < req.arrival:
        pass
      topo = self.topology(req.topology_key)
      solver = topo.mas_solver
      req.t_admit = clock() - t0
      saved = solver.mixed_spmv, solver.stop_rule
      solver.mixed_spmv, solver.stop_rule = False, "residual"
      try:
        topo.load_inputs(req)
        H = topo.scene.minimizer.computeNumericValue()
        code = solver.computeSolution(H, H.gradient, None, tolerance=self.tolerance,
                                      maxIterations=self.max_iterations, zero_initial_guess=True)
        req.solution = solver.solution.cpu().numpy()
      finally:
        solver.mixed_spmv, solver.stop_rule = saved
      req.t_done = clock() - t0
      req.phase = L.YS_SERVE_DONE if code == 0 else L.YS_SERVE_FAILED
      req.iterations = int(solver.statistics.get("iterations", 0))
    torch.cuda.synchronize()
    return reqs


def stream_stats(reqs: List[NewtonRequest]) -> dict:
  """Throughput and latency percentiles of a served stream."""
  lat = np.array([r.latency for r in reqs]) * 1e3
  span = max(r.t_done for r in reqs) - min(r.arrival for r in reqs)
  return {"requests": len(reqs), "solves_per_s": len(reqs) / span, "makespan_s": span,
          "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
          "converged": int(sum(r.converged for r in reqs)),
          "mean_iterations": float(np.mean([r.iterations for r in reqs]))}


def poisson_fem_stream(count: int = 512, mean_spacing: float = 2e-3, side_range=(8, 48), young_range=(1e4, 1e6),
                       poisson_range=(0.3, 0.45), noise: float = 0.01, seed: int = 0,
                       spacing: float = 0.1) -> List[NewtonRequest]:
  """Seeded FEM Newton-step stream: Poisson arrivals (exponential gaps of mean
  ``mean_spacing`` s), cube side uniform in ``side_range``, Young's modulus
  log-uniform, Poisson ratio uniform, positions rest + U(-noise, noise).
  Inputs live in one pinned host buffer."""
  torch = _torch()
  rng = np.random.default_rng(seed)
  gaps = rng.exponential(mean_spacing, count)
  arrivals = np.cumsum(gaps) - gaps[0]
  sides = rng.integers(side_range[0], side_range[1] + 1, count)
  young = np.exp(rng.uniform(np.log(young_range[0]), np.log(young_range[1]), count))
  nu = rng.uniform(poisson_range[0], poisson_range[1], count)
  sizes = [3 * int(s) ** 3 for s in sides]
  buf = torch.empty(int(sum(sizes)), dtype=torch.float64)
  if torch.cuda.is_available():
    buf = buf.pin_memory()
  reqs, off = [], 0
  for k in range(count):
    side = int(sides[k])
    pinned, free = scenes.fem_positions(side, spacing=spacing, noise=noise, seed=seed * 1000003 + k)
    a, b = off + free.size, off + free.size + pinned.size
    buf[off:a].copy_(torch.from_numpy(free.reshape(-1)))
    buf[a:b].copy_(torch.from_numpy(pinned.reshape(-1)))
    mu, lam = scenes.lame(float(young[k]), float(nu[k]))
    reqs.append(NewtonRequest(side, mu, lam, buf[off:a], buf[a:b], float(arrivals[k]), k))
    off = b
  return reqs


# ---- mixed serving: cloth + affine-body + contact scenes beside large FEM cubes -------

@dataclass
class ClothSceneSpec:
  """One scene of the cloth-over-obstacle type with affine bodies
  (``scenes.cloth_contact``): its topology key and generator arguments."""

  key: object
  side: int
  bodies: int
  pairs: int
  seed: int


def cloth_scene_topology(spec: ClothSceneSpec, solver_options: Optional[dict] = None) -> SceneTopology:
  """Build the scene of ``spec`` and make it a serving topology whose
  requests set the cloth positions, the positions of the last step and the
  bodies' affine matrices and translations."""
  cc = scenes.cloth_contact(spec.side, spec.pairs, num_bodies=spec.bodies, seed=spec.seed)
  sc, handles = scenes.cloth_contact_scene(cc)
  names = [k for k in ("position", "old_position", "affine_matrices", "translations") if k in handles]
  topo = SceneTopology(spec.key, sc, {k: handles[k] for k in names}, solver_options)
  topo.cloth = cc
  topo.spec = spec
  return topo


def cloth_scene_request(topo: SceneTopology, arrival: float = 0.0, tag=None) -> NewtonRequest:
  """The Newton step of a cloth-scene topology at its generated state."""
  cc = topo.cloth
  inputs = {"position": cc.cloth_position, "old_position": cc.cloth_position}
  if cc.bodies is not None:
    inputs.update(affine_matrices=cc.bodies.affine, translations=cc.bodies.translation)
  return scene_request(topo.key, inputs, arrival, tag)


@dataclass
class MixedWorkload:
  """A mixed stream: cloth scenes (one request each) interleaved with FEM
  cube requests of one side; ``order[k]`` names the k-th arrival as
  ``("cloth", i)`` or ``("fem", j)``."""

  scenes: List[ClothSceneSpec]
  fem_side: int
  fem: List[dict]
  order: List[tuple]
  arrivals: np.ndarray

  def requests(self, server: "NewtonServer", all_at_once: bool = False) -> List[NewtonRequest]:
    """Requests in arrival order (the topologies must be resident); with
    ``all_at_once`` every request arrives at time 0."""
    out = []
    for k, (kind, i) in enumerate(self.order):
      at = 0.0 if all_at_once else float(self.arrivals[k])
      if kind == "cloth":
        out.append(cloth_scene_request(server.topology(self.scenes[i].key), at, tag=k))
      else:
        f = self.fem[i]
        out.append(fem_request(self.fem_side, f["young"], f["poisson"], f["noise"], f["seed"], arrival=at, tag=k))
    return out


def mixed_workload(num_scenes: int = 64, num_fem: int = 8, fem_side: int = 126, side_range=(64, 256),
                   body_range=(2, 16), pair_range=(10_000, 200_000), fem_young: float = 1e6,
                   fem_poisson: float = 0.45, fem_noise: float = 0.005, mean_spacing: float = 2e-3,
                   seed: int = 0) -> MixedWorkload:
  """Seeded mixed stream: ``num_scenes`` cloth scenes with cloth side, body
  count and contact pair count drawn uniform in their ranges, and
  ``num_fem`` FEM cubes of ``fem_side``^3 vertices, in a random interleaving
  with Poisson arrivals of mean gap ``mean_spacing`` s."""
  rng = np.random.default_rng(seed)
  specs = [ClothSceneSpec(("cloth", k), int(rng.integers(side_range[0], side_range[1] + 1)),
                          int(rng.integers(body_range[0], body_range[1] + 1)),
                          int(rng.integers(pair_range[0], pair_range[1] + 1)), seed * 1000003 + k)
           for k in range(num_scenes)]
  fem = [dict(young=fem_young, poisson=fem_poisson, noise=fem_noise, seed=seed * 1000003 + 500 + j)
         for j in range(num_fem)]
  order = [("cloth", k) for k in range(num_scenes)] + [("fem", j) for j in range(num_fem)]
  order = [order[i] for i in rng.permutation(len(order))]
  gaps = rng.exponential(mean_spacing, len(order)) if mean_spacing > 0 else np.zeros(len(order))
  return MixedWorkload(specs, int(fem_side), fem, order, np.cumsum(gaps) - gaps[0])
