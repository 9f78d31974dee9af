"""Linear solvers: block-Jacobi PCG and MAS-preconditioned CG.

Mirrors the reference solver surface (``PKG/solver/solver.py:9-68``,
``PKG/solver/jacobianPCGSolver.pyx:14-166``, ``PKG/solver/masSolver.py:13-126``):
``computeSolution(active_hessian, right_hand_side, initial_guess, tolerance,
maxIterations, zero_initial_guess) -> int``, ``reset()``, ``solution`` and
``statistics``.  The tolerance keeps the reference meaning (a squared,
preconditioned ratio ``r^T M^-1 r <= tol * r0^T M^-1 r0``) unless
``stop_rule="residual"`` is given, in which case it is the true relative
residual ``||g - H x|| / ||g||``.

``masSolver(mixed_spmv=True)`` is the precision form: FP32 Hessian blocks in
the PCG SpMV (FP32 products and row sums), FP32 MAS application, FP64 PCG
vectors and reductions, and FP64 iterative refinement ``r = g - H x`` with
the FP64 blocks until the FP64 residual meets the tolerance (the
reference's ``mixed_spmv`` FP64 audit + corrective solve,
``mas/solver.py:643-688``, iterated).
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib as L
from .hessian import vector, _dev, _torch
from . import mas_hierarchy

_STOP = {"preconditioned": L.YS_STOP_PRECONDITIONED, "residual": L.YS_STOP_RESIDUAL}


class _PcgCache:
  def __init__(self):
    self.key = None
    self.handle = None
    self.keepalive = None

  def get(self, key, build):
    if key != self.key:
      self.release()
      self.handle, self.keepalive = build()
      self.key = key
    return self.handle

  def release(self):
    if self.handle is not None:
      L.call("ys_pcg_destroy", self.handle)
    self.handle, self.key, self.keepalive = None, None, None


def _as_tensor(v):
  if v is None:
    return None
  return v.value if hasattr(v, "value") else v


class _PcgBase:
  def __init__(self, stop_rule="preconditioned"):
    if stop_rule not in _STOP:
      raise ValueError("stop_rule must be 'preconditioned' or 'residual'")
    self.stop_rule = stop_rule
    self._solution = None
    self._work = None
    self._cache = _PcgCache()
    self._statistics = {}
    self.last_result = None

  @property
  def solution(self):
    return self._solution

  @property
  def statistics(self) -> dict:
    return dict(self._statistics)

  def reset(self):
    self._cache.release()
    self._solution = None
    self._work = None
    self._statistics = {}

  def _buffers(self, n):
    torch = _torch()
    if self._solution is None or self._solution.numel() != n:
      self._solution = torch.zeros(n, dtype=torch.float64, device=_dev())
      self._work = torch.zeros(int(L.load().ys_pcg_workspace_doubles(n)), dtype=torch.float64, device=_dev())
      self._cache.release()

  def _run_pcg(self, H, rhs, x, fp32, prec_kind, jinv, mas_handle, tol, maxit, zero_guess, stop_rule, jgroup=None):
    """One device PCG solve into ``x``; returns the ys_pcg_result."""
    # the graph holds every device pointer of the matrix: a rebuilt pattern
    # (dynamic terms) gives new row plans and must give a new graph
    # (an FP32 solve first refreshes the streamed SpMV's packed blocks from
    # the current FP32 values; the graph holds the plan's pointers)
    streams = [H.stream_plan(bs) if fp32 and len(H.block_sets) == 1 else None for bs in H.block_sets]
    plans = tuple(tuple(t.data_ptr() for t in H.spmv_plan(bs)) + (bs.pattern.num_unique,) +
                  tuple(0 if t is None else (t.data_ptr() if hasattr(t, "data_ptr") else t) for t in H.tile_plan(bs)) +
                  (sp.pointers() if sp is not None else ())
                  for bs, sp in zip(H.block_sets, streams))
    key = (id(H), H.rows, rhs.data_ptr(), x.data_ptr(), fp32, prec_kind, None if jinv is None else jinv.data_ptr(),
           mas_handle, bool(zero_guess), stop_rule, None if jgroup is None else jgroup.data_ptr(),
           tuple(bs.values.data_ptr() for bs in H.block_sets),
           tuple(0 if bs.values32 is None else bs.values32.data_ptr() for bs in H.block_sets), plans)

    def build():
      args = L.PcgArgs()
      args.matrix = H.matrix3()
      args.precision = 1 if fp32 else 0
      args.preconditioner = prec_kind
      args.jacobi_inverse = L.ptr(jinv)
      args.mas = mas_handle
      args.stop_rule = _STOP[stop_rule]
      args.tolerance = tol
      args.max_iterations = maxit
      args.rhs = L.ptr(rhs)
      args.solution = L.ptr(x)
      args.zero_initial_guess = 1 if zero_guess else 0
      args.workspace = L.ptr(self._work)
      args.jacobi_group = L.ptr(jgroup)
      h = ctypes.c_void_p()
      L.call("ys_pcg_create", ctypes.byref(args), ctypes.byref(h))
      return h, args

    handle = self._cache.get(key, build)
    L.call("ys_pcg_set_params", handle, float(tol), int(maxit))
    res = L.PcgResult()
    L.call("ys_pcg_run", handle, L.stream_ptr(), ctypes.byref(res))
    self.last_result = res
    return res


def upload_mas_tables(t):
  """Device copies of the structural MAS tables (shared by every numeric state)."""
  torch = _torch()
  up = lambda a, dt=torch.int32: torch.from_numpy(np.ascontiguousarray(a).view(
      np.int32 if dt == torch.int32 else np.int64)).to(_dev())
  return dict(cmap=up(t.cmap), child_ptr=up(t.child_ptr), child_fine=up(t.child_fine),
              dom_node_ptr=up(t.dom_node_ptr), dom_nodes=up(t.dom_nodes),
              inv_offset=up(t.inv_offset, torch.int64), dom_entry_ptr=up(t.dom_entry_ptr),
              dom_entry=up(t.dom_entry), cb_src_ptr=up(t.cb_src_ptr), cb_src=up(t.cb_src))


def mas_numeric_buffers(t):
  """Per-solve numeric MAS state: Galerkin blocks, FP32 inverses, level vectors."""
  torch = _torch()
  nb_coarse = int(t.cb_level_begin[-1])
  packed = int(t.level_node_offset[-1])
  return dict(coarse_values=torch.zeros(max(9 * nb_coarse, 1), dtype=torch.float64, device=_dev()),
              inverse=torch.zeros(max(t.inverse_floats, 1), dtype=torch.float32, device=_dev()),
              rl=torch.zeros(3 * packed, dtype=torch.float32, device=_dev()),
              zl=torch.zeros(3 * packed, dtype=torch.float32, device=_dev()),
              rl64=torch.zeros(3 * packed, dtype=torch.float64, device=_dev()),
              status=torch.zeros(1, dtype=torch.int32, device=_dev()))


def create_mas_handle(t, nv, weights, dev):
  """``ys_mas_create`` over tables ``t`` (host) / ``dev`` (device tables and
  numeric buffers); returns the handle and the host arrays it borrowed."""
  nl = len(t.level_node_offset) - 1
  lno = (L.u32 * (nl + 1))(*t.level_node_offset.tolist())
  lw = (L.f64 * nl)(*weights)
  cbl = (L.u32 * (nl + 1))(*t.cb_level_begin.tolist())
  d = L.MasDesc()
  d.num_fine_vars, d.num_levels = nv, nl
  d.level_node_offset, d.level_weights = lno, lw
  d.cmap, d.child_ptr, d.child_fine = L.ptr(dev["cmap"]), L.ptr(dev["child_ptr"]), L.ptr(dev["child_fine"])
  d.num_domains = len(t.dom_node_ptr) - 1
  d.dom_node_ptr, d.dom_nodes, d.inv_offset = L.ptr(dev["dom_node_ptr"]), L.ptr(dev["dom_nodes"]), L.ptr(
      dev["inv_offset"])
  d.dom_entry_ptr, d.dom_entry = L.ptr(dev["dom_entry_ptr"]), L.ptr(dev["dom_entry"])
  d.fine_blocks, d.coarse_blocks = t.fine_blocks, int(t.cb_level_begin[-1])
  d.cb_src_ptr, d.cb_src, d.cb_level_begin = L.ptr(dev["cb_src_ptr"]), L.ptr(dev["cb_src"]), cbl
  d.max_domain_dofs = t.max_domain_dofs
  d.coarse_values, d.inverse = L.ptr(dev["coarse_values"]), L.ptr(dev["inverse"])
  d.level_residual, d.level_correction, d.status = L.ptr(dev["rl"]), L.ptr(dev["zl"]), L.ptr(dev["status"])
  d.level_residual64 = L.ptr(dev["rl64"])
  h = ctypes.c_void_p()
  L.call("ys_mas_create", ctypes.byref(d), ctypes.byref(h))
  return h, (lno, lw, cbl)


class jacobianPCGSolver(_PcgBase):
  """Block-Jacobi PCG (``PKG/solver/jacobianPCGSolver.pyx:84-166``)."""

  def __init__(self, stop_rule="preconditioned"):
    super().__init__(stop_rule)
    self._jinv = None

  def computeSolution(self, active_hessian, right_hand_side, initial_guess=None, tolerance=1e-3,
                      maxIterations=20000, zero_initial_guess=False):
    t0 = time.perf_counter()
    rhs = _as_tensor(right_hand_side)
    n = rhs.numel()
    if n == 0:
      self._statistics = {"solver": "jacobian", "converged": True, "iterations": 0}
      return 0
    self._buffers(n)
    if active_hessian is None:
      self._solution.zero_()
      return 0
    if n != active_hessian.rows:
      raise ValueError("jacobianPCGSolver.computeSolution: right_hand_side size must match the Hessian size.")
    torch = _torch()
    H = active_hessian
    if any(w.size not in (3, 9) for w in H.wrt):
      raise NotImplementedError("the device block-Jacobi PCG takes 3- and 9-DoF targets")
    if self._jinv is None or self._jinv.numel() != H.diagonal_blocks.numel():
      self._jinv = torch.zeros_like(H.diagonal_blocks)
    nat = len(H.wrt)
    arr = lambda v: (L.u32 * len(v))(*v)
    L.call("ys_invert_diagonal_blocks", L.ptr(H.diagonal_blocks), L.ptr(self._jinv), nat,
           arr(H.diagonal_blocks_start_cpu[:nat]), arr([w.correspondance.numInstances for w in H.wrt]),
           arr([w.size for w in H.wrt]), L.stream_ptr())
    jinv, jgroup = self._jinv, None
    if any(w.size == 9 for w in H.wrt):
      jinv, jgroup = self._group_strips(H)
    if not zero_initial_guess:
      self._solution.copy_(_as_tensor(initial_guess))
    res = self._run_pcg(H, rhs, self._solution, False, L.YS_PREC_BLOCK_JACOBI, jinv, None, tolerance,
                        maxIterations, zero_initial_guess, self.stop_rule, jgroup)
    self._statistics = {"solver": "jacobian", "converged": res.status >= 0, "iterations": int(res.iterations),
                        "result": int(res.status), "solve_seconds": time.perf_counter() - t0,
                        "matrix_size": int(H.rows), "tolerance": float(tolerance)}
    return int(res.status)


  def _group_strips(self, H):
    """Per 3-DoF variable, the 3 x 9 row strip of its attribute block's
    pseudo-inverse and its group word (first variable | size << 30): a
    3-DoF target is a group of one, a 9-DoF target (the affine matrix of a
    body, three internal 3-DoF rows) a group of three."""
    torch = _torch()
    nv = H.rows // 3
    key = (nv, tuple((w.size, w.correspondance.numInstances) for w in H.wrt))
    if getattr(self, "_strip_key", None) != key:
      self._strips = torch.zeros((nv, 3, 9), dtype=torch.float64, device=_dev())
      grp = np.zeros(nv, dtype=np.int64)
      for k, w in enumerate(H.wrt):
        v0, cnt = H.gradient_segments_start_cpu[k] // 3, w.correspondance.numInstances
        if w.size == 3:
          ids = v0 + np.arange(cnt)
          grp[ids] = ids | (1 << 30)
        else:
          first = v0 + 3 * np.arange(cnt)
          grp[v0:v0 + 3 * cnt] = np.repeat(first, 3) | (3 << 30)
      self._jgroup = torch.from_numpy(grp.astype(np.uint32).view(np.int32)).to(_dev())
      self._strip_key = key
    strips = self._strips
    for k, w in enumerate(H.wrt):
      v0, cnt = H.gradient_segments_start_cpu[k] // 3, w.correspondance.numInstances
      d0 = H.diagonal_blocks_start_cpu[k]
      if w.size == 3:
        strips[v0:v0 + cnt, :, :3] = self._jinv[d0:d0 + 9 * cnt].view(cnt, 3, 3)
      else:
        strips[v0:v0 + 3 * cnt] = self._jinv[d0:d0 + 81 * cnt].view(cnt, 3, 3, 9).reshape(3 * cnt, 3, 9)
    return strips.view(-1), self._jgroup


class masSolver(_PcgBase):
  """MAS-preconditioned CG (``PKG/solver/masSolver.py:13-126``, ``mas/solver.py``)."""

  def __init__(self, max_domain_dofs=96, max_levels=6, target_nodes_per_partition=32, coarsest_level_weight=2.5,
               fine_level_weight=1.5, level_weights=None, global_coarse_domain=True, mixed_spmv=False,
               stop_rule="preconditioned", refinement_tolerance=1e-3, max_refinements=8,
               adaptive_fine_level_weight=None, dense_collision_fine_level_weight=3.0,
               dense_collision_block_ratio=0.1, **unused):
    """Options follow ``MASSolver`` (``PKG/solver/mas/solver.py:89-120``).

    Level weights default to the reference's device runtime
    (``mas/cuda_runtime.py:1238-1243``): ``fine_level_weight`` on level 0, 1 on
    the intermediate levels and ``coarsest_level_weight`` on the coarsest
    (``fine_level_weight=1.0`` gives the CPU reference's weights,
    ``mas/preconditioner.py:32-36``).  ``level_weights`` overrides both.
    With a dynamic (contact) block set holding at least
    ``dense_collision_block_ratio`` blocks per fine variable, the fine-level
    weight is raised to ``dense_collision_fine_level_weight``
    (``adaptive_fine_level_weight``, on by default unless ``level_weights``
    is given; ``mas/solver.py:106-182``, ``mas/cuda_runtime.py:2716-2731``).
    """
    super().__init__(stop_rule)
    self.max_domain_dofs = int(max_domain_dofs)
    self.max_levels = int(max_levels)
    self.target_nodes = int(target_nodes_per_partition)
    self.coarsest_level_weight = float(coarsest_level_weight)
    self.fine_level_weight = float(fine_level_weight)
    self.level_weights = None if level_weights is None else tuple(float(w) for w in level_weights)
    self.global_coarse_domain = bool(global_coarse_domain)
    self.mixed_spmv = bool(mixed_spmv)
    self.adaptive_fine_level_weight = (level_weights is None if adaptive_fine_level_weight is None
                                       else bool(adaptive_fine_level_weight))
    if not (np.isfinite(dense_collision_fine_level_weight) and dense_collision_fine_level_weight > 0):
      raise ValueError("dense collision fine-level weight must be positive")
    if not (np.isfinite(dense_collision_block_ratio) and dense_collision_block_ratio > 0):
      raise ValueError("dense collision block ratio must be positive")
    self.dense_collision_fine_level_weight = float(dense_collision_fine_level_weight)
    self.dense_collision_block_ratio = float(dense_collision_block_ratio)
    self.active_fine_level_weight = None
    self.refinement_tolerance = float(refinement_tolerance)
    self.max_refinements = int(max_refinements)
    self.hierarchy = None
    self._mas = None
    self._mas_key = None
    self._tables = None
    self._dev_tables = None

  def weights_for(self, nl):
    """Level weights of an ``nl``-level hierarchy."""
    if self.level_weights is None:
      return ((self.coarsest_level_weight,) if nl == 1 else
              (self.fine_level_weight,) + (1.0,) * (nl - 2) + (self.coarsest_level_weight,))
    if len(self.level_weights) < nl:
      raise ValueError("level_weights needs one weight per level")
    return self.level_weights[:nl - 1] + self.level_weights[-1:] if len(self.level_weights) > nl else \
        self.level_weights

  def reset(self):
    super().reset()
    if self._mas is not None:
      L.call("ys_mas_destroy", self._mas)
    self._mas, self._mas_key, self.hierarchy, self._tables, self._dev_tables = None, None, None, None, None
    self._hierarchy_key, self._union = None, None

  def _ensure_hierarchy(self, H):
    """The hierarchy is built on the static block set's graph (the reference's
    default, ``include_dynamic_edges=False``, ``mas/hierarchy.py:158``); with a
    dynamic (contact) set, the fine level of the numeric update is the union
    of both sets, so its blocks enter the domain matrices of every level as
    the reference assembles them (``mas/numeric_assembly.py:64-83``); the
    tables follow the dynamic pattern."""
    torch = _torch()
    sets = H.block_sets
    if not sets or len(sets) > 2:
      raise NotImplementedError("the device MAS takes a static and at most one dynamic 3x3 block set")
    bs = sets[0]
    dyn = sets[1] if len(sets) == 2 else None
    key = (id(bs.pattern), None if dyn is None else id(dyn.pattern), H.rows)
    if key == self._mas_key:
      return
    if self._mas is not None:
      L.call("ys_mas_destroy", self._mas)
      self._mas = None
    if not all(s.pattern.all3 for s in sets):
      raise NotImplementedError("the device MAS supports 3x3 blocks (3-DoF variables)")
    pos = bs.pattern.positions[:2 * bs.pattern.num_unique].cpu().numpy().astype(np.int64).reshape(-1, 2)
    nv = H.rows // 3
    hkey = (id(bs.pattern), H.rows)
    if getattr(self, "_hierarchy_key", None) != hkey or self.hierarchy is None:
      edges = pos[pos[:, 0] != pos[:, 1]] // 3
      self.hierarchy = mas_hierarchy.build_hierarchy(np.full(nv, 3), edges, self.max_domain_dofs, self.max_levels,
                                                     self.target_nodes, self.global_coarse_domain)
      self._hierarchy_key = hkey
    self._union = None
    if dyn is not None:
      dpos = dyn.pattern.positions[:2 * dyn.pattern.num_unique].cpu().numpy().astype(np.int64).reshape(-1, 2)
      n = H.rows
      keys = np.concatenate([pos[:, 0] * n + pos[:, 1], dpos[:, 0] * n + dpos[:, 1]])
      uniq, inv = np.unique(keys, return_inverse=True)
      ia = np.full(uniq.size, -1, dtype=np.int32)
      ib = np.full(uniq.size, -1, dtype=np.int32)
      ia[inv[:len(pos)]] = np.arange(len(pos), dtype=np.int32)
      ib[inv[len(pos):]] = np.arange(len(dpos), dtype=np.int32)
      pos = np.stack([uniq // n, uniq % n], axis=1)
      self._union = (torch.from_numpy(ia).to(_dev()), torch.from_numpy(ib).to(_dev()),
                     torch.zeros(9 * uniq.size, dtype=torch.float64, device=_dev()), int(uniq.size))
    t = mas_hierarchy.build_tables(self.hierarchy, pos)
    self._tables = t
    weights = list(self.weights_for(len(self.hierarchy.levels)))
    dynamic_blocks = 0 if dyn is None else int(dyn.pattern.num_unique)
    if self.adaptive_fine_level_weight and dynamic_blocks / max(1, nv) >= self.dense_collision_block_ratio:
      weights[0] = max(weights[0], self.dense_collision_fine_level_weight)
    self.active_fine_level_weight = weights[0]
    dev = upload_mas_tables(t)
    dev.update(mas_numeric_buffers(t))
    h, keep = create_mas_handle(t, nv, weights, dev)
    self._mas = h
    self._dev_tables = (dev, keep)
    self._mas_key = key
    self._cache.release()

  def numeric_update(self, H, check=True):
    failed = ctypes.c_int32(0)
    values = H.block_sets[0].values
    if getattr(self, "_union", None) is not None:
      ia, ib, out, nu = self._union
      L.call("ys_mas_union_values", L.ptr(values), L.ptr(ia), L.ptr(H.block_sets[1].values), L.ptr(ib), nu,
             L.ptr(out), L.stream_ptr())
      values = out
    L.call("ys_mas_numeric_update", self._mas, L.ptr(values), L.stream_ptr(),
           ctypes.byref(failed) if check else None)
    return int(failed.value)

  def computeSolution(self, active_hessian, right_hand_side, initial_guess=None, tolerance=1e-3,
                      maxIterations=20000, zero_initial_guess=False, check_domains=True):
    t0 = time.perf_counter()
    rhs = _as_tensor(right_hand_side)
    n = rhs.numel()
    if n == 0:
      return 0
    self._buffers(n)
    if active_hessian is None:
      self._solution.zero_()
      return 0
    H = active_hessian
    if n != H.rows:
      raise ValueError("masSolver right-hand side size must match the matrix size")
    if not zero_initial_guess and initial_guess is not None:
      raise NotImplementedError("the device MAS PCG starts from a zero initial guess")
    self._ensure_hierarchy(H)
    # the singular-domain check is read after the solve (its status read
    # synchronises anyway); a failed domain voids the solve
    self.numeric_update(H, check=False)
    if not self.mixed_spmv:
      res = self._run_pcg(H, rhs, self._solution, False, L.YS_PREC_MAS, None, self._mas, tolerance, maxIterations,
                          True, self.stop_rule)
      status = int(res.status)
      its = int(res.iterations)
      refinements = 0
    else:
      status, its, refinements = self._solve_mixed(H, rhs, tolerance, maxIterations)
    if check_domains:
      failed = L.i32(0)
      L.call("ys_mas_failed_domains", self._mas, L.stream_ptr(), ctypes.byref(failed), ok=(L.YS_OK, L.YS_ERR_SINGULAR_DOMAIN))
      if failed.value:
        raise np.linalg.LinAlgError(f"MAS: {failed.value} domain(s) are singular")
    self._statistics = {"solver": "mas", "converged": status >= 0, "iterations": its, "refinements": refinements,
                        "result": 0 if status >= 0 else -4, "solve_seconds": time.perf_counter() - t0,
                        "levels": len(self.hierarchy.levels), "domains_per_level": self.hierarchy.domains_per_level,
                        "fine_level_weight": self.active_fine_level_weight,
                        "matrix_size": int(H.rows), "tolerance": float(tolerance)}
    return 0 if status >= 0 else -4

  def _solve_mixed(self, H, rhs, tolerance, max_iterations):
    """FP32 inner PCG + FP64 iterative refinement (true FP64 residual test)."""
    torch = _torch()
    H.ensure_fp32()
    n = H.rows
    if getattr(self, "_mixed", None) is None or self._mixed[0].numel() != n:
      ws = int(L.load().ys_refine_workspace_doubles(n // 3))
      self._mixed = (torch.zeros(n, dtype=torch.float64, device=_dev()),
                     torch.zeros(n, dtype=torch.float64, device=_dev()),
                     torch.zeros(ws, dtype=torch.float64, device=_dev()))
    r, delta, work = self._mixed
    x = self._solution
    m = H.matrix3()
    norms = (L.f64 * 2)()
    target = tolerance if self.stop_rule == "residual" else np.sqrt(tolerance)
    total_its, refinements, status = 0, 0, -4
    # the zero guess's residual is g itself (a device copy, so every inner
    # solve reads r and keeps one cached graph); the first inner tolerance
    # needs no norm (||r|| = ||g||), so the first synchronising residual
    # read comes after the first inner solve
    x.zero_()
    r.copy_(rhs)
    gnorm = rnorm = None
    for _ in range(self.max_refinements):
      if rnorm is None:
        inner_tol = max(self.refinement_tolerance, 0.5 * target)
      else:
        inner_tol = max(self.refinement_tolerance, 0.5 * target * gnorm / max(rnorm, 1e-300))
      res = self._run_pcg(H, r, delta, True, L.YS_PREC_MAS, None, self._mas, min(inner_tol, 0.5),
                          max(1, max_iterations - total_its), True, "residual")
      total_its += int(res.iterations)
      refinements += 1
      L.call("ys_refine_residual", ctypes.byref(m), L.ptr(rhs), L.ptr(x), L.ptr(delta), L.ptr(r), L.ptr(work),
             norms, L.stream_ptr())
      rnorm = float(np.sqrt(norms[0]))
      gnorm = float(np.sqrt(norms[1]))
      if rnorm <= target * gnorm:
        status = total_its
        break
      if total_its >= max_iterations or res.status < -4:
        break
    self.final_relative_residual = rnorm / max(gnorm, 1e-300)
    return status, total_its, refinements


class solver:
  """Solver dispatcher (``PKG/solver/solver.py:9-68``)."""

  def __init__(self, solver="mas", **options):
    self.solverName = ""
    self.implementation = None
    self.setSolver(solver, **options)

  @property
  def solution(self):
    return self.implementation.solution

  @property
  def statistics(self):
    return self.implementation.statistics

  def setSolver(self, solver="mas", **options):
    name = solver.strip().lower()
    if name == "jacobian":
      impl = jacobianPCGSolver(**options)
    elif name == "mas":
      impl = masSolver(**options)
    else:
      raise ValueError("solver must be either 'jacobian' or 'mas'")
    if self.implementation is not None:
      self.implementation.reset()
    self.solverName = name
    self.implementation = impl
    return self

  def reset(self):
    self.implementation.reset()

  def computeSolution(self, *args, **kwargs):
    return self.implementation.computeSolution(*args, **kwargs)
