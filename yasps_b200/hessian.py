"""Assembled Hessian and gradient of a set of energy terms.

Mirrors the reference ``hessian`` (``PKG/matrixAndVector/matrix/hessian.pyx``):
the same public attributes (``blocks_flattened``, ``block_positions``,
``blocks_start_indices``, ``block_counts``, ``block_dimensions``, their
``_dynamic`` twins, ``diagonal``, ``diagonal_blocks``, ``gradient``, ``wrt``,
``gradient_segments_start_cpu``, ``diagonal_blocks_start_cpu``), ``compute``,
``spmv`` and ``+``.  Storage is the reference's: upper-triangle duplicate-free
block COO sorted by ``(h, w, row, col)``, values row-major per block,
diagonal blocks full, off-diagonal blocks implying their transpose.

Pipeline (all on the device through libys_newton.so):

* setup (once per static structure; dynamic terms every ``compute``):
  slot codes -> local compression -> coordinates -> unique sort giving the
  pattern, the lookup and the deterministic assembly plan;
* ``compute``: element kernels write per-occurrence records, assembly sums
  them in a fixed order (bit-reproducible), diagonal blocks are extracted.
"""

from __future__ import annotations

from typing import List, Optional

import numpy as np

from . import _lib as L
from .graph import AFFINE, CONSTANT, DATA, JOIN, UNION, resolve_leaf_children


def _torch():
  import torch
  return torch


def _dev():
  from .graph import _device
  return _device()


class vector:
  """Device vector (``PKG/matrixAndVector/vector/vector.pyx``)."""

  def __init__(self, size: int, value=None):
    torch = _torch()
    self.size = int(size)
    self.value = torch.zeros(self.size, dtype=torch.float64, device=_dev()) if value is None else value

  def updateValue(self, values) -> None:
    torch = _torch()
    src = values if isinstance(values, torch.Tensor) else torch.from_numpy(np.asarray(values, dtype=np.float64))
    self.value.copy_(src.reshape(-1))

  def get(self) -> np.ndarray:
    return self.value.detach().cpu().numpy()


def fp32_slots(num_blocks: int) -> int:
  """Floats of the FP32 copy of a 3x3 block set (16-byte aligned 12-float slots)."""
  return max(12 * int(num_blocks), 12)


class _Term:
  """One energy applied to all instances of its primitive."""

  def __init__(self, request, wrt, wrt_start):
    self.request = request
    self.energy_att = request.energy
    self.expr = request.energy.expr
    self.prim = request.energy.correspondance
    self.projection_method = int(request.projection_method)
    self.dynamic = bool(request.dynamic_instances)
    self.local_targets = list(request.targets)
    self.wrt = wrt
    self.wrt_start = wrt_start
    self._const_cache = {}

  @property
  def n(self) -> int:
    return int(self.prim.numInstances)

  def leaf_kind(self, leaf):
    if leaf.operator == CONSTANT:
      return 0, 0
    if self.local_targets and not any(leaf is t for t in self.local_targets):
      return 0, 0
    for k, w in enumerate(self.wrt):
      if w is leaf:
        return 2, int(self.wrt_start[k])
    return 1, 0

  # -- affine bodies --------------------------------------------------------------
  def _affine_position(self):
    e = self.expr
    return e.x.expr if e.kind == "affine_inertia" else e.position.source.expr

  def affine_bodies(self):
    """Device body index of every element (int32): the vertex-to-body
    connectivity, through the tets for SNH (all four vertices of a tet must
    belong to one body)."""
    torch = _torch()
    key = ("affine_body", self.n)
    if key in self._const_cache:
      return self._const_cache[key]
    ap = self._affine_position()
    vb = ap.conn.value.reshape(-1)
    if self.expr.kind == "affine_inertia":
      body = vb
    else:
      tets = self.expr.position.through.value.reshape(-1, 4).to(torch.int64)
      tb = vb.to(torch.int64)[tets] if self.n else torch.zeros((0, 4), dtype=torch.int64, device=_dev())
      if self.n and not bool((tb == tb[:, :1]).all().item()):
        raise ValueError("stable_neo_hookean: every tetrahedron of affine bodies must lie in one body")
      body = tb[:, 0].to(torch.int32).contiguous() if self.n else torch.zeros(1, dtype=torch.int32, device=_dev())
    if self.n and int(body[:self.n].max().item()) >= ap.bodies.numInstances:
      raise ValueError("affine bodies: a vertex refers to a body beyond the body primitive")
    self._const_cache[key] = body
    return body

  def coupled(self):
    """``(leaves, prefix, affine child, AffinePosition)`` when the barrier's
    position union holds the vertices of affine bodies (``x = A xbar + t``,
    the collision union of ``dropping_in_container.py:344``), else None."""
    key = ("coupled",)
    if key in self._const_cache:
      return self._const_cache[key]
    out = None
    if self.expr.kind == "vertex":
      leaves, prefix = resolve_leaf_children(self.expr.position.source)
      idx = [i for i, l in enumerate(leaves) if l.operator == AFFINE]
      if len(idx) > 1:
        raise ValueError("a position union may hold one primitive of affine-body vertices")
      if idx:
        if self.expr.code not in (1, 2, 3, 4, 8, 9, 10, 11):
          raise ValueError(f"{type(self.expr).__name__}: only the contact barriers and the lagged friction kinds "
                           "take affine-body vertices")
        ap = leaves[idx[0]].expr
        vb = ap.conn.value.reshape(-1)
        if vb.numel() and int(vb.max().item()) >= ap.bodies.numInstances:
          raise ValueError("affine bodies: a vertex refers to a body beyond the body primitive")
        out = (leaves, prefix, idx[0], ap)
    self._const_cache[key] = out
    return out

  # -- slot codes ---------------------------------------------------------------
  def codes(self):
    """Device (codes int32 [n*K], sizes int16 [n*K], K, slot_stride)."""
    torch = _torch()
    n = self.n
    cp = self.coupled()
    if cp is not None:
      leaves, prefix, ac, ap = cp
      kinds, starts = zip(*((0, 0) if i == ac else self.leaf_kind(l) for i, l in enumerate(leaves)))
      ak, aw = self.leaf_kind(ap.affine)
      tk, tw = self.leaf_kind(ap.translation)
      K = 4 * self.expr.arity
      codes = torch.empty(max(n * K, 1), dtype=torch.int32, device=_dev())
      sizes = torch.empty(max(n * K, 1), dtype=torch.int16, device=_dev())
      arr = lambda v, t: (t * len(v))(*v)
      L.call("ys_coupled_indices", L.ptr(self.expr.position.through.value), n, self.expr.arity, len(leaves),
             arr(prefix, L.u32), arr(kinds, L.i32), arr(starts, L.u32), ac, L.ptr(ap.conn.value),
             ap.bodies.numInstances, ak, aw, tk, tw, L.ptr(codes), L.ptr(sizes), L.stream_ptr())
      return codes, sizes, K, 1
    if self.expr.kind == "snh":
      join = self.expr.position
      conn = join.through.value
      leaves, prefix = resolve_leaf_children(join.source)
      dim = 4
    elif self.expr.kind == "vertex":
      join = self.expr.position
      conn = join.through.value
      leaves, prefix = resolve_leaf_children(join.source)
      dim = self.expr.arity
    elif self.expr.kind == "inertia":
      key = ("identity", n)
      if key not in self._const_cache:
        self._const_cache[key] = torch.arange(max(n, 1), dtype=torch.int32, device=_dev())
      conn = self._const_cache[key]
      leaves, prefix = [self.expr.x], [0, n]
      dim = 1
    elif self.expr.kind == "affine_ortho":
      # arguments: the rows of A, gathered from A seen as 3 row-vectors a body
      key = ("rows", n)
      if key not in self._const_cache:
        self._const_cache[key] = torch.arange(max(3 * n, 1), dtype=torch.int32, device=_dev())
      conn = self._const_cache[key]
      leaves, prefix = [self.expr.rotation], [0, 3 * n]
      dim = 3
    elif self.expr.kind in ("affine_inertia", "affine_snh"):
      ap = self._affine_position()
      nb = ap.bodies.numInstances
      body = self.affine_bodies()
      key = ("affine_conn", n, nb)
      if key not in self._const_cache:
        b = body[:n].to(torch.int64)
        c = torch.stack([3 * b, 3 * b + 1, 3 * b + 2, 3 * nb + b], dim=1) if n else torch.zeros((1, 4), dtype=torch.int64, device=_dev())
        self._const_cache[key] = c.to(torch.int32).contiguous()
      conn = self._const_cache[key]
      leaves, prefix = [ap.affine, ap.translation], [0, 3 * nb, 4 * nb]
      dim = 4
    else:  # pragma: no cover
      raise NotImplementedError(self.expr.kind)
    nc = len(leaves)
    kinds, starts = zip(*(self.leaf_kind(l) for l in leaves))
    stride = 2 if nc > 1 else 1
    K = dim * stride
    codes = torch.empty(max(n * K, 1), dtype=torch.int32, device=_dev())
    sizes = torch.empty(max(n * K, 1), dtype=torch.int16, device=_dev())
    arr = lambda v, t: (t * len(v))(*v)
    L.call("ys_join_union_indices", L.ptr(conn), n, dim, nc, arr(prefix, L.u32), arr(kinds, L.i32),
           arr(starts, L.u32), 3, L.ptr(codes), L.ptr(sizes), L.stream_ptr())
    return codes, sizes, K, stride

  # -- element evaluation --------------------------------------------------------
  def _param(self, p, n):
    torch = _torch()
    kind, v = p
    if kind == "value":
      return None, float(v)
    if kind == "scene":
      return None, v.scalar()
    return v.value, 0.0

  def _union3(self, att):
    leaves, prefix = resolve_leaf_children(att)
    u = L.Union3()
    for c, leaf in enumerate(leaves):
      u.child[c] = None if leaf.operator == AFFINE else L.ptr(leaf.value)
    for c, p in enumerate(prefix):
      u.prefix[c] = p
    u.num_children = len(leaves)
    return u

  def evaluate(self, plan, block_records, grad_records, energy=None):
    torch = _torch()
    n = self.n
    if n == 0:
      return
    e = self.expr
    s = L.stream_ptr()
    if e.kind == "snh":
      if e.rest.through is not e.position.through:
        raise ValueError("stable_neo_hookean: rest and current positions must use the same connectivity")
      a = L.SnhArgs()
      a.position = self._union3(e.position.source)
      a.rest = self._union3(e.rest.source)
      a.tets = L.ptr(e.position.through.value)
      a.num_elements = n
      mu_arr, a.mu_value = self._param(e.mu_p, n)
      lam_arr, a.lam_value = self._param(e.lam_p, n)
      a.mu, a.lam = L.ptr(mu_arr), L.ptr(lam_arr)
      a.dt = self._param(e.dt_p, n)[1]
      a.projection_method = self.projection_method
      a.plan = plan
      a.block_records, a.grad_records = L.ptr(block_records), L.ptr(grad_records)
      a.energy = L.ptr(energy)
      key = ("work", n)
      if key not in self._const_cache:
        self._const_cache[key] = (torch.empty(n, dtype=torch.int32, device=_dev()),
                                  torch.zeros(1, dtype=torch.int32, device=_dev()))
      wl, wc = self._const_cache[key]
      a.work_list, a.work_count = L.ptr(wl), L.ptr(wc)
      import ctypes
      L.call("ys_snh_eval", ctypes.byref(a), s)
    elif e.kind == "vertex":
      import ctypes
      a = L.EnergyArgs()
      a.kind = e.code
      a.position = self._union3(e.position.source)
      if e.rest is not None:
        a.rest = self._union3(e.rest.source)
      else:
        a.rest.num_children = 0
      if e.needs_rest and e.rest is None:
        raise ValueError(f"{type(e).__name__} needs rest positions")
      a.conn = L.ptr(e.position.through.value)
      a.arity = e.arity
      a.num_elements = n
      if e.per_element is not None:
        a.params = L.ptr(e.per_element.value)
        a.param_stride = e.per_element.size
      for k, p in enumerate(e.params_p):
        a.values[k] = self._param(p, n)[1]
      a.projection_method = self.projection_method
      a.plan = plan
      a.block_records, a.grad_records = L.ptr(block_records), L.ptr(grad_records)
      a.energy = L.ptr(energy)
      cp = self.coupled()
      if cp is None:
        L.call("ys_energy_eval", ctypes.byref(a), s)
      else:
        ap = cp[3]
        c = L.CoupledArgs()
        c.base = a
        c.affine_child = cp[2]
        c.vertex_body = L.ptr(ap.conn.value)
        c.rest = L.ptr(ap.rest.value)
        c.affine, c.translation = L.ptr(ap.affine.value), L.ptr(ap.translation.value)
        c.num_bodies = ap.bodies.numInstances
        if "status" not in self._const_cache:
          self._const_cache["status"] = torch.zeros(1, dtype=torch.int32, device=_dev())
        st = self._const_cache["status"]
        st.zero_()
        c.status = L.ptr(st)
        L.call("ys_coupled_energy_eval", ctypes.byref(c), s)
    elif e.kind in ("affine_ortho", "affine_inertia", "affine_snh"):
      import ctypes
      a = L.AffineArgs()
      a.num_elements = n
      a.projection_method = self.projection_method
      a.plan = plan
      a.block_records, a.grad_records = L.ptr(block_records), L.ptr(grad_records)
      a.energy = L.ptr(energy)
      if e.kind == "affine_ortho":
        a.kind = L.YS_AFFINE_ORTHOGONALITY
        a.affine = L.ptr(e.rotation.value)
        a.num_bodies = n
        a.stiffness = e.stiffness
      else:
        ap = self._affine_position()
        a.affine, a.translation = L.ptr(ap.affine.value), L.ptr(ap.translation.value)
        a.num_bodies = ap.bodies.numInstances
        a.body = L.ptr(self.affine_bodies())
        a.dt = self._param(e.dt_p, n)[1]
        if e.kind == "affine_inertia":
          a.kind = L.YS_AFFINE_INERTIA
          a.rest = L.ptr(ap.rest.value)
          a.x_before = L.ptr(e.x_before.value)
          a.velocity = L.ptr(e.vel.value) if e.vel is not None else None
          m_arr, m_val = self._param(e.mass_p, n)
          if m_arr is None:
            key = ("mass", n, m_val)
            if key not in self._const_cache:
              self._const_cache[key] = torch.full((n,), m_val, dtype=torch.float64, device=_dev())
            m_arr = self._const_cache[key]
          a.mass = L.ptr(m_arr)
          for k in range(3):
            a.gravity[k] = e.gravity[k]
        else:
          a.kind = L.YS_AFFINE_SNH
          a.rest = L.ptr(e.rest.source.value)
          a.num_rest = e.rest.source.correspondance.numInstances
          a.tets = L.ptr(e.position.through.value)
          mu_arr, a.mu_value = self._param(e.mu_p, n)
          lam_arr, a.lam_value = self._param(e.lam_p, n)
          a.mu, a.lam = L.ptr(mu_arr), L.ptr(lam_arr)
      L.call("ys_affine_eval", ctypes.byref(a), s)
    elif e.kind == "inertia":
      import ctypes
      a = L.InertiaArgs()
      a.position = L.ptr(e.x.value)
      a.x_before = L.ptr(e.x_before.value)
      a.velocity = L.ptr(e.vel.value) if e.vel is not None else None
      m_arr, m_val = self._param(e.mass_p, n)
      if m_arr is None:
        key = ("mass", n, m_val)
        if key not in self._const_cache:
          self._const_cache[key] = torch.full((n,), m_val, dtype=torch.float64, device=_dev())
        m_arr = self._const_cache[key]
      a.mass = L.ptr(m_arr)
      a.dt = self._param(e.dt_p, n)[1]
      for k in range(3):
        a.gravity[k] = e.gravity[k]
      a.num_vertices = n
      a.plan = plan
      a.block_records, a.grad_records = L.ptr(block_records), L.ptr(grad_records)
      a.energy = L.ptr(energy)
      L.call("ys_inertia_eval", ctypes.byref(a), s)


class _Pattern:
  """Device pattern + assembly plan of one occurrence set."""

  def __init__(self, coords, dims, m):
    import ctypes
    torch = _torch()
    self.m = m
    cap = max(m, 1)
    i32 = lambda k: torch.empty(max(k, 1), dtype=torch.int32, device=_dev())
    self.positions = i32(2 * cap)
    self.dims = torch.empty(2 * cap, dtype=torch.int16, device=_dev())
    self.value_offset = i32(cap + 1)
    self.lookup = i32(cap)
    self.record = i32(cap)
    self.record_begin = i32(cap)
    self.record_count = i32(cap)
    ws = L.u64(0)
    L.call("ys_pattern_workspace_bytes", m, ctypes.byref(ws))
    work = torch.empty(int(ws.value), dtype=torch.uint8, device=_dev())
    out = L.PatternOut()
    out.positions, out.block_dims, out.value_offset = L.ptr(self.positions), L.ptr(self.dims), L.ptr(self.value_offset)
    out.lookup, out.record = L.ptr(self.lookup), L.ptr(self.record)
    out.record_begin, out.record_count = L.ptr(self.record_begin), L.ptr(self.record_count)
    L.call("ys_pattern_build", L.ptr(coords), L.ptr(dims), m, L.ptr(work), int(ws.value), ctypes.byref(out),
           L.stream_ptr())
    self.num_unique = int(out.num_unique)
    nc = int(out.num_categories)
    self.category_dims = [int(x) for x in out.category_dims[:2 * nc]]
    self.category_counts = [int(x) for x in out.category_counts[:nc]]
    self.category_starts = [int(x) for x in out.category_starts[:nc + 1]] if nc else [0]
    self.total_records = int(out.total_records)
    self.total_values = self.category_starts[-1] if nc else 0
    self.all3 = nc == 1 and self.category_dims == [3, 3]


class _StreamPlan:
  """Device arrays of a streamed-tile SpMV plan (``ys_spmv_stream_plan``)
  and the packed FP32 blocks it streams (``ys_spmv_stream_fill``)."""

  def __init__(self, desc, rows, words, halo, src, slot_of, blocks32, caps, slots):
    self.desc, self.rows, self.words, self.halo, self.src, self.blocks32 = desc, rows, words, halo, src, blocks32
    self.slot_of = slot_of  # each stored block's own and cross slot (the streamed assembly writes both)
    self.block_cap, self.entry_cap, self.halo_cap = caps
    self.slots = slots
    self.filled = None  # values32 version the blocks were packed from

  def struct(self):
    st = L.SpmvStream()
    st.blocks32, st.desc, st.rows = L.ptr(self.blocks32), L.ptr(self.desc), L.ptr(self.rows)
    st.words, st.halo = L.ptr(self.words), L.ptr(self.halo)
    st.block_cap, st.entry_cap, st.halo_cap = self.block_cap, self.entry_cap, self.halo_cap
    return st

  def pointers(self):
    return (self.blocks32.data_ptr(), self.desc.data_ptr(), self.words.data_ptr())


class _BlockSet:
  def __init__(self):
    self.terms: List[_Term] = []
    self.pattern: Optional[_Pattern] = None
    self.values = None
    self.values32 = None
    self.records = None
    self.infos = []
    self.spmv = None  # (row_ptr, entry_block, entry_col)
    self.tiles = None  # (row_block, tile capacity) of the tiled SpMV, or (None, 0)
    self.stream = None  # _StreamPlan of the streamed-tile SpMV, False when the set has none
    self.stream_written = False  # the last assembly wrote the packed blocks too


class hessian:
  """Assembled Hessian of energy terms w.r.t. the minimisation targets."""

  def __init__(self, wrt, requests_static=(), requests_dynamic=()):
    self.__wrt = list(wrt)
    sizes = [w.size * w.correspondance.numInstances for w in self.__wrt]
    self.gradient_segments_start_cpu = [0] + np.cumsum(sizes).tolist()
    dsz = [w.size * w.size * w.correspondance.numInstances for w in self.__wrt]
    self.diagonal_blocks_start_cpu = [0] + np.cumsum(dsz).tolist()
    self.wrt_start_indices = self.gradient_segments_start_cpu
    self.rows = self.cols = int(self.gradient_segments_start_cpu[-1])
    if self.rows <= 0:
      raise ValueError("hessian: total target size must be positive")
    self.symmetric_storage = True
    self._requests_static = list(requests_static)
    self._requests_dynamic = list(requests_dynamic)
    self._setup = False
    self.want_fp32 = False
    # diagonal / diagonal_blocks are extracted from the assembled blocks when
    # first read after a compute (block-Jacobi reads them, MAS does not);
    # want_diagonal = True extracts them with every compute
    self.want_diagonal = False
    self._diag_stale = True
    self.values32_current = False
    # bumped whenever the FP32 block values change (the streamed SpMV's
    # packed copy is refreshed from them before the next FP32 solve)
    self.values32_version = 0
    self.gradient: Optional[vector] = None
    self._diagonal = None
    self._diagonal_blocks = None
    self.energy_buffers = {}

  # -- composition ----------------------------------------------------------------
  @property
  def wrt(self):
    return self.__wrt

  def __add__(self, other: "hessian") -> "hessian":
    if not isinstance(other, hessian):
      raise TypeError("hessian.__add__: unsupported operand")
    if len(self.wrt) != len(other.wrt) or any(a is not b for a, b in zip(self.wrt, other.wrt)):
      raise ValueError("hessian.__add__: wrt mismatch")
    return hessian(self.wrt, self._requests_static + other._requests_static,
                   self._requests_dynamic + other._requests_dynamic)

  # -- setup -----------------------------------------------------------------------
  def _plan_terms(self, terms):
    """Codes, compression, coordinates for a list of terms (device)."""
    import ctypes
    torch = _torch()
    s = L.stream_ptr()
    info = []
    total = 0
    for t in terms:
      n = t.n
      codes, sizes, K, stride = t.codes()
      perm = torch.empty(max(n * K, 1), dtype=torch.int16, device=_dev())
      outer = torch.empty(n + 1, dtype=torch.int32, device=_dev())
      L.call("ys_compress_indices", L.ptr(codes), L.ptr(sizes), n, K, L.ptr(perm), None, L.ptr(outer), s)
      m = int(outer[n].item()) if n else 0
      info.append(dict(term=t, codes=codes, sizes=sizes, K=K, stride=stride, perm=perm, outer=outer, m=m, off=total))
      total += m
    coords = torch.empty(max(2 * total, 2), dtype=torch.int32, device=_dev())
    dims = torch.empty(max(2 * total, 2), dtype=torch.int16, device=_dev())
    for d in info:
      if d["m"] == 0:
        continue
      off = d["off"]
      L.call("ys_compute_coordinates", L.ptr(d["codes"]), L.ptr(d["perm"]), L.ptr(d["sizes"]), L.ptr(d["outer"]),
             d["term"].n, d["K"], coords.data_ptr() + 8 * off, dims.data_ptr() + 4 * off, s)
    return info, coords, dims, total

  def _gradient_plan(self, infos):
    torch = _torch()
    s = L.stream_ptr()
    total = 0
    for d in infos:
      n, K = d["term"].n, d["K"]
      d["gouter"] = torch.empty(n + 1, dtype=torch.int32, device=_dev())
      L.call("ys_gradient_coordinates", L.ptr(d["codes"]), L.ptr(d["sizes"]), n, K, L.ptr(d["gouter"]), None, None,
             None, s)
      d["gm"] = int(d["gouter"][n].item()) if n else 0
      d["goff"] = total
      total += d["gm"]
    coords = torch.empty(max(2 * total, 2), dtype=torch.int32, device=_dev())
    dims = torch.empty(max(2 * total, 2), dtype=torch.int16, device=_dev())
    for d in infos:
      if d["gm"] == 0:
        continue
      n, K = d["term"].n, d["K"]
      L.call("ys_gradient_coordinates", L.ptr(d["codes"]), L.ptr(d["sizes"]), n, K, L.ptr(d["gouter"]),
             coords.data_ptr() + 8 * d["goff"], dims.data_ptr() + 4 * d["goff"], s)
    pat = _Pattern(coords, dims, total)
    self._grad_pattern = pat
    self._grad_records = torch.empty(max(pat.total_records, 1), dtype=torch.float64, device=_dev())

  def _build_set(self, bs: _BlockSet, infos, coords, dims, total):
    torch = _torch()
    bs.pattern = _Pattern(coords, dims, total)
    bs.records = torch.empty(max(bs.pattern.total_records, 1), dtype=torch.float64, device=_dev())
    if bs.values is None or bs.values.numel() < max(bs.pattern.total_values, 1):
      bs.values = torch.zeros(max(bs.pattern.total_values, 1), dtype=torch.float64, device=_dev())
    bs.values32 = None
    bs.infos = infos
    # every plan of the old pattern goes with it
    bs.spmv = None
    bs.tiles = None
    bs.stream = None
    bs.stream_written = False

  def _term_plan(self, d, bs):
    p = L.TermPlan()
    p.codes = L.ptr(d["codes"])
    p.K = d["K"]
    p.slot_stride = d["stride"]
    p.coord_outer = L.ptr(d["outer"])
    p.record = bs.pattern.record.data_ptr() + 4 * d["off"]
    p.grad_outer = L.ptr(d["gouter"])
    p.grad_record = self._grad_pattern.record.data_ptr() + 4 * d["goff"]
    return p

  def _setup_compute(self):
    torch = _torch()
    wrt = self.__wrt
    self._static = _BlockSet()
    self._dynamic = _BlockSet()
    self._static.terms = [_Term(r, wrt, self.wrt_start_indices) for r in self._requests_static]
    self._dynamic.terms = [_Term(r, wrt, self.wrt_start_indices) for r in self._requests_dynamic]
    self._static_infos = self._plan_terms(self._static.terms)
    self._build_set(self._static, *self._static_infos)
    self.gradient = vector(self.rows)
    self._diagonal = torch.zeros(self.rows, dtype=torch.float64, device=_dev())
    self._diagonal_blocks = torch.zeros(max(self.diagonal_blocks_start_cpu[-1], 1), dtype=torch.float64,
                                       device=_dev())
    self._setup = True

  def _refresh_dynamic(self):
    infos = self._plan_terms(self._dynamic.terms)
    self._build_set(self._dynamic, *infos)
    self._gradient_plan(self._static_infos[0] + infos[0])

  # -- numeric --------------------------------------------------------------------
  def compute(self, local_gradient: Optional[vector] = None):
    torch = _torch()
    if not self._setup:
      self._setup_compute()
      if not self._dynamic.terms:
        self._gradient_plan(self._static_infos[0])
    if self._dynamic.terms:
      self._refresh_dynamic()
    if local_gradient is not None:
      self.gradient = local_gradient
    s = L.stream_ptr()
    for bs in (self._static, self._dynamic):
      for d in bs.infos:
        t = d["term"]
        eng = self.energy_buffers.get(id(t))
        t.evaluate(self._term_plan(d, bs), bs.records, self._grad_records, eng)
    statuses = [d["term"]._const_cache["status"] for bs in (self._static, self._dynamic) for d in bs.infos
                if "status" in d["term"]._const_cache]
    if statuses:
      st = torch.cat(statuses).cpu()
      if bool((st != 0).any()):
        k = int((st != 0).nonzero()[0, 0])
        raise ValueError(f"contact with affine bodies: element {int(st[k]) - 1} of a term names a vertex "
                         "outside the position union or a body beyond the body primitive")
    for bs in (self._static, self._dynamic):
      self._assemble(bs)
    self.gradient.value.zero_()
    gp = self._grad_pattern
    if gp.num_unique:
      L.call("ys_assemble_strided", L.ptr(self._grad_records), L.ptr(gp.record_begin), L.ptr(gp.record_count),
             L.ptr(gp.positions), 2, L.ptr(gp.dims), gp.num_unique, L.ptr(self.gradient.value), s)
    self._diag_stale = True
    if self.want_diagonal:
      self._extract_diagonal()
    self.values32_current = self.want_fp32
    self.values32_version += 1
    for bs in (self._static, self._dynamic):
      if bs.stream and bs.stream_written:
        bs.stream.filled = (self.values32_version, bs.values32.data_ptr())
      bs.stream_written = False
    return self

  def term_energies(self):
    """Per-element energies of every term (device tensors), energy kernels only."""
    torch = _torch()
    if not self._setup:
      self._setup_compute()
      if not self._dynamic.terms:
        self._gradient_plan(self._static_infos[0])
    out = []
    plan = L.TermPlan()
    for bs in (self._static, self._dynamic):
      for t in bs.terms:
        key = ("energy_values", t.n)
        if key not in t._const_cache:
          t._const_cache[key] = torch.empty(max(t.n, 1), dtype=torch.float64, device=_dev())
        e = t._const_cache[key]
        if t.n:
          t.evaluate(plan, None, None, e)
        out.append((t, e[:t.n]))
    return out

  def computeTotalEnergy(self) -> float:
    """Sum of all terms' energies: each term summed on the device in a fixed
    order (``ys_sum``), the terms added on the host in request order
    (``minimizer.pyx:396-407``)."""
    torch = _torch()
    terms = self.term_energies()
    if getattr(self, "_sum_work", None) is None:
      self._sum_work = torch.empty(int(L.load().ys_sum_workspace_doubles()), dtype=torch.float64, device=_dev())
    sums = torch.zeros(max(len(terms), 1), dtype=torch.float64, device=_dev())
    s = L.stream_ptr()
    for k, (t, e) in enumerate(terms):
      L.call("ys_sum", L.ptr(e), t.n, sums.data_ptr() + 8 * k, L.ptr(self._sum_work), s)
    total = 0.0
    for v in sums[:len(terms)].cpu().tolist():
      total += v
    return total

  @property
  def diagonal(self):
    """Diagonal entries of the assembled matrix (``hessian.pyx`` ``diagonal``)."""
    if self._diag_stale and self._setup:
      self._extract_diagonal()
    return self._diagonal

  @property
  def diagonal_blocks(self):
    """Per-variable diagonal blocks (``hessian.pyx`` ``diagonal_blocks``)."""
    if self._diag_stale and self._setup:
      self._extract_diagonal()
    return self._diagonal_blocks

  def _extract_diagonal(self):
    s = L.stream_ptr()
    self._diag_stale = False
    self._diagonal.zero_()
    self._diagonal_blocks.zero_()
    nat = len(self.__wrt)
    arr = lambda v: (L.u32 * len(v))(*v)
    seg = arr(self.gradient_segments_start_cpu)
    asz = arr([w.size for w in self.__wrt])
    dst = arr(self.diagonal_blocks_start_cpu[:nat])
    for bs in (self._static, self._dynamic):
      p = bs.pattern
      if p is None or p.num_unique == 0:
        continue
      L.call("ys_extract_diagonal", L.ptr(bs.values), L.ptr(p.positions), L.ptr(p.dims), L.ptr(p.value_offset),
             p.num_unique, nat, seg, asz, dst, L.ptr(self._diagonal_blocks), L.ptr(self._diagonal), 1, s)

  def _assemble(self, bs: _BlockSet):
    torch = _torch()
    p = bs.pattern
    if p is None or p.num_unique == 0:
      return
    s = L.stream_ptr()
    v32 = None
    if self.want_fp32 and p.all3:
      n32 = fp32_slots(p.num_unique)
      if bs.values32 is None or bs.values32.numel() < n32:
        bs.values32 = torch.zeros(n32, dtype=torch.float32, device=_dev())
      v32 = bs.values32
    sp = bs.stream
    if (p.all3 and sp and v32 is not None and bs.spmv is not None and
        sp.slot_of.numel() == 2 * p.num_unique):
      # the streamed SpMV's packed blocks are written by the assembly itself
      L.call("ys_assemble3_streamed", L.ptr(bs.records), L.ptr(p.record_begin), L.ptr(p.record_count),
             L.ptr(p.value_offset), p.num_unique, L.ptr(bs.values), L.ptr(v32), L.ptr(sp.slot_of),
             L.ptr(sp.blocks32), s)
      bs.stream_written = True
    elif p.all3:
      L.call("ys_assemble3", L.ptr(bs.records), L.ptr(p.record_begin), L.ptr(p.record_count), L.ptr(p.value_offset),
             p.num_unique, L.ptr(bs.values), L.ptr(v32), s)
    else:
      L.call("ys_assemble", L.ptr(bs.records), L.ptr(p.record_begin), L.ptr(p.record_count), L.ptr(p.value_offset),
             L.ptr(p.dims), p.num_unique, L.ptr(bs.values), L.ptr(v32), s)

  # -- reference layout of wide (9-DoF) targets -------------------------------------
  @property
  def wide_targets(self) -> bool:
    """True when a target is wider than 3 (the 9-DoF ``affine_matrices``)."""
    return any(w.size != 3 for w in self.__wrt)

  def _reference_view(self, bs: _BlockSet):
    """The block set in the reference's layout, for scenes with 9-DoF
    targets: internally the affine matrix of a body is three 3-DoF rows (so
    the SpMV, the MAS hierarchy and the FP32 copy see 3x3 blocks only); the
    reference keeps one 9-DoF slot (``dropping_in_container.py:241-243``), so
    its pattern has 9x9 / 9x3 / 3x9 / 3x3 categories sorted by (h, w, row,
    col) (``coordinateCompressionKernel.pyx:34-53``).  The view re-runs the
    compression, coordinates and pattern build on the slot codes with each
    body's three A-row slots folded into one slot of size 9 (the other two
    become padding), which gives the reference's positions, dims, category
    counts and starts, and lookups; its values are gathered from the 3x3
    blocks.  Returns ``(pattern, value map)`` cached per pattern."""
    import ctypes
    torch = _torch()
    p = bs.pattern
    cached = getattr(bs, "ref_view", None)
    if cached is not None and cached[0] is p:
      return cached[1], cached[2]
    s = L.stream_ptr()
    a_ranges = [(self.wrt_start_indices[k], self.wrt_start_indices[k + 1]) for k, w in enumerate(self.__wrt)
                if w.size == 9]
    info, total = [], 0
    for d in bs.infos:
      t = d["term"]
      n, K = t.n, d["K"]
      codes = d["codes"][:n * K].to(torch.int64).clone()
      sizes = d["sizes"][:n * K].to(torch.int64).clone()
      for a0, a1 in a_ranges:
        off = codes - 2 - a0
        inside = (codes >= 2) & (off >= 0) & (codes - 2 < a1)
        row = torch.div(off, 3, rounding_mode="floor")
        body = torch.div(row, 3, rounding_mode="floor")
        first = inside & (row % 3 == 0)
        codes = torch.where(first, a0 + 9 * body + 2, torch.where(inside, torch.zeros_like(codes), codes))
        sizes = torch.where(first, torch.full_like(sizes, 9), torch.where(inside, torch.zeros_like(sizes), sizes))
      codes = codes.to(torch.int32).contiguous()
      sizes = sizes.to(torch.int16).contiguous()
      perm = torch.empty(max(n * K, 1), dtype=torch.int16, device=_dev())
      outer = torch.empty(n + 1, dtype=torch.int32, device=_dev())
      L.call("ys_compress_indices", L.ptr(codes), L.ptr(sizes), n, K, L.ptr(perm), None, L.ptr(outer), s)
      m = int(outer[n].item()) if n else 0
      info.append((codes, sizes, perm, outer, n, K, m, total))
      total += m
    coords = torch.empty(max(2 * total, 2), dtype=torch.int32, device=_dev())
    dims = torch.empty(max(2 * total, 2), dtype=torch.int16, device=_dev())
    for codes, sizes, perm, outer, n, K, m, off in info:
      if m:
        L.call("ys_compute_coordinates", L.ptr(codes), L.ptr(perm), L.ptr(sizes), L.ptr(outer), n, K,
               coords.data_ptr() + 8 * off, dims.data_ptr() + 4 * off, s)
    ref = _Pattern(coords, dims, total)
    # value map: every reference entry (R + a, C + b) from the 3x3 block that
    # holds it in the internal upper storage (transposed below the diagonal)
    nu, N = ref.num_unique, self.rows
    pos = ref.positions[:2 * nu].view(nu, 2).to(torch.int64)
    dm = ref.dims[:2 * nu].view(nu, 2).to(torch.int64)
    voff = ref.value_offset[:nu].to(torch.int64)
    hw = dm[:, 0] * dm[:, 1]
    blk = torch.repeat_interleave(torch.arange(nu, device=_dev()), hw)
    local = torch.arange(int(hw.sum().item()), device=_dev()) - torch.repeat_interleave(torch.cumsum(hw, 0) - hw, hw)
    a_ = torch.div(local, dm[blk, 1], rounding_mode="floor")
    b_ = local % dm[blk, 1]
    r, c = pos[blk, 0] + a_, pos[blk, 1] + b_
    lo, hi = torch.minimum(r, c), torch.maximum(r, c)
    swap = r > c
    ipos = p.positions[:2 * p.num_unique].view(-1, 2).to(torch.int64)
    keys = ipos[:, 0] * N + ipos[:, 1]
    want = (lo - lo % 3) * N + (hi - hi % 3)
    ib = torch.searchsorted(keys, want)
    ib = torch.clamp(ib, max=max(p.num_unique - 1, 0))
    if not bool((keys[ib] == want).all()):
      raise RuntimeError("hessian: reference layout names a block the internal pattern does not hold")
    er = torch.where(swap, c % 3, r % 3)
    ec = torch.where(swap, r % 3, c % 3)
    src = p.value_offset[:p.num_unique].to(torch.int64)[ib] + 3 * er + ec
    dst = voff[blk] + local
    vmap = torch.empty(max(ref.total_values, 1), dtype=torch.int64, device=_dev())
    vmap[dst] = src
    bs.ref_view = (p, ref, vmap)
    return ref, vmap

  # -- reference attribute surface ---------------------------------------------------
  def _set_attr(self, bs, name):
    p = bs.pattern if bs is not None else None
    if p is not None and p.num_unique and self.wide_targets:
      ref, vmap = self._reference_view(bs)
      if name == "values":
        return bs.values[vmap[:max(ref.total_values, 1)]]
      if name == "lookups":
        return ref.lookup[:ref.m]
      return {"positions": ref.positions[:2 * ref.num_unique], "starts": ref.category_starts,
              "counts": ref.category_counts, "dims": ref.category_dims}[name]
    if p is None or p.num_unique == 0:
      return {"values": _torch().zeros(1, dtype=_torch().float64, device=_dev()),
              "positions": _torch().zeros(2, dtype=_torch().int32, device=_dev()), "starts": [],
              "counts": [], "dims": [], "lookups": _torch().zeros(0, dtype=_torch().int32, device=_dev())}[name]
    return {"values": bs.values, "positions": p.positions[:2 * p.num_unique], "starts": p.category_starts,
            "counts": p.category_counts, "dims": p.category_dims, "lookups": p.lookup[:p.m]}[name]

  blocks_flattened = property(lambda self: self._set_attr(self._static, "values"))
  block_positions = property(lambda self: self._set_attr(self._static, "positions"))
  blocks_start_indices = property(lambda self: self._set_attr(self._static, "starts"))
  block_counts = property(lambda self: self._set_attr(self._static, "counts"))
  block_dimensions = property(lambda self: self._set_attr(self._static, "dims"))
  blocks_flattened_dynamic = property(lambda self: self._set_attr(self._dynamic, "values"))
  block_positions_dynamic = property(lambda self: self._set_attr(self._dynamic, "positions"))
  blocks_start_indices_dynamic = property(lambda self: self._set_attr(self._dynamic, "starts"))
  block_counts_dynamic = property(lambda self: self._set_attr(self._dynamic, "counts"))
  block_dimensions_dynamic = property(lambda self: self._set_attr(self._dynamic, "dims"))
  # occurrence -> value offset of every element block, flattened over the
  # terms in order (the reference's lookup arrays, hessian.pyx:782-808)
  lookups = property(lambda self: self._set_attr(self._static, "lookups"))
  lookups_dynamic = property(lambda self: self._set_attr(self._dynamic, "lookups"))

  def blocks3(self):
    """``(positions [2 nu], values [9 nu])`` of the static set in the internal
    3x3 storage the device kernels run on (the public attributes give the
    reference's layout, which differs for 9-DoF targets)."""
    p = self._static.pattern
    return p.positions[:2 * p.num_unique], self._static.values[:9 * p.num_unique]

  @property
  def block_sets(self):
    return [bs for bs in (self._static, self._dynamic) if bs.pattern is not None and bs.pattern.num_unique]

  def ensure_fp32(self):
    """FP32 copies of the block values (assembled FP64 sums cast once)."""
    torch = _torch()
    if self.values32_current:
      return
    for bs in self.block_sets:
      nu = bs.pattern.num_unique
      v = torch.zeros((max(nu, 1), 12), dtype=torch.float32, device=_dev())
      v[:nu, :9] = bs.values[:9 * nu].view(nu, 9).to(torch.float32)
      bs.values32 = v.reshape(-1)
    self.values32_current = True
    self.values32_version += 1

  def spmv_plan(self, bs: _BlockSet):
    """Row plan of a 3x3 block set for the deterministic SpMV."""
    import ctypes
    torch = _torch()
    if bs.spmv is not None:
      return bs.spmv
    p = bs.pattern
    if not p.all3:
      raise NotImplementedError("the device SpMV and PCG support 3x3 blocks (3-DoF variables)")
    nv = self.rows // 3
    ws = L.u64(0)
    L.call("ys_spmv_plan_workspace_bytes", p.num_unique, nv, ctypes.byref(ws))
    work = torch.empty(int(ws.value), dtype=torch.uint8, device=_dev())
    # padded for the tiled SpMV's 16-byte copies (ys_spmv3_x32_tiled)
    row_ptr = torch.zeros(nv + 4, dtype=torch.int32, device=_dev())
    eb = torch.zeros(2 * p.num_unique + 4, dtype=torch.int32, device=_dev())
    ec = torch.zeros(2 * p.num_unique + 4, dtype=torch.int32, device=_dev())
    L.call("ys_spmv_plan_build", L.ptr(p.positions), p.num_unique, nv, L.ptr(work), int(ws.value), L.ptr(row_ptr),
           L.ptr(eb), L.ptr(ec), L.stream_ptr())
    bs.spmv = (row_ptr, eb, ec)
    bs.tiles = None
    bs.stream = None
    return bs.spmv

  def tile_plan(self, bs: _BlockSet):
    """``(row_block, tile block capacity, tile entry capacity)`` of the tiled
    SpMV for a 3x3 block set (``ys_spmv_tile_plan``); ``(None, 0, 0)`` when
    the set has none."""
    import ctypes
    torch = _torch()
    row_ptr, eb, _ = self.spmv_plan(bs)
    if bs.tiles is None:
      nv = self.rows // 3
      row_block = torch.zeros(nv + 4, dtype=torch.int32, device=_dev())
      cap, ecap = L.u32(0), L.u32(0)
      rc = L.call("ys_spmv_tile_plan", L.ptr(bs.pattern.positions), bs.pattern.num_unique, L.ptr(row_ptr), L.ptr(eb),
                  nv, L.ptr(row_block), ctypes.byref(cap), ctypes.byref(ecap), L.stream_ptr(),
                  ok=(L.YS_OK, L.YS_ERR_INVALID))
      bs.tiles = (row_block, int(cap.value), int(ecap.value)) if rc == L.YS_OK else (None, 0, 0)
    return bs.tiles

  def stream_plan(self, bs: _BlockSet):
    """The streamed-tile SpMV plan of a 3x3 block set with FP32 values
    (``ys_spmv_stream_plan``), its packed blocks current with the FP32
    values; None when the set has no FP32 values or no such plan (a tile
    beyond the plan's limits: the tiled SpMV stays in use)."""
    import ctypes
    torch = _torch()
    if bs.values32 is None:
      return None
    row_ptr, eb, ec = self.spmv_plan(bs)
    row_block, cap, _ = self.tile_plan(bs)
    if bs.stream is None:
      bs.stream = False
      if row_block is not None and cap > 0:
        nv = self.rows // 3
        entries = int(row_ptr[nv].item())
        words = L.u64(0)
        L.call("ys_spmv_stream_words", entries, nv, ctypes.byref(words))
        nw = int(words.value)
        ntiles = (nv + L.YS_SPMV_TILE_ROWS - 1) // L.YS_SPMV_TILE_ROWS
        i32 = lambda k: torch.zeros(k, dtype=torch.int32, device=_dev())
        desc, rows, wd, halo, src = i32(4 * (ntiles + 1)), i32(68 * ntiles), i32(nw), i32(nw), i32(nw)
        caps = (L.u32 * 3)()
        nu = bs.pattern.num_unique
        slot_of = i32(2 * nu)
        rc = L.call("ys_spmv_stream_plan", L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), L.ptr(row_block), nv, nw,
                    L.ptr(desc), L.ptr(rows), L.ptr(wd), L.ptr(halo), L.ptr(src), nu, L.ptr(slot_of), caps,
                    L.stream_ptr(), ok=(L.YS_OK, L.YS_ERR_CAPACITY))
        if rc == L.YS_OK:
          blocks32 = torch.zeros(9 * nw, dtype=torch.float32, device=_dev())
          bs.stream = _StreamPlan(desc, rows, wd, halo, src, slot_of, blocks32, tuple(int(c) for c in caps), nw)
    sp = bs.stream
    if not sp:
      return None
    if sp.filled != (self.values32_version, bs.values32.data_ptr()):
      L.call("ys_spmv_stream_fill", L.ptr(bs.values32), L.ptr(sp.src), sp.slots, L.ptr(sp.blocks32),
             L.stream_ptr())
      sp.filled = (self.values32_version, bs.values32.data_ptr())
    return sp

  def spmv(self, direction: vector, transpose: bool = False, fp32: bool = False) -> vector:
    """``H x`` (symmetric, so ``transpose`` gives the same product)."""
    out = vector(self.rows)
    first = True
    for bs in self.block_sets:
      row_ptr, eb, ec = self.spmv_plan(bs)
      vals = (None, bs.values32) if fp32 else (bs.values, None)
      L.call("ys_spmv3", L.ptr(vals[0]), L.ptr(vals[1]), L.ptr(row_ptr), L.ptr(eb), L.ptr(ec), self.rows // 3,
             L.ptr(direction.value), L.ptr(out.value), 0 if first else 1, L.stream_ptr())
      first = False
    return out

  def matrix3(self, fp32=False):
    """C descriptor of the (up to two) 3x3 block sets."""
    m = L.Matrix3()
    sets = self.block_sets
    m.num_sets = len(sets)
    for k, bs in enumerate(sets):
      row_ptr, eb, ec = self.spmv_plan(bs)
      m.values[k] = L.ptr(bs.values)
      m.values32[k] = L.ptr(bs.values32) if bs.values32 is not None else None
      m.row_ptr[k], m.entry_block[k], m.entry_col[k] = L.ptr(row_ptr), L.ptr(eb), L.ptr(ec)
      row_block, cap, ecap = self.tile_plan(bs)
      m.row_block[k], m.tile_cap[k], m.entry_cap[k] = L.ptr(row_block), cap, ecap
      # (the PCG runs the streamed SpMV for a single block set only)
      sp = self.stream_plan(bs) if len(sets) == 1 else None
      if sp is not None:
        m.stream[k] = sp.struct()
    m.num_vars = self.rows // 3
    return m
