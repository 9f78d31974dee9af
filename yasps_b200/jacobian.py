"""Rectangular second-order Jacobians and the differentiator front end.

Mirrors ``PKG/matrixAndVector/matrix/secondOrderJacobian.pyx`` (the
rectangular matrix ``d2E / (d row_wrt d column_wrt)``: ``row_wrt``,
``column_wrt``, their start indices, ``compute``, ``spmv(x, transpose)``,
``+`` and the reference's block attributes) and the entry points of
``PKG/differentiator/differentiator.pyx:174-489``: ``diff2`` with equal
target lists gives the projected Hessian, with different lists the
rectangular Jacobian (never projected, as the reference's no-project
Jacobian kernel); ``diff1`` of scalar energies gives their gradient.

Values on the device through libys_newton.so: the unprojected local
Hessian of every instance over the energy's arguments
(``ys_local_hessians``, ``ys_snh_local_hessians``,
``ys_inertia_local_hessians``), the (row target, column target) pairs of
every instance (``ys_rect_coordinates``), the unique sort of
``ys_pattern_build`` (no upper-triangle fold), merged records
(``ys_rect_records``) summed in a fixed order (``ys_assemble3``), and the
deterministic products ``ys_rect_spmv``.

An argument of an energy is a row (column) slot when its leaf is one of the
row (column) targets: for the vertex-tuple energies and the SNH tetrahedra
the leaves of the position union (so ``row_wrt=[cloth position]``,
``column_wrt=[obstacle position]`` gives the cloth-obstacle coupling
blocks), for the inertia term its ``x``, ``x_before`` and ``vel``
attributes (the adjoint blocks ``d2E / (dx dx_before)`` and
``d2E / (dx dvel)`` of the reference's differentiable-simulation examples,
``examples/bunny_dropping_on_ground/bunny_dropping_on_ground.py:333-334``),
for the lagged friction kinds, functions of ``x - x_old``, also the
leaves of their step-start positions, and for the SNH tetrahedra the
leaves of their rest positions against the position leaves (shape
derivatives ``d2E / (dx dX)``) and against each other (``d2E / dX2``);
the same for the cloth energies (bending, Baraff-Witkin and StVK
membranes) through their rest frames.  Mixed derivatives through the rest
argument of the other energies and through affine-body vertices are not
built (a target among those leaves raises).
"""

from __future__ import annotations

import ctypes
from typing import List

import numpy as np

from . import _lib as L
from .graph import AFFINE, attribute, resolve_leaf_children
from .hessian import _Pattern, _dev, _torch, hessian, vector


def _start_indices(targets):
  starts = [0]
  for t in targets:
    starts.append(starts[-1] + t.size * t.correspondance.numInstances)
  return starts


def _validate_targets(targets, name, sizes=(1, 3)):
  if not isinstance(targets, list) or len(targets) == 0:
    raise ValueError(f"secondOrderJacobian.__init__: {name} must be a non-empty list.")
  seen = set()
  for t in targets:
    if not isinstance(t, attribute):
      raise TypeError(f"secondOrderJacobian.__init__: every {name} item must be an attribute.")
    if t.isDynamic:
      raise ValueError(f"secondOrderJacobian.__init__: {name} cannot contain dynamic attributes.")
    if t.hash in seen:
      raise ValueError(f"secondOrderJacobian.__init__: {name} contains a duplicate target.")
    if t.size not in sizes:
      raise NotImplementedError(f"secondOrderJacobian: target {t.fullName} of size {t.size} is not built")
    seen.add(t.hash)
  return list(targets)


class _RectTerm:
  """One energy's instances: argument connectivity and leaves, row and
  column slot codes, and its unprojected local Hessians."""

  def __init__(self, energy: attribute, jac: "secondOrderJacobian"):
    e = getattr(energy, "expr", None)
    if e is None:
      raise ValueError(f"secondOrderJacobian: {energy.fullName} is not a computed energy")
    self.energy, self.expr, self.jac = energy, e, jac
    self.prim = energy.correspondance
    self._cache = {}

  @property
  def n(self) -> int:
    return int(self.prim.numInstances)

  @property
  def difference_args(self) -> int:
    """The lagged friction kinds are functions of x - x_old: their
    step-start positions are arguments too (``ys_rect_records``'s
    difference form); 0 for the other energies."""
    e = self.expr
    return int(e.arity) if e.kind == "vertex" and e.code in (8, 9, 10, 11) and e.rest is not None else 0

  @property
  def rest_form(self) -> bool:
    """SNH or a cloth energy (bending, Baraff-Witkin, StVK) with a target
    among its rest leaves: the arguments are the element's positions and rest
    positions (``ys_snh_rest_local_hessians``, ``ys_rest_local_hessians``)."""
    return getattr(self, "_rest_form", False)

  def rest_leaves(self):
    """Leaves of the energy's rest / step-start argument (empty without one)."""
    e = self.expr
    rest = getattr(e, "rest", None)
    return resolve_leaf_children(rest.source)[0] if rest is not None else []

  def arguments(self):
    """(connectivity [n, A] int32 into the leaf union, leaves, prefix, A)."""
    torch = _torch()
    e, n = self.expr, self.n
    if e.kind in ("affine_inertia", "affine_snh") or (
        e.kind == "vertex" and any(l.operator == AFFINE for l in resolve_leaf_children(e.position.source)[0])):
      raise NotImplementedError("secondOrderJacobian: energies through affine-body vertices are not built")
    if e.kind in ("snh", "vertex"):
      leaves, prefix = resolve_leaf_children(e.position.source)
      A = 4 if e.kind == "snh" else e.arity
      if not self.difference_args and not self.rest_form:
        return e.position.through.value, leaves, prefix, A
      # [position arguments, step-start (or rest) arguments] over the union
      # of both leaf lists
      rleaves, rprefix = resolve_leaf_children(e.rest.source)
      if len(leaves) + len(rleaves) > 8:
        raise NotImplementedError("secondOrderJacobian: more than 8 leaves in the position and step-start unions")
      key = ("difference_conn", n)
      if key not in self._cache:
        c = e.position.through.value.reshape(-1)[:n * A].to(torch.int64).view(n, A) if n else \
            torch.zeros((1, A), dtype=torch.int64, device=_dev())
        self._cache[key] = torch.cat([c, c + int(prefix[-1])], dim=1).to(torch.int32).contiguous()
      return (self._cache[key], list(leaves) + list(rleaves),
              list(prefix[:-1]) + [int(prefix[-1]) + int(p) for p in rprefix], 2 * A)
    if e.kind == "inertia":
      leaves = [e.x, e.x_before] + ([e.vel] if e.vel is not None else [])
      key = ("inertia_conn", n, len(leaves))
      if key not in self._cache:
        i = torch.arange(n, dtype=torch.int64, device=_dev())
        conn = torch.stack([i + k * n for k in range(len(leaves))], dim=1) if n else \
            torch.zeros((1, len(leaves)), dtype=torch.int64, device=_dev())
        self._cache[key] = conn.to(torch.int32).contiguous()
      return self._cache[key], leaves, [k * n for k in range(len(leaves) + 1)], len(leaves)
    raise NotImplementedError(f"secondOrderJacobian: energy kind {e.kind!r} is not built")

  def codes(self, targets, starts):
    torch = _torch()
    conn, leaves, prefix, A = self.arguments()
    kinds, wstart = [], []
    for leaf in leaves:
      k = next((i for i, t in enumerate(targets) if t is leaf), None)
      kinds.append(0 if k is None else 2)
      wstart.append(0 if k is None else int(starts[k]))
    nc = len(leaves)
    stride = 2 if nc > 1 else 1
    K = A * stride
    n = self.n
    codes = torch.empty(max(n * K, 1), dtype=torch.int32, device=_dev())
    sizes = torch.empty(max(n * K, 1), dtype=torch.int16, device=_dev())
    arr = lambda v, t: (t * len(v))(*v)
    L.call("ys_join_union_indices", L.ptr(conn), n, A, nc, arr(prefix, L.u32), arr(kinds, L.i32),
           arr(wstart, L.u32), 3, L.ptr(codes), L.ptr(sizes), L.stream_ptr())
    return codes, K, stride, A

  def parameters(self):
    """``(which, attribute)`` of the energy's per-element scalar parameters
    that a Jacobian column can take: the SNH tets' Lame arrays (0 mu,
    1 lambda) and the inertia vertices' masses (0)."""
    e = self.expr
    out = []
    if e.kind == "snh":
      for which, p in ((0, e.mu_p), (1, e.lam_p)):
        if p[0] == "array":
          out.append((which, p[1]))
    elif e.kind == "inertia" and e.mass_p[0] == "array":
      out.append((0, e.mass_p[1]))
    return out

  def parameter_derivatives(self, which, out):
    """d(dE/d argument)/d parameter per element, ``[n x 3 args]``."""
    e, n = self.expr, self.n
    s = L.stream_ptr()
    if n == 0:
      return
    from .hessian import _Term
    from .scene import energyRequest
    helper = _Term(energyRequest(self.energy, [], -1, False), [], [0])
    if e.kind == "snh":
      a = self._snh_args(helper)
      L.call("ys_snh_param_jacobian", ctypes.byref(a), int(which), L.ptr(out), s)
      return
    a = L.InertiaArgs()
    a.position, a.x_before = L.ptr(e.x.value), L.ptr(e.x_before.value)
    a.velocity = L.ptr(e.vel.value) if e.vel is not None else None
    a.mass = L.ptr(e.mass_p[1].value)
    a.dt = e.dt_p[1] if e.dt_p[0] == "value" else e.dt_p[1].scalar()
    for k in range(3):
      a.gravity[k] = e.gravity[k]
    a.num_vertices = n
    L.call("ys_inertia_mass_jacobian", ctypes.byref(a), 3 if e.vel is not None else 2, L.ptr(out), s)

  def _snh_args(self, helper):
    e, n = self.expr, self.n
    a = L.SnhArgs()
    a.position = helper._union3(e.position.source)
    a.rest = helper._union3(e.rest.source)
    a.tets = L.ptr(e.position.through.value)
    a.num_elements = n
    mu_arr, a.mu_value = helper._param(e.mu_p, n)
    lam_arr, a.lam_value = helper._param(e.lam_p, n)
    a.mu, a.lam = L.ptr(mu_arr), L.ptr(lam_arr)
    a.dt = helper._param(e.dt_p, n)[1]
    return a

  def local_hessians(self, out):
    e, n = self.expr, self.n
    s = L.stream_ptr()
    if n == 0:
      return
    if e.kind == "inertia":
      m_kind, m_val = e.mass_p
      mass = m_val.value if m_kind == "array" else None
      mass_value = 0.0 if mass is not None else (m_val.scalar() if m_kind == "scene" else float(m_val))
      dt = e.dt_p[1] if e.dt_p[0] == "value" else e.dt_p[1].scalar()
      L.call("ys_inertia_local_hessians", L.ptr(mass), float(mass_value), float(dt), n,
             3 if e.vel is not None else 2, L.ptr(out), s)
      return
    from .hessian import _Term
    from .scene import energyRequest
    helper = _Term(energyRequest(self.energy, [], -1, False), [], [0])
    if e.kind == "snh":
      entry = "ys_snh_rest_local_hessians" if self.rest_form else "ys_snh_local_hessians"
      a = self._snh_args(helper)
      L.call(entry, ctypes.byref(a), L.ptr(out), s)
      return
    a = L.EnergyArgs()
    a.kind = e.code
    a.position = helper._union3(e.position.source)
    if e.rest is not None:
      a.rest = helper._union3(e.rest.source)
    else:
      a.rest.num_children = 0
    a.conn = L.ptr(e.position.through.value)
    a.arity = e.arity
    a.num_elements = n
    if e.per_element is not None:
      a.params = L.ptr(e.per_element.value)
      a.param_stride = e.per_element.size
    for k, p in enumerate(e.params_p):
      a.values[k] = helper._param(p, n)[1]
    L.call("ys_rest_local_hessians" if self.rest_form else "ys_local_hessians", ctypes.byref(a), L.ptr(out), s)


class secondOrderJacobian:
  """Rectangular matrix ``d2E / (d row_wrt d column_wrt)`` of a sum of
  scalar energies (``secondOrderJacobian.pyx:17-52``)."""

  def __init__(self, row_wrt: List[attribute], column_wrt: List[attribute], _column_sizes=(1, 3)):
    self.__row_wrt = _validate_targets(row_wrt, "row_wrt")
    self.__column_wrt = _validate_targets(column_wrt, "column_wrt", _column_sizes)
    self.__row_start = _start_indices(self.__row_wrt)
    self.__column_start = _start_indices(self.__column_wrt)
    self.rows = int(self.__row_start[-1])
    self.cols = int(self.__column_start[-1])
    self.sources: List[attribute] = []
    self.sources_dynamic: List[attribute] = []
    self._setup = None
    self.blocks_flattened = None
    self.block_positions = None
    self.block_dimensions: List[List[int]] = []
    self.blocks_start_indices: List[int] = [0]
    self.block_counts: List[int] = []
    self.blocks_flattened_dynamic = None
    self.block_positions_dynamic = None
    self.block_dimensions_dynamic: List[List[int]] = []
    self.blocks_start_indices_dynamic: List[int] = [0]
    self.block_counts_dynamic: List[int] = []

  @property
  def row_wrt(self):
    return self.__row_wrt

  @property
  def column_wrt(self):
    return self.__column_wrt

  @property
  def row_start_indices(self):
    return self.__row_start

  @property
  def column_start_indices(self):
    return self.__column_start

  def __add__(self, other: "secondOrderJacobian") -> "secondOrderJacobian":
    if not isinstance(other, secondOrderJacobian):
      raise TypeError("secondOrderJacobian.__add__: unsupported operand type(s) for +: 'secondOrderJacobian' and "
                      f"'{type(other).__name__}'")
    if len(self.row_wrt) != len(other.row_wrt) or any(a is not b for a, b in zip(self.row_wrt, other.row_wrt)):
      raise ValueError("secondOrderJacobian.__add__: row_wrt mismatch.")
    if len(self.column_wrt) != len(other.column_wrt) or any(
        a is not b for a, b in zip(self.column_wrt, other.column_wrt)):
      raise ValueError("secondOrderJacobian.__add__: column_wrt mismatch.")
    out = secondOrderJacobian(self.row_wrt, self.column_wrt)
    out.sources = self.sources + other.sources
    out.sources_dynamic = self.sources_dynamic + other.sources_dynamic
    return out

  # -- structure --------------------------------------------------------------------
  def _build(self, sources):
    torch = _torch()
    s = L.stream_ptr()
    terms = []
    total = 0
    for src in sources:
      t = _RectTerm(src, self)
      n = t.n
      diff = t.difference_args
      if not diff:
        rest = t.rest_leaves()
        in_rows = any(any(x is r for r in rest) for x in self.__row_wrt)
        in_cols = any(any(x is r for r in rest) for x in self.__column_wrt)
        rest_kinds = t.expr.kind == "snh" or (t.expr.kind == "vertex" and t.expr.code in (5, 6, 7))
        if (in_rows or in_cols) and not rest_kinds:
          raise NotImplementedError("secondOrderJacobian: mixed derivatives through the rest argument of "
                                    f"{type(t.expr).__name__} are not built")
        t._rest_form = in_rows or in_cols
      params = []
      for which, att in t.parameters():
        if any(att is x for x in self.__row_wrt):
          raise NotImplementedError("secondOrderJacobian: parameter rows are not built (take the transposed "
                                    "target lists and spmv(transpose=True))")
        k = next((i for i, x in enumerate(self.__column_wrt) if x is att), None)
        if k is not None:
          if t.rest_form:
            raise NotImplementedError("secondOrderJacobian: rest positions and parameters in one Jacobian")
          params.append((which, int(self.__column_start[k])))
      rc, K, stride, A = t.codes(self.__row_wrt, self.__row_start)
      cc, _, _, _ = t.codes(self.__column_wrt, self.__column_start)
      outer = torch.empty(n + 1, dtype=torch.int32, device=_dev())
      L.call("ys_rect_coordinates", L.ptr(rc), L.ptr(cc), n, K, stride, A, L.ptr(outer), None, None, s)
      m = int(outer[n].item()) if n else 0
      N = 3 * (diff if diff else A)  # the rest form's local Hessian covers all 8 arguments
      local_h = torch.empty(max(n * N * (N + 1) // 2, 1), dtype=torch.float64, device=_dev())
      d = dict(term=t, rc=rc, cc=cc, K=K, stride=stride, A=A, diff=diff, outer=outer, m=m, off=total,
               local_h=local_h, params=[])
      total += m
      for which, start in params:
        pouter = torch.empty(n + 1, dtype=torch.int32, device=_dev())
        L.call("ys_rect_param_coordinates", L.ptr(rc), n, K, stride, A, start, L.ptr(pouter), None, None, s)
        pm = int(pouter[n].item()) if n else 0
        deriv = torch.empty(max(3 * A * n, 1), dtype=torch.float64, device=_dev())
        d["params"].append(dict(which=which, start=start, outer=pouter, m=pm, off=total, deriv=deriv))
        total += pm
      terms.append(d)
    coords = torch.empty(max(2 * total, 2), dtype=torch.int32, device=_dev())
    dims = torch.empty(max(2 * total, 2), dtype=torch.int16, device=_dev())
    for d in terms:
      if d["m"]:
        L.call("ys_rect_coordinates", L.ptr(d["rc"]), L.ptr(d["cc"]), d["term"].n, d["K"], d["stride"], d["A"],
               L.ptr(d["outer"]), coords.data_ptr() + 8 * d["off"], dims.data_ptr() + 4 * d["off"], s)
      for q in d["params"]:
        if q["m"]:
          L.call("ys_rect_param_coordinates", L.ptr(d["rc"]), d["term"].n, d["K"], d["stride"], d["A"], q["start"],
                 L.ptr(q["outer"]), coords.data_ptr() + 8 * q["off"], dims.data_ptr() + 4 * q["off"], s)
    pat = _Pattern(coords, dims, total)
    records = torch.empty(max(pat.total_records, 1), dtype=torch.float64, device=_dev())
    values = torch.zeros(max(pat.total_values, 1), dtype=torch.float64, device=_dev())
    return dict(terms=terms, pattern=pat, records=records, values=values, plans=self._plans(pat))

  def _plans(self, pat):
    """Row and column pointers of every block category (3 rows; 1, 3 or 9
    columns) for the products."""
    torch = _torch()
    s = L.stream_ptr()
    plans = []
    b0 = 0
    nc = len(pat.category_counts) if pat.num_unique else 0
    for c in range(nc):
      h, w = pat.category_dims[2 * c], pat.category_dims[2 * c + 1]
      nb = pat.category_counts[c]
      if h != 3 or w not in (1, 3, 9):
        raise NotImplementedError(f"secondOrderJacobian: {h}x{w} blocks are not built")
      br, bc = self.rows // 3, self.cols // w
      row_ptr = torch.empty(br + 1, dtype=torch.int32, device=_dev())
      col_ptr = torch.empty(bc + 1, dtype=torch.int32, device=_dev())
      col_order = torch.empty(max(nb, 1), dtype=torch.int32, device=_dev())
      ws = L.u64(0)
      L.call("ys_rect_plan_workspace_bytes", nb, ctypes.byref(ws))
      work = torch.empty(int(ws.value), dtype=torch.uint8, device=_dev())
      pos = pat.positions.data_ptr() + 8 * b0
      L.call("ys_rect_plan", pos, nb, br, bc, w, L.ptr(row_ptr), L.ptr(col_ptr), L.ptr(col_order), L.ptr(work),
             int(ws.value), s)
      plans.append(dict(width=w, blocks=nb, first=b0, value_start=pat.category_starts[c], row_ptr=row_ptr,
                        col_ptr=col_ptr, col_order=col_order, block_cols=bc))
      b0 += nb
    return plans

  def compute(self):
    """Evaluate every term and assemble (``secondOrderJacobian.pyx:530-559``;
    dynamic sources rebuild their pattern on every call)."""
    torch = _torch()
    if any(t.size != 3 for t in self.__row_wrt):
      raise NotImplementedError("secondOrderJacobian: row targets of 3-vectors only")
    s = L.stream_ptr()
    if self._setup is None:
      self._setup = self._build(self.sources)
    dyn = self._build(self.sources_dynamic) if self.sources_dynamic else None
    for part, name in ((self._setup, ""), (dyn, "_dynamic")):
      if part is None:
        continue
      pat = part["pattern"]
      for d in part["terms"]:
        t = d["term"]
        if t.n == 0:
          continue
        if d["m"]:
          t.local_hessians(d["local_h"])
          L.call("ys_rect_records", L.ptr(d["local_h"]), d["A"], d["diff"], L.ptr(d["rc"]), L.ptr(d["cc"]), t.n,
                 d["K"], d["stride"], L.ptr(d["outer"]), pat.record.data_ptr() + 4 * d["off"],
                 L.ptr(part["records"]), s)
        for q in d["params"]:
          if not q["m"]:
            continue
          t.parameter_derivatives(q["which"], q["deriv"])
          L.call("ys_rect_param_records", L.ptr(q["deriv"]), d["A"], L.ptr(d["rc"]), t.n, d["K"], d["stride"],
                 L.ptr(q["outer"]), pat.record.data_ptr() + 4 * q["off"], L.ptr(part["records"]), s)
      nu = pat.num_unique
      if nu:
        if pat.all3:
          L.call("ys_assemble3", L.ptr(part["records"]), L.ptr(pat.record_begin), L.ptr(pat.record_count),
                 L.ptr(pat.value_offset), nu, L.ptr(part["values"]), None, s)
        else:
          L.call("ys_assemble", L.ptr(part["records"]), L.ptr(pat.record_begin), L.ptr(pat.record_count),
                 L.ptr(pat.value_offset), L.ptr(pat.dims), nu, L.ptr(part["values"]), None, s)
      setattr(self, "blocks_flattened" + name, part["values"][:pat.total_values] if nu else part["values"][:0])
      setattr(self, "block_positions" + name, pat.positions[:2 * nu])
      setattr(self, "block_dimensions" + name, list(pat.category_dims) if nu else [])
      setattr(self, "blocks_start_indices" + name, list(pat.category_starts) if nu else [0])
      setattr(self, "block_counts" + name, list(pat.category_counts) if nu else [])
    self._dynamic_part = dyn
    return self

  # -- products -----------------------------------------------------------------------
  def spmv(self, x: vector, transpose: bool = False) -> vector:
    """``J x`` (or ``J^T x``) as a new vector (``matrix.pyx:393-408``)."""
    if not isinstance(x, vector):
      raise TypeError("matrix.spmv: x must be a vector.")
    if not isinstance(transpose, (bool, np.bool_)):
      raise TypeError("matrix.spmv: transpose must be a bool.")
    n_in, n_out = (self.rows, self.cols) if transpose else (self.cols, self.rows)
    if x.size != n_in:
      orientation = "transposed " if transpose else ""
      raise ValueError(f"matrix.spmv: input vector for {orientation}matrix has size {x.size}, expected {n_in}.")
    if self._setup is None:
      raise RuntimeError("secondOrderJacobian.spmv: call compute() first")
    out = vector(n_out)
    s = L.stream_ptr()
    br = self.rows // 3
    parts = [p for p in (self._setup, getattr(self, "_dynamic_part", None)) if p is not None]
    for part in parts:
      pat = part["pattern"]
      for pl in part["plans"]:
        L.call("ys_rect_spmv", part["values"].data_ptr() + 8 * pl["value_start"],
               pat.positions.data_ptr() + 8 * pl["first"], L.ptr(pl["row_ptr"]), L.ptr(pl["col_ptr"]),
               L.ptr(pl["col_order"]), br, pl["block_cols"], pl["width"], L.ptr(x.value), L.ptr(out.value),
               int(bool(transpose)), 1, s)
    return out


class firstOrderJacobian(secondOrderJacobian):
  """Sparse first derivative of a vector attribute with respect to targets
  (``PKG/matrixAndVector/matrix/firstOrderJacobian.pyx:87-117``): rows follow
  the source's instance-major storage, columns the targets.  Built for the
  affine-body vertex positions ``x = A xbar + t`` (``affine_position``)
  against the bodies' ``affine_matrices`` (3 x 9 blocks) and
  ``translations`` (3 x 3 identities)."""

  def __init__(self, row_source: attribute, wrt: List[attribute]):
    from .energies import AffinePosition
    e = getattr(row_source, "expr", None)
    if not isinstance(e, AffinePosition):
      raise NotImplementedError("firstOrderJacobian: vector sources other than affine-body vertex positions are "
                                "not built")
    if row_source.isDynamic:
      raise ValueError("firstOrderJacobian.__init__: dynamically sized row sources are not supported because "
                       "matrix dimensions must remain fixed.")
    super().__init__([row_source], list(wrt), _column_sizes=(3, 9))
    self.__row_source = row_source
    self._map = e
    starts = self.column_start_indices
    self._a_col = next((int(starts[k]) for k, t in enumerate(self.column_wrt) if t is e.affine), -1)
    self._t_col = next((int(starts[k]) for k, t in enumerate(self.column_wrt) if t is e.translation), -1)

  @property
  def row_source(self):
    return self.__row_source

  @property
  def wrt(self):
    return self.column_wrt

  def compute(self):
    torch = _torch()
    s = L.stream_ptr()
    e = self._map
    n = int(self.__row_source.correspondance.numInstances)
    if self._setup is None:
      per = (self._a_col >= 0) + (self._t_col >= 0)
      m = n * per
      coords = torch.empty(max(2 * m, 2), dtype=torch.int32, device=_dev())
      dims = torch.empty(max(2 * m, 2), dtype=torch.int16, device=_dev())
      vb = e.conn.value
      if m:
        L.call("ys_affine_position_jacobian", L.ptr(vb), None, n, self._a_col, self._t_col, L.ptr(coords),
               L.ptr(dims), None, None, s)
      pat = _Pattern(coords, dims, m)
      records = torch.empty(max(pat.total_records, 1), dtype=torch.float64, device=_dev())
      values = torch.zeros(max(pat.total_values, 1), dtype=torch.float64, device=_dev())
      self._setup = dict(terms=[], pattern=pat, records=records, values=values, plans=self._plans(pat), m=m)
    part = self._setup
    pat = part["pattern"]
    if part["m"]:
      L.call("ys_affine_position_jacobian", None, L.ptr(e.rest.value), n, self._a_col, self._t_col, None, None,
             L.ptr(pat.record), L.ptr(part["records"]), s)
      L.call("ys_assemble", L.ptr(part["records"]), L.ptr(pat.record_begin), L.ptr(pat.record_count),
             L.ptr(pat.value_offset), L.ptr(pat.dims), pat.num_unique, L.ptr(part["values"]), None, s)
    nu = pat.num_unique
    self.blocks_flattened = part["values"][:pat.total_values] if nu else part["values"][:0]
    self.block_positions = pat.positions[:2 * nu]
    self.block_dimensions = list(pat.category_dims) if nu else []
    self.blocks_start_indices = list(pat.category_starts) if nu else [0]
    self.block_counts = list(pat.category_counts) if nu else []
    self._dynamic_part = None
    return self


class gradient(vector):
  """Gradient of scalar energies with respect to targets, as ``diff1``
  returns it (``differentiator.pyx:174-239``): ``compute`` evaluates the
  energies and fills ``value``."""

  def __init__(self, wrt, parent: hessian):
    self.wrt = list(wrt)
    self.parent = parent
    super().__init__(parent.rows)

  def compute(self):
    self.parent.compute()
    self.value = self.parent.gradient.value
    return self


class differentiator:
  """``diff1`` / ``diff2`` (``PKG/differentiator/differentiator.pyx:174-489``)."""

  @staticmethod
  def _same(a, b):
    return len(a) == len(b) and all(x is y for x, y in zip(a, b))

  def diff2(self, source, target1, target2, local_targets=(), projection_method=1, save_intermediate=False,
            separate_hessian_jacobian=False, dynamic_instances=False, grouped_add=False, lto=False):
    from .scene import energyRequest
    src = list(source) if isinstance(source, (list, tuple)) else [source]
    if not src:
      raise ValueError("differentiator.diff2: source can not be empty.")
    if self._same(list(target1), list(target2)):
      reqs = [energyRequest(e, list(local_targets), int(projection_method), bool(dynamic_instances)) for e in src]
      return hessian(list(target1), [] if dynamic_instances else reqs, reqs if dynamic_instances else [])
    for e in src:
      if e.size != 1:
        raise ValueError("differentiator.__diff2_jacobian_single: source must be a scalar attribute.")
    jac = secondOrderJacobian(list(target1), list(target2))
    if dynamic_instances:
      jac.sources_dynamic = src
    else:
      jac.sources = src
    return jac

  def diff1(self, source, global_targets, local_targets=(), dynamic_instances=False):
    from .scene import energyRequest
    src = list(source) if isinstance(source, (list, tuple)) else [source]
    if not src:
      raise ValueError("differentiator.diff1: source can not be empty.")
    if not isinstance(global_targets, list) or not global_targets:
      raise ValueError("differentiator.diff1: global_targets can not be empty.")
    vector_valued = [e.size != 1 for e in src]
    if any(vector_valued):
      if not all(vector_valued):
        raise ValueError("differentiator.diff1: scalar and vector-valued sources cannot be mixed in one call.")
      if len(src) != 1:
        raise NotImplementedError("differentiator.diff1: one vector-valued source a call")
      return firstOrderJacobian(src[0], list(global_targets))
    reqs = [energyRequest(e, list(local_targets), -1, bool(dynamic_instances)) for e in src]
    parent = hessian(list(global_targets), [] if dynamic_instances else reqs, reqs if dynamic_instances else [])
    return gradient(global_targets, parent)
