"""Scene graph: primitives, unions, connectivities and attributes.

Mirrors the reference's scene-graph API (``PKG/mesh/mesh.pyx:66-96``,
``PKG/primitive/primitive.pyx:91-262``, ``PKG/primitive/primitiveUnion.pyx:115-191``,
``PKG/connectivity/connectivity.pyx:13-118``) for the attribute kinds the
Newton inner loop consumes:

* ``DATA``      -- ``primitive.addAttribute(name, rows, cols)``: values that can
  be minimisation targets;
* ``CONSTANT``  -- ``primitive.addConstant(name, rows, cols)`` / ``scene.addConstant``;
* ``JOIN``      -- ``primitive.addAttribute(name, through=conn, source=attr)``:
  the source attribute gathered through a connectivity;
* ``UNION``     -- ``primitiveUnion.addAttribute(name)``: the same-named attribute
  of every child, stacked in child order;
* ``ENERGY``    -- ``primitive.addAttribute(name, computed_attribute=expr)`` with an
  energy expression from :mod:`yasps_b200.energies`;
* ``AFFINE``    -- ``primitive.addAttribute(name, computed_attribute=affine_position(...))``:
  the positions ``A xbar + t`` of the vertices of affine bodies
  (``examples/dropping_in_container_mixed/dropping_in_container.py:261-270``).

The symbolic expression language of the reference (its ``attribute``
arithmetic, autodiff and code generator) is not part of this library: the
energies of the hot path are fixed CUDA element kernels.

Values live on the host until first used on the device; ``attribute.value``
returns the device tensor (float64, instance-major, ``rows*cols`` per instance).
"""

from __future__ import annotations

import itertools
from typing import List, Optional

import numpy as np

DATA, CONSTANT, JOIN, UNION, ENERGY, AFFINE = "DATA", "CONSTANT", "JOIN", "UNION", "ENERGY", "AFFINE"

_ids = itertools.count()


def _device():
  import torch
  if not torch.cuda.is_available():
    raise RuntimeError("yasps_b200 needs a CUDA device for numeric work")
  return torch.device("cuda", torch.cuda.current_device())


class attribute:
  """One attribute of a primitive, union or scene."""

  def __init__(self, name: str, owner, operator: str, rows: int = 1, cols: int = 1, *, through=None, source=None,
               children=None, expr=None):
    self.name = name
    self.correspondance = owner
    self.operator = operator
    self.rows, self.cols = int(rows), int(cols)
    self.through = through
    self.source = source
    self.children = list(children or [])
    self.expr = expr
    self.hash = next(_ids)
    self._host: Optional[np.ndarray] = None
    self._dev = None
    self._version = 0

  # -- identity ---------------------------------------------------------------
  @property
  def size(self) -> int:
    return self.rows * self.cols

  @property
  def fullName(self) -> str:
    return f"{self.correspondance.fullName}_{self.name}"

  @property
  def isDynamic(self) -> bool:
    return bool(getattr(self.correspondance, "isDynamic", False))

  def __repr__(self):
    return f"attribute({self.fullName}, {self.operator}, {self.rows}x{self.cols})"

  def resize(self, rows: int, cols: int) -> "attribute":
    """The same attribute seen as ``rows x cols`` (``PKG/attribute/attribute.pyx:250-255``);
    a JOIN keeps its connectivity and source."""
    if int(rows) * int(cols) != self.size:
      raise ValueError(f"attribute.resize: {self.fullName} has {self.size} entries, not {rows}x{cols}")
    view = attribute(self.name, self.correspondance, self.operator, rows, cols, through=self.through,
                     source=self.source, children=self.children, expr=self.expr)
    view._host, view._dev = self._host, self._dev
    view.hash = self.hash
    return view

  # -- values -----------------------------------------------------------------
  def updateValue(self, values) -> None:
    """Set the values (host array-like or a CUDA tensor) of a DATA/CONSTANT attribute."""
    if self.operator not in (DATA, CONSTANT):
      raise ValueError(f"attribute.updateValue: {self.fullName} is {self.operator}, not DATA/CONSTANT")
    n = getattr(self.correspondance, "numInstances", 1)
    try:
      import torch
      is_tensor = isinstance(values, torch.Tensor)
    except ImportError:  # pragma: no cover
      is_tensor = False
    if is_tensor:
      if values.numel() != n * self.size:
        raise ValueError(f"attribute.updateValue: expected {n * self.size} values, got {values.numel()}")
      self._dev = values.detach().reshape(-1).to(dtype=torch.float64).contiguous()
      self._host = None
    else:
      arr = np.asarray(values, dtype=np.float64).reshape(-1)
      if arr.size == 1 and n * self.size != 1:
        arr = np.full(n * self.size, float(arr[0]))
      if arr.size != n * self.size:
        raise ValueError(f"attribute.updateValue: expected {n * self.size} values, got {arr.size}")
      self._host = arr.copy()
      if self._dev is not None and self._dev.numel() == arr.size:
        import torch
        self._dev.copy_(torch.from_numpy(arr), non_blocking=False)
      else:
        self._dev = None
    self._version += 1

  def setScalar(self, v: float) -> None:
    """Set a constant's value on the host only (no device copy; a device
    mirror is rebuilt when ``value`` is next read)."""
    n = getattr(self.correspondance, "numInstances", 1)
    self._host = np.full(n * self.size, float(v))
    self._dev = None
    self._version += 1

  def copyValueFrom(self, src, non_blocking: bool = True) -> None:
    """Copy ``src`` (a tensor, e.g. pinned host memory) into the existing
    device values on the current stream; the host mirror is dropped."""
    dst = self.value
    if src.numel() != dst.numel():
      raise ValueError(f"attribute.copyValueFrom: expected {dst.numel()} values, got {src.numel()}")
    dst.copy_(src.reshape(-1), non_blocking=non_blocking)
    self._host = None
    self._version += 1

  @property
  def host_value(self) -> np.ndarray:
    if self._host is None:
      if self._dev is None:
        raise ValueError(f"attribute {self.fullName} has no value")
      self._host = self._dev.detach().cpu().numpy().copy()
    return self._host

  @property
  def value(self):
    """Device tensor (float64) of a DATA/CONSTANT attribute."""
    if self.operator not in (DATA, CONSTANT):
      raise ValueError(f"attribute.value: {self.fullName} is {self.operator}")
    if self._dev is None:
      import torch
      if self._host is None:
        n = getattr(self.correspondance, "numInstances", 1)
        self._host = np.zeros(n * self.size)
      self._dev = torch.from_numpy(self._host).to(_device())
    return self._dev

  def scalar(self) -> float:
    """Host scalar of a 1x1 scene-level constant."""
    return float(self.host_value[0])


class connectivity:
  """Fixed-dimension index map from a primitive's instances to a target's
  instances (``PKG/connectivity/connectivity.pyx:13-41``)."""

  def __init__(self, name, owner, target, values, dimension: int):
    if dimension <= 0:
      raise ValueError("connectivity: only fixed dimensions (> 0) are supported on the hot path")
    self.name = name
    self.correspondance = owner
    self.target = target
    self.dimension = int(dimension)
    self._host = None
    self._dev = None
    self.updateConnectivity(values)

  @property
  def fullName(self):
    return f"{self.correspondance.fullName}_{self.name}"

  def updateConnectivity(self, values) -> None:
    arr = np.asarray(values, dtype=np.uint32).reshape(-1, self.dimension)
    if arr.size and int(arr.max()) >= self.target.numInstances:
      raise ValueError(f"connectivity {self.fullName}: index beyond {self.target.fullName}")
    self._host = np.ascontiguousarray(arr)
    self._dev = None

  @property
  def host_value(self) -> np.ndarray:
    return self._host

  @property
  def value(self):
    if self._dev is None:
      import torch
      # int32 storage of uint32 indices (bit-identical below 2^31).
      self._dev = torch.from_numpy(self._host.astype(np.int32).reshape(-1)).to(_device())
    return self._dev


class primitive:
  """A set of instances carrying attributes (``PKG/primitive/primitive.pyx``)."""

  def __init__(self, name: str, numInstances: int, owner=None, isDynamic: bool = False):
    self.name = name
    self.correspondance = owner
    self.numInstances = int(numInstances)
    self.isDynamic = bool(isDynamic)
    self.attributes = {}
    self.connectivities = {}
    self.type = "primitive"

  @property
  def fullName(self):
    return self.name if self.correspondance is None else f"{self.correspondance.fullName}_{self.name}"

  def __getitem__(self, name):
    return self.attributes[name]

  def addAttribute(self, name: str, rows: int = 1, cols: int = 1, *, through: connectivity = None,
                   source: attribute = None, computed_attribute=None) -> attribute:
    if name in self.attributes:
      raise ValueError(f"primitive.addAttribute: {name} already exists on {self.fullName}")
    if through is not None:
      if source is None:
        raise ValueError("primitive.addAttribute: a JOIN needs a source attribute")
      if through.correspondance is not self:
        raise ValueError("primitive.addAttribute: the connectivity must belong to this primitive")
      if source.correspondance is not through.target:
        raise ValueError("primitive.addAttribute: the source must live on the connectivity target")
      att = attribute(name, self, JOIN, through.dimension, source.size, through=through, source=source)
    elif computed_attribute is not None:
      from .energies import AffinePosition, EnergyExpr
      if isinstance(computed_attribute, AffinePosition):
        att = attribute(name, self, AFFINE, 3, 1, expr=computed_attribute)
      elif isinstance(computed_attribute, EnergyExpr):
        att = attribute(name, self, ENERGY, 1, 1, expr=computed_attribute)
      else:
        raise TypeError("primitive.addAttribute: computed attributes must be energy expressions "
                        "or affine_position from yasps_b200.energies")
      computed_attribute.bind(att)
    else:
      att = attribute(name, self, DATA, rows, cols)
    self.attributes[name] = att
    return att

  def addConstant(self, name: str, rows: int = 1, cols: int = 1) -> attribute:
    if name in self.attributes:
      raise ValueError(f"primitive.addConstant: {name} already exists on {self.fullName}")
    att = attribute(name, self, CONSTANT, rows, cols)
    self.attributes[name] = att
    return att

  def addConnectivity(self, name: str, target, values, dimension: int) -> connectivity:
    con = connectivity(name, self, target, values, dimension)
    self.connectivities[name] = con
    return con

  def updateNumInstances(self, n: int) -> None:
    """Change the instance count of a dynamic primitive (contact terms)."""
    if not self.isDynamic:
      raise ValueError("primitive.updateNumInstances: only dynamic primitives can change size")
    self.numInstances = int(n)


class primitiveUnion:
  """Primitives stacked in child order (``PKG/primitive/primitiveUnion.pyx:115-191``)."""

  def __init__(self, name: str, children: List[primitive], owner=None):
    if not children:
      raise ValueError("primitiveUnion: needs at least one child")
    self.name = name
    self.correspondance = owner
    self.children = list(children)
    self.attributes = {}
    self.type = "union"
    self.isDynamic = False

  @property
  def fullName(self):
    return self.name if self.correspondance is None else f"{self.correspondance.fullName}_{self.name}"

  @property
  def numInstances(self) -> int:
    return sum(c.numInstances for c in self.children)

  @property
  def children_prefix(self) -> List[int]:
    out = [0]
    for c in self.children:
      out.append(out[-1] + c.numInstances)
    return out

  def __getitem__(self, name):
    return self.attributes[name]

  def addAttribute(self, name: str) -> attribute:
    kids = []
    for c in self.children:
      if name not in c.attributes:
        raise ValueError(f"primitiveUnion.addAttribute: child {c.fullName} has no attribute {name}")
      kids.append(c.attributes[name])
    rows, cols = kids[0].rows, kids[0].cols
    if any(k.size != kids[0].size for k in kids):
      raise ValueError("primitiveUnion.addAttribute: children attributes differ in size")
    att = attribute(name, self, UNION, rows, cols, children=kids)
    self.attributes[name] = att
    return att


class mesh:
  """Container of primitives (``PKG/mesh/mesh.pyx:66-96``)."""

  def __init__(self, name: str, owner=None):
    self.name = name
    self.correspondance = owner
    self.primitives = {}

  @property
  def fullName(self):
    return self.name if self.correspondance is None else f"{self.correspondance.fullName}_{self.name}"

  def addPrimitive(self, name: str, numInstances: int, isDynamic: bool = False) -> primitive:
    p = primitive(name, numInstances, self, isDynamic)
    self.primitives[name] = p
    return p

  def addPrimitiveUnion(self, name: str, children: List[primitive]) -> primitiveUnion:
    u = primitiveUnion(name, children, self)
    self.primitives[name] = u
    return u


def resolve_leaf_children(att: attribute):
  """Leaf attributes reached by a gathered attribute, with union prefixes.

  Returns ``(children, prefix)``: for a DATA/CONSTANT source a single child
  with prefix ``[0, n]``; for a UNION the child attributes in union order.
  """
  if att.operator in (DATA, CONSTANT):
    return [att], [0, att.correspondance.numInstances]
  if att.operator == UNION:
    return list(att.children), list(att.correspondance.children_prefix)
  raise ValueError(f"{att.fullName}: only DATA, CONSTANT or UNION attributes can be gathered")
