"""Energy expressions of the Newton inner loop (fixed CUDA element kernels).

Each function mirrors the signature of the reference example helper that
builds the same energy symbolically, and returns an expression to pass to
``primitive.addAttribute(name, computed_attribute=...)``:

* :func:`stable_neo_hookean` -- ``examples/dropping_in_container_mixed/helpers.py:102-127``
* :func:`inertia`            -- ``examples/dropping_in_container_mixed/helpers.py:138-141``

Parameters (``mu``, ``lam``, ``dt``, ``mass``) may be Python floats, 1x1
scene constants, or per-instance attributes of the energy's primitive.
"""

from __future__ import annotations

from .graph import AFFINE, CONSTANT, DATA, JOIN, UNION, attribute


class EnergyExpr:
  kind = "energy"

  def __init__(self):
    self.attribute = None

  def bind(self, att) -> None:
    if self.attribute is not None:
      raise ValueError("an energy expression can be bound to one attribute only")
    self.attribute = att
    self.validate(att.correspondance)

  def validate(self, prim) -> None:  # pragma: no cover - overridden
    pass


def _param(v, prim, name):
  """Normalise a parameter to ('value', float) or ('array', attribute)."""
  if isinstance(v, attribute):
    if v.size != 1:
      raise ValueError(f"{name} must be a scalar attribute")
    owner = v.correspondance
    if getattr(owner, "type", None) == "scene":
      return ("scene", v)
    if owner is not prim:
      raise ValueError(f"{name} must live on the energy's primitive or on the scene")
    return ("array", v)
  return ("value", float(v))


def _join_of_positions(att, name, dim, affine=False):
  if not isinstance(att, attribute) or att.operator != JOIN:
    raise ValueError(f"{name} must be a JOIN attribute (addAttribute(..., through=..., source=...))")
  if att.through.dimension != dim or att.source.size != 3:
    raise ValueError(f"{name} must gather {dim} 3-vectors")
  allowed = (DATA, CONSTANT, UNION, AFFINE) if affine else (DATA, CONSTANT, UNION)
  if att.source.operator not in allowed:
    raise ValueError(f"{name}: the gathered attribute must be DATA, CONSTANT or a UNION of them"
                     + (" (or affine body positions)" if affine else ""))


class SnhEnergy(EnergyExpr):
  kind = "snh"

  def __init__(self, tet_position_rest, tet_position, mu, lam, dt):
    super().__init__()
    _join_of_positions(tet_position, "tet_position", 4, affine=True)
    _join_of_positions(tet_position_rest, "tet_position_rest", 4)
    self.position = tet_position
    self.rest = tet_position_rest
    self.mu, self.lam, self.dt = mu, lam, dt
    if tet_position.source.operator == AFFINE:
      # tetrahedra of affine bodies: the element's arguments are its body's
      # A rows and t (ys_affine_eval, YS_AFFINE_SNH)
      if tet_position_rest.through is not tet_position.through:
        raise ValueError("stable_neo_hookean: rest and current positions must use the same connectivity")
      if tet_position_rest.source.operator not in (DATA, CONSTANT) or \
          tet_position_rest.source.correspondance is not tet_position.source.correspondance:
        raise ValueError("stable_neo_hookean: the rest positions of affine-body tets must be a DATA/CONSTANT "
                         "attribute of the body vertices")
      self.kind = "affine_snh"

  def validate(self, prim) -> None:
    if self.position.correspondance is not prim or self.rest.correspondance is not prim:
      raise ValueError("stable_neo_hookean: the tet attributes must live on the energy's primitive")
    self.mu_p = _param(self.mu, prim, "mu")
    self.lam_p = _param(self.lam, prim, "lam")
    self.dt_p = _param(self.dt, prim, "dt")
    if self.dt_p[0] == "array":
      raise ValueError("dt must be a scalar")


class InertiaEnergy(EnergyExpr):
  kind = "inertia"

  def __init__(self, x_before, vel, dt, x, mass, gravity):
    super().__init__()
    for a, name in ((x, "x"), (x_before, "x_before")):
      ok = (DATA, CONSTANT, AFFINE) if name == "x" else (DATA, CONSTANT)
      if not isinstance(a, attribute) or a.size != 3 or a.operator not in ok:
        raise ValueError(f"inertia: {name} must be a 3-vector DATA/CONSTANT attribute of the primitive")
    if x.operator == AFFINE:
      # vertices of affine bodies: 1/2 m |A xbar + t - x~|^2 over the body's
      # A rows and t (ys_affine_eval, YS_AFFINE_INERTIA)
      self.kind = "affine_inertia"
    if vel is not None and (not isinstance(vel, attribute) or vel.size != 3):
      raise ValueError("inertia: vel must be a 3-vector attribute or None")
    self.x, self.x_before, self.vel = x, x_before, vel
    self.dt, self.mass = dt, mass
    self.gravity = tuple(float(g) for g in gravity)

  def validate(self, prim) -> None:
    for a in (self.x, self.x_before, self.vel):
      if a is not None and a.correspondance is not prim:
        raise ValueError("inertia: attributes must live on the energy's primitive")
    if self.x.operator not in (DATA, AFFINE):
      raise ValueError("inertia: x must be a DATA attribute or affine body positions")
    self.dt_p = _param(self.dt, prim, "dt")
    self.mass_p = _param(self.mass, prim, "mass")


def stable_neo_hookean(tet_position_rest, tet_position, mu, lam, dt) -> SnhEnergy:
  """Stable Neo-Hookean tetrahedral energy scaled by ``dt^2``."""
  return SnhEnergy(tet_position_rest, tet_position, mu, lam, dt)


def inertia(x_before, vel, dt, x, mass, gravity=(0.0, -9.8, 0.0)) -> InertiaEnergy:
  """``1/2 (x - x~)^T m (x - x~)`` with ``x~ = x_before + vel dt + gravity dt^2``.

  The reference helper hard-codes ``gravity = (0, -9.8, 0)``; it is a
  parameter here.
  """
  return InertiaEnergy(x_before, vel, dt, x, mass, gravity)


# ---- vertex-tuple energies (cloth, contact, friction) -----------------------------

class VertexEnergy(EnergyExpr):
  """An energy over a JOIN of ``arity`` 3-vectors, evaluated by ``ys_energy_eval``."""

  kind = "vertex"
  code = 0
  arity = 0
  param_names = ()

  def __init__(self, position, rest=None, params=(), per_element=None):
    super().__init__()
    _join_of_positions(position, "position", self.arity)
    if rest is not None:
      _join_of_positions(rest, "rest", self.arity)
      if rest.through is not position.through:
        raise ValueError(f"{type(self).__name__}: rest and current positions must use the same connectivity")
    self.position, self.rest = position, rest
    self.params = tuple(params)
    self.per_element = per_element

  def validate(self, prim) -> None:
    if self.position.correspondance is not prim:
      raise ValueError(f"{type(self).__name__}: the position JOIN must live on the energy's primitive")
    self.params_p = [_param(v, prim, n) for v, n in zip(self.params, self.param_names)]
    for p, n in zip(self.params_p, self.param_names):
      if p[0] == "array":
        raise ValueError(f"{n} must be a scalar")
    if self.per_element is not None:
      if self.per_element.correspondance is not prim:
        raise ValueError("per-element parameters must live on the energy's primitive")


def _vertex_energy(name, code, arity, names, needs_rest):
  cls = type(name, (VertexEnergy,), {"code": code, "arity": arity, "param_names": names})
  cls.needs_rest = needs_rest
  return cls


PointPointBarrier = _vertex_energy("PointPointBarrier", 1, 2, ("dHat", "kappa"), False)
PointEdgeBarrier = _vertex_energy("PointEdgeBarrier", 2, 3, ("dHat", "kappa"), False)
PointTriangleBarrier = _vertex_energy("PointTriangleBarrier", 3, 4, ("dHat", "kappa"), False)
EdgeEdgeBarrier = _vertex_energy("EdgeEdgeBarrier", 4, 4, ("dHat", "kappa"), False)
BendingEnergy = _vertex_energy("BendingEnergy", 5, 4, ("bendStiff", "dt"), True)
BaraffWitkinEnergy = _vertex_energy("BaraffWitkinEnergy", 6, 3, ("stretchS", "shearS", "thickness", "dt"), True)
StvkMembraneEnergy = _vertex_energy("StvkMembraneEnergy", 7, 3, ("mu", "lam", "thickness", "dt"), True)
FrictionPointTriangle = _vertex_energy("FrictionPointTriangle", 8, 4, ("fDhat", "dt", "frictionRate"), True)
FrictionPointEdge = _vertex_energy("FrictionPointEdge", 9, 3, ("fDhat", "dt", "frictionRate"), True)
FrictionEdgeEdge = _vertex_energy("FrictionEdgeEdge", 10, 4, ("fDhat", "dt", "frictionRate"), True)
FrictionPointPoint = _vertex_energy("FrictionPointPoint", 11, 2, ("fDhat", "dt", "frictionRate"), True)


def point_point(position, dHat, kappa):
  """IPC barrier on the squared point-point distance (``helpers.py:143-152``)."""
  return PointPointBarrier(position, None, (dHat, kappa))


def point_edge(position, dHat, kappa):
  """IPC barrier on the squared point-edge distance (``helpers.py:154-165``)."""
  return PointEdgeBarrier(position, None, (dHat, kappa))


def point_triangle(position, dHat, kappa):
  """IPC barrier on the squared point-triangle distance (``helpers.py:167-180``)."""
  return PointTriangleBarrier(position, None, (dHat, kappa))


def edge_edge(position, dHat, kappa):
  """IPC barrier on the squared edge-edge distance (``helpers.py:182-195``)."""
  return EdgeEdgeBarrier(position, None, (dHat, kappa))


def bending(x, x_init, bendStiff, dt):
  """Dihedral bending ``kb (theta - theta0)^2 |e0| dt^2`` (``helpers.py:213-234``)."""
  return BendingEnergy(x, x_init, (bendStiff, dt))


def baraff_witkin(x_init, x, stretchS, shearS, thickness, dt):
  """Baraff-Witkin cloth stretch + shear (``helpers.py:272-292``)."""
  return BaraffWitkinEnergy(x, x_init, (stretchS, shearS, thickness, dt))


def stvk_membrane(x_init, x, mu, lam, thickness, dt):
  """StVK membrane on the Baraff-Witkin rest frame (no counterpart in the reference)."""
  return StvkMembraneEnergy(x, x_init, (mu, lam, thickness, dt))


def friction_point_triangle(position, old_position, fDhat, dt, frictionRate, lagged):
  """Lagged point-triangle friction (``friction_helpers.py:12-66, 73-182``).

  ``lagged`` is a 9-vector attribute of the energy's primitive per pair:
  ``beta1, beta2, tangent0 (3), tangent1 (3), lambda_last_h``, fixed over the
  Newton step as in the reference.
  """
  return FrictionPointTriangle(position, old_position, (fDhat, dt, frictionRate), per_element=lagged)


def friction_point_edge(position, old_position, fDhat, dt, frictionRate, lagged):
  """Lagged point-edge friction (``friction_helpers.py:12-66, 188-276``);
  ``lagged``: ``eta, 0, tangent0 (3), tangent1 (3), lambda_last_h``."""
  return FrictionPointEdge(position, old_position, (fDhat, dt, frictionRate), per_element=lagged)


def friction_edge_edge(position, old_position, fDhat, dt, frictionRate, lagged):
  """Lagged edge-edge friction (``friction_helpers.py:12-66, 283-405``);
  ``lagged``: ``gamma1, gamma2, tangent0 (3), tangent1 (3), lambda_last_h``."""
  return FrictionEdgeEdge(position, old_position, (fDhat, dt, frictionRate), per_element=lagged)


def friction_point_point(position, old_position, fDhat, dt, frictionRate, lagged):
  """Lagged point-point friction (``friction_helpers.py:12-66, 411-500``);
  ``lagged``: ``0, 0, tangent0 (3), tangent1 (3), lambda_last_h``."""
  return FrictionPointPoint(position, old_position, (fDhat, dt, frictionRate), per_element=lagged)


# ---- affine (ABD) bodies ------------------------------------------------------------

class AffinePosition:
  """``x = A xbar + t`` of the vertices of affine bodies, the computed position
  of ``examples/dropping_in_container_mixed/dropping_in_container.py:261-270``.

  ``affine_matrix`` and ``translation`` are JOINs of dimension 1 through one
  vertex-to-body connectivity of the bodies' 3x3 (row-major) and 3-vector
  DATA attributes; ``rest_position`` is the body-frame rest position of the
  vertices.  Bound with ``vertices.addAttribute("position",
  computed_attribute=affine_position(...))``; :func:`inertia` and
  :func:`stable_neo_hookean` accept the result (directly, or gathered by a
  JOIN of tetrahedra) and differentiate with respect to A and t.
  """

  kind = "affine_position"

  def __init__(self, affine_matrix, rest_position, translation):
    for a, name, size in ((affine_matrix, "affine_matrix", 9), (translation, "translation", 3)):
      if not isinstance(a, attribute) or a.operator != JOIN or a.through.dimension != 1 or a.source.size != size:
        raise ValueError(f"affine_position: {name} must be a JOIN (dimension 1) of a {size}-entry body attribute")
      if a.source.operator != DATA:
        raise ValueError(f"affine_position: {name} must gather a DATA attribute of the bodies")
    if affine_matrix.through is not translation.through:
      raise ValueError("affine_position: affine_matrix and translation must use the same connectivity")
    if affine_matrix.source.correspondance is not translation.source.correspondance:
      raise ValueError("affine_position: A and t must live on the same body primitive")
    if not isinstance(rest_position, attribute) or rest_position.size != 3 or \
        rest_position.operator not in (DATA, CONSTANT):
      raise ValueError("affine_position: rest_position must be a 3-vector DATA/CONSTANT attribute")
    self.affine = affine_matrix.source
    self.translation = translation.source
    self.conn = affine_matrix.through
    self.rest = rest_position
    self.attribute = None

  @property
  def bodies(self):
    return self.affine.correspondance

  def bind(self, att) -> None:
    if self.attribute is not None:
      raise ValueError("affine_position can be bound to one attribute only")
    prim = att.correspondance
    if self.conn.correspondance is not prim or self.rest.correspondance is not prim:
      raise ValueError("affine_position: the JOINs and the rest position must live on the vertex primitive")
    self.attribute = att


def affine_position(affine_matrix, rest_position, translation) -> AffinePosition:
  """``affine_matrix * rest_position + translation`` for affine-body vertices."""
  return AffinePosition(affine_matrix, rest_position, translation)


class AffineOrthogonalityEnergy(EnergyExpr):
  kind = "affine_ortho"

  def __init__(self, rotation, stiffness):
    super().__init__()
    if not isinstance(rotation, attribute) or rotation.size != 9 or rotation.operator != DATA:
      raise ValueError("affine_energy: rotation must be the bodies' 3x3 DATA attribute")
    self.rotation = rotation
    self.stiffness = float(stiffness)

  def validate(self, prim) -> None:
    if self.rotation.correspondance is not prim:
      raise ValueError("affine_energy: the energy must live on the bodies' primitive")


def affine_energy(rotation, stiffness=1.0) -> AffineOrthogonalityEnergy:
  """``stiffness * 1/2 |A^T A - I|_F^2`` per body (``helpers.py:201-211``; the
  reference helper has no stiffness, i.e. 1)."""
  return AffineOrthogonalityEnergy(rotation, stiffness)
