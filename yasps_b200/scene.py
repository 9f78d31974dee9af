"""Scene and minimizer: the user-facing Newton-step API.

Mirrors ``PKG/scene/scene.pyx:155-200`` (``addEnergy``, ``addMinimizeTarget``,
``minimizeEnergy``) and ``PKG/minimizer/minimizer.pyx:85-407``: energies are
recorded as requests, the active Hessian is the sum of the static and
dynamic terms, ``minimizeEnergy`` computes the gradient and Hessian and
solves ``H x = g`` with the selected linear solver (MAS by default) from a
zero initial guess, and returns one solution segment per target.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import List

from .graph import CONSTANT, DATA, ENERGY, attribute, mesh
from .hessian import hessian
from .solver import solver


@dataclass
class energyRequest:
  """One ``addEnergy`` call (``PKG/minimizer/minimizer.pyx:20-84``)."""

  energy: attribute
  targets: List[attribute] = field(default_factory=list)
  projection_method: int = 1
  dynamic_instances: bool = False


class minimizer:
  def __init__(self):
    self.requests: List[energyRequest] = []
    self.requests_dynamic: List[energyRequest] = []
    self.wrt: List[attribute] = []
    self._hessian = None
    self._ignored = set()
    self.linearSolver = solver("mas")
    self.solutionSegments = []

  def setSolver(self, solver_name="mas", **options):
    self.linearSolver.reset()
    self.linearSolver = solver(solver_name, **options)
    self.solutionSegments = []
    return self.linearSolver

  @property
  def solverName(self):
    return self.linearSolver.solverName

  def addEnergy(self, e, targets=(), projection_method=1, dynamic_instances=False, **flags):
    if e.operator != ENERGY:
      raise ValueError("minimizer.addEnergy: the attribute must be an energy")
    # separate_hessian_jacobian: the reference then evaluates J^T H J from
    # explicit Jacobian blocks instead of a symbolic expansion; the matrix is
    # the same (for a linear map from the targets the inner Hessian is
    # projected either way, PKG/differentiator/differentiator.pyx:795-799;
    # for a nonlinear one the flag is ignored, PKG/matrixAndVector/matrix/
    # hessian.pyx:905).  Every element kernel here already forms J^T H J from
    # explicit blocks, so the flag is accepted and changes nothing.
    unsupported = {k: v for k, v in flags.items() if v and k in ("gradient_only", "lto")}
    if unsupported:
      raise NotImplementedError(f"minimizer.addEnergy: unsupported options {sorted(unsupported)}")
    if any(r.energy is e for r in self.requests + self.requests_dynamic):
      raise ValueError("minimizer.addEnergy: energy already exists.")
    req = energyRequest(e, list(targets), int(projection_method), bool(dynamic_instances))
    (self.requests_dynamic if dynamic_instances else self.requests).append(req)
    self._hessian = None

  def addWrt(self, wrt):
    seen = set()
    for a in wrt:
      if a.hash in seen:
        raise ValueError(f"minimizer.addWrt: wrt {a.fullName} is duplicate attribute.")
      if a.operator != DATA:
        raise ValueError(f"minimizer.addWrt: wrt {a.fullName} is non-data attribute.")
      if a.isDynamic:
        raise ValueError(f"minimizer.addWrt: wrt {a.fullName} is dynamic attribute.")
      seen.add(a.hash)
    self.wrt = list(wrt)
    self._hessian = None
    self.linearSolver.reset()
    self.solutionSegments = []

  def ignoreEnergies(self, energies):
    self._ignored = {e.hash for e in energies}
    self._hessian = None

  def activeHessian(self) -> hessian:
    if self._hessian is None:
      st = [r for r in self.requests if r.energy.hash not in self._ignored]
      dy = [r for r in self.requests_dynamic if r.energy.hash not in self._ignored]
      self._hessian = hessian(self.wrt, st, dy)
    return self._hessian

  def computeNumericValue(self) -> hessian:
    if not self.wrt:
      raise ValueError("minimizer.computeNumericValue: wrt is not initialized. Please call addWrt first.")
    H = self.activeHessian()
    impl = self.linearSolver.implementation
    H.want_fp32 = bool(getattr(impl, "mixed_spmv", False))
    H.compute()
    return H

  @property
  def gradient(self):
    return self.activeHessian().gradient.value

  def computeTotalEnergy(self) -> float:
    """Total energy of the active (not ignored) energies (``minimizer.pyx:396-407``)."""
    return self.activeHessian().computeTotalEnergy()

  def backtrackingLineSearch(self, direction=None, step=1.0, shrink=0.5, max_steps=8):
    """Move the targets to ``x - alpha d`` with the largest ``alpha = step *
    shrink^k`` (k < max_steps) that does not increase the total energy, as the
    reference examples' substep loop does after their CCD step bound
    (``examples/dropping_in_container/dropping_in_container.py:486-560``).
    ``direction`` defaults to the last solution segments.  Returns the
    accepted alpha (0.0 when no step decreased the energy: targets restored).
    """
    segs = self.solutionSegments if direction is None else direction
    if len(segs) != len(self.wrt):
      raise ValueError("minimizer.backtrackingLineSearch: one direction segment per target")
    before = self.computeTotalEnergy()
    saved = [w.value.clone() for w in self.wrt]
    alpha = float(step)
    for _ in range(int(max_steps)):
      for w, x0, d in zip(self.wrt, saved, segs):
        w.copyValueFrom(x0 - alpha * d.reshape(x0.shape), non_blocking=False)
      if self.computeTotalEnergy() <= before:
        return alpha
      alpha *= shrink
    for w, x0 in zip(self.wrt, saved):
      w.copyValueFrom(x0, non_blocking=False)
    return 0.0

  def computeHessianAndGradient(self, tolerance=1e-3, maxIterations=20000):
    H = self.computeNumericValue()
    code = self.linearSolver.computeSolution(H, H.gradient, None, tolerance=tolerance, maxIterations=maxIterations,
                                             zero_initial_guess=True)
    sol = self.linearSolver.solution
    self.solutionSegments = []
    c = 0
    for w in self.wrt:
      k = w.size * w.correspondance.numInstances
      self.solutionSegments.append(sol[c:c + k])
      c += k
    return code


class scene:
  """Top-level container (``PKG/scene/scene.pyx``)."""

  def __init__(self, name: str):
    self.name = name
    self.type = "scene"
    self.numInstances = 1
    self.meshes = {}
    self.attributes = {}
    self.minimizer = minimizer()
    self._pre_targets = set()

  @property
  def fullName(self):
    return self.name

  def addMesh(self, name: str) -> mesh:
    m = mesh(name, self)
    self.meshes[name] = m
    return m

  def addConstant(self, name: str, rows: int = 1, cols: int = 1) -> attribute:
    a = attribute(name, self, CONSTANT, rows, cols)
    self.attributes[name] = a
    return a

  def __getitem__(self, name):
    return self.attributes[name]

  def addEnergy(self, e, targets=(), projection_method=1, save_intermediate=False, gradient_only=False,
                dynamic_instances=False, separate_hessian_jacobian=False, grouped_add=False, lto=False):
    if e.name == "":
      raise ValueError("scene.addEnergy: energy attribute must have a name.")
    for t in targets:
      self._pre_targets.add(t.fullName)
    self.minimizer.addEnergy(e, targets, projection_method, dynamic_instances, gradient_only=gradient_only,
                             separate_hessian_jacobian=separate_hessian_jacobian, lto=lto)

  def addMinimizeTarget(self, target):
    names = {t.fullName for t in target}
    if len(names) != len(target):
      raise ValueError("scene.addMinimizeTarget: target contains duplicate attributes.")
    if not self._pre_targets.issubset(names):
      raise ValueError(f"scene.addMinimizeTarget: target is missing attributes {self._pre_targets - names}")
    self.minimizer.addWrt(target)

  def minimizeEnergy(self, tolerance=1e-3, maxIterations=20000):
    code = self.minimizer.computeHessianAndGradient(tolerance=tolerance, maxIterations=maxIterations)
    if code < 0:
      print("scene.minimizeEnergy: got error code", code)
    return self.minimizer.solutionSegments

  @property
  def gradient(self):
    return self.minimizer.gradient

  def computeTotalEnergy(self) -> float:
    return self.minimizer.computeTotalEnergy()

  def backtrackingLineSearch(self, direction=None, step=1.0, shrink=0.5, max_steps=8):
    return self.minimizer.backtrackingLineSearch(direction, step, shrink, max_steps)

  def ignoreEnergies(self, energies):
    self.minimizer.ignoreEnergies(energies)
