"""Regenerate the golden fixtures in this folder from the reference itself.

Run in a container where the reference checkout is available::

    python tests/golden/make_golden.py /path/to/yasps-reference

It executes the reference's own Python code and stores its outputs:

* ``snh_torch_single_tet.npz`` -- the reference's float64 PyTorch SNH
  formulation (``examples/backup/pytorch_energy_hessian_and_gradient/
  stable_neo_hookean.py``): its rest-invariant and energy functions are
  extracted from the script's syntax tree (the benchmark part of the script is
  not run) and differentiated with ``torch.autograd`` on the script's own
  single-tet rest/current positions and material (mu=2000, lam=1000).
* ``snh_sympy_six_tets.npz`` -- the reference's SymPy check script
  (``tests/energy/check_stable_neo_hookean.py``) run as-is; its assembled
  24x24 Hessian, gradient and energy over the six-tet cube fixture.
* ``cloth_torch.npz`` -- bending and Baraff-Witkin energies and gradients
  from the reference's float64 PyTorch scripts (``bending.py``,
  ``baraff_witkin.py`` in the same folder), see :func:`torch_cloth`.
* ``helpers_torch.npz`` -- the contact barriers, affine-body terms and the
  four lagged friction kinds from the reference's own formula code
  (``examples/dropping_in_container_mixed/helpers.py``,
  ``examples/dropping_in_container/friction_helpers.py``), run over a float64
  torch stand-in for the symbolic ``attribute`` class, see
  :func:`helper_energies`.
* ``mas_cpu_reference.npz`` -- the reference's NumPy MAS solver
  (``yasps/yasps/solver/mas``) on a small SNH + inertia system, with pymetis
  replaced by the chunk-ordering shim documented in ``oracle/mas.py`` (the
  reference's own BFS component split is used inside the shim).

Nothing in the test suite reads the reference checkout; the tests only read
the ``.npz`` files written here.
"""

from __future__ import annotations

import ast
import os
import runpy
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)


def torch_single_tet(ref):
  import torch
  path = os.path.join(ref, "examples/backup/pytorch_energy_hessian_and_gradient/stable_neo_hookean.py")
  tree = ast.parse(open(path).read())
  keep = []
  for node in tree.body:
    if isinstance(node, (ast.Import, ast.ImportFrom)):
      keep.append(node)
    elif isinstance(node, ast.FunctionDef) and node.name in ("precompute_rest_invariants",
                                                              "stable_neo_hookean_energy_precomp"):
      keep.append(node)
    elif isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id in (
        "rest_position_np", "current_position_np") for t in node.targets):
      keep.append(node)
  env = {}
  exec(compile(ast.Module(body=keep, type_ignores=[]), path, "exec"), env)
  torch.set_default_dtype(torch.float64)
  rest = torch.tensor(env["rest_position_np"])[None]
  cur = torch.tensor(env["current_position_np"])[None]
  mu, lam = torch.tensor(2000.0), torch.tensor(1000.0)
  ib, vol = env["precompute_rest_invariants"](rest)
  f = lambda flat: env["stable_neo_hookean_energy_precomp"](flat.reshape(1, 4, 3), ib, vol, mu, lam).sum()
  x = cur.reshape(12).clone().requires_grad_(True)
  e = f(x)
  (g,) = torch.autograd.grad(e, x)
  h = torch.autograd.functional.hessian(f, cur.reshape(12).clone())
  np.savez(os.path.join(HERE, "snh_torch_single_tet.npz"), rest=env["rest_position_np"],
           current=env["current_position_np"], mu=2000.0, lam=1000.0, energy=e.item(), grad=g.numpy(),
           hess=h.numpy(), ib=ib[0].numpy(), vol=vol[0].item())


def _extract(path, names, assigns=()):
  tree = ast.parse(open(path).read())
  keep = [n for n in tree.body if isinstance(n, (ast.Import, ast.ImportFrom)) or
          (isinstance(n, ast.FunctionDef) and n.name in names) or
          (isinstance(n, ast.Assign) and any(isinstance(t, ast.Name) and t.id in assigns for t in n.targets))]
  env = {}
  exec(compile(ast.Module(body=keep, type_ignores=[]), path, "exec"), env)
  return env


def torch_cloth(ref):
  """Bending and Baraff-Witkin from the reference's float64 PyTorch scripts
  (functions extracted from their syntax trees) on the scripts' own base
  element scaled by 1.54 plus seeded noise (stretched, so every stretch
  coefficient of the helper formula is 1).  The scripts add 1e-8 guards
  (axis norm, normal norm, 1 + cos), so they pin the formulas to ~1e-7."""
  import torch
  torch.set_default_dtype(torch.float64)
  base = os.path.join(ref, "examples/backup/pytorch_energy_hessian_and_gradient")
  gen = torch.Generator().manual_seed(7)
  out = {}
  env = _extract(os.path.join(base, "bending.py"), ("angle", "edgeTheta_from_x", "bending_energy_precomp"))
  pos = np.array([[0, 0, 1], [1, 0, 2], [0, 0, 0], [0, 2, 0]], dtype=np.float64)
  pos -= pos.mean(axis=0)
  rest = torch.tensor(pos)[None].expand(6, -1, -1).contiguous()
  x = (rest * 1.54 + 1e-2 * torch.randn((6, 4, 3), generator=gen)).requires_grad_(True)
  t0 = env["edgeTheta_from_x"](rest).detach()
  len0 = torch.norm(rest[:, 1, :] - rest[:, 0, :], dim=1)
  e = env["bending_energy_precomp"](x, t0, len0, torch.tensor(1000.0))
  (g,) = torch.autograd.grad(e.sum(), x)
  out.update(bend_rest=rest.numpy(), bend_x=x.detach().numpy(), bend_energy=e.detach().numpy(),
             bend_grad=g.numpy(), bend_stiff=1000.0)
  env = _extract(os.path.join(base, "baraff_witkin.py"), ("compute_rest_shape", "baraff_witkin_energy"))
  pos = np.array([[0, 0, 1], [1, 0, 2], [0, 0, 0]], dtype=np.float64)
  pos -= pos.mean(axis=0)
  rest = torch.tensor(pos)[None].expand(6, -1, -1).contiguous()
  x = (rest * 1.54 + 1e-2 * torch.randn((6, 3, 3), generator=gen)).requires_grad_(True)
  e = env["baraff_witkin_energy"](rest, x, torch.tensor(2000.0), torch.tensor(1000.0), 0.01, 1.0)
  (g,) = torch.autograd.grad(e.sum(), x)
  out.update(bw_rest=rest.numpy(), bw_x=x.detach().numpy(), bw_energy=e.detach().numpy(), bw_grad=g.numpy(),
             bw_params=np.array([2000.0, 1000.0, 0.01, 1.0]))
  np.savez(os.path.join(HERE, "cloth_torch.npz"), **out)


class TorchAttribute:
  """Float64 torch stand-in for the reference's symbolic ``attribute`` class
  (``yasps/yasps/attribute/attribute.pyx``), covering the operators its
  example energy helpers use: ``row``, indexing, ``+ - * /`` (``*`` is a
  matrix product unless one side is a scalar), ``dot``, ``cross``, ``norm``,
  ``log``, ``sqrt``, ``atan2``, ``transpose``, ``determinant``, ``inverse``,
  ``trace``, comparisons, and the static ``to_array``, ``identity`` and
  ``select``.  Values are 2-D tensors (a scalar is 1x1), so autograd
  differentiates the helpers exactly as written."""

  def __init__(self, value=None, float_value=None):
    import torch
    if float_value is not None:
      value = float(float_value)
    v = value if isinstance(value, torch.Tensor) else torch.tensor(value, dtype=torch.float64)
    if v.dim() == 0:
      v = v.reshape(1, 1)
    elif v.dim() == 1:
      v = v.reshape(1, -1)
    self.v = v

  @classmethod
  def wrap(cls, x):
    return x if isinstance(x, cls) else cls(x)

  def scalar(self):
    return self.v.numel() == 1

  def __add__(self, o):
    return TorchAttribute(self.v + TorchAttribute.wrap(o).v)

  __radd__ = __add__

  def __sub__(self, o):
    return TorchAttribute(self.v - TorchAttribute.wrap(o).v)

  def __rsub__(self, o):
    return TorchAttribute(TorchAttribute.wrap(o).v - self.v)

  def __neg__(self):
    return TorchAttribute(-self.v)

  def __mul__(self, o):
    o = TorchAttribute.wrap(o)
    if self.scalar() or o.scalar():
      return TorchAttribute(self.v * o.v)
    return TorchAttribute(self.v @ o.v)

  def __rmul__(self, o):
    return TorchAttribute.wrap(o) * self

  def __truediv__(self, o):
    return TorchAttribute(self.v / TorchAttribute.wrap(o).v)

  def __rtruediv__(self, o):
    return TorchAttribute(TorchAttribute.wrap(o).v / self.v)

  def __lt__(self, o):
    return TorchAttribute(self.v < TorchAttribute.wrap(o).v)

  def __gt__(self, o):
    return TorchAttribute(self.v > TorchAttribute.wrap(o).v)

  def row(self, i):
    return TorchAttribute(self.v[i:i + 1, :])

  def __getitem__(self, i):
    return TorchAttribute(self.v.reshape(-1)[i])

  def dot(self, o):
    return TorchAttribute((self.v.reshape(-1) * TorchAttribute.wrap(o).v.reshape(-1)).sum())

  def cross(self, o):
    import torch
    c = torch.linalg.cross(self.v.reshape(-1), TorchAttribute.wrap(o).v.reshape(-1))
    return TorchAttribute(c.reshape(self.v.shape))

  def norm(self):
    import torch
    return TorchAttribute(torch.linalg.norm(self.v))

  def log(self):
    return TorchAttribute(self.v.log())

  def sqrt(self):
    return TorchAttribute(self.v.sqrt())

  def atan2(self, o):
    import torch
    return TorchAttribute(torch.atan2(self.v, TorchAttribute.wrap(o).v))

  def transpose(self):
    return TorchAttribute(self.v.T)

  def determinant(self):
    import torch
    return TorchAttribute(torch.linalg.det(self.v))

  def inverse(self):
    import torch
    return TorchAttribute(torch.linalg.inv(self.v))

  def trace(self):
    return TorchAttribute(self.v.diagonal().sum())

  @staticmethod
  def to_array(values, rows, cols):
    import torch
    vs = [TorchAttribute.wrap(x).v.reshape(()) for x in values]
    return TorchAttribute(torch.stack(vs).reshape(rows, cols))

  @staticmethod
  def identity(n):
    import torch
    return TorchAttribute(torch.eye(n, dtype=torch.float64))

  @staticmethod
  def select(cond, a, b):
    import torch
    a, b = TorchAttribute.wrap(a), TorchAttribute.wrap(b)
    return TorchAttribute(torch.where(cond.v, a.v, b.v))


def _helpers(path, names):
  """Functions ``names`` of a reference helper module, run over the stand-in."""
  tree = ast.parse(open(path).read())
  keep = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
  env = {"attribute": TorchAttribute}
  exec(compile(ast.Module(body=keep, type_ignores=[]), path, "exec"), env)
  return env


def _ghess(f, flat):
  """Energy, gradient and Hessian of the scalar ``f`` at the flat input."""
  import torch
  x = flat.clone().requires_grad_(True)
  e = f(x)
  (g,) = torch.autograd.grad(e, x)
  h = torch.autograd.functional.hessian(f, flat.clone())
  return float(e.detach()), g.numpy(), h.numpy()


def _contact_configs(rng, kind, n, dhat):
  """Seeded element positions [n, A, 3] of a contact kind with the squared
  (line / plane) distance in (0.1, 0.9) dhat."""
  out = []
  for _ in range(n):
    d = np.sqrt(rng.uniform(0.1, 0.9) * dhat)
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    base = rng.normal(size=3) * 0.1
    if kind == "pp":
      x = np.array([[0, 0, 0], [0, 0, d]])
    elif kind == "pe":
      x = np.array([[0.3, 0, d], [0, 0, 0], [1.0, 0, 0]])
    elif kind == "pt":
      x = np.array([[0.25, 0.3, d], [0, 0, 0], [1.0, 0, 0], [0, 1.0, 0]])
    else:  # ee
      x = np.array([[-0.6, 0.1, 0], [0.7, -0.1, 0], [0.05, -0.5, d], [-0.1, 0.8, d]])
    x = x + rng.normal(size=x.shape) * 1e-3 * np.array([1.0, 1.0, 0.0])
    out.append(base + x @ q.T)
  return np.asarray(out)


def helper_energies(ref):
  """Barriers, orthogonality, inertia, SNH and lagged friction from the
  reference's own formula code, ``examples/dropping_in_container_mixed/
  helpers.py`` (``inertia``, ``point_point``, ``point_edge``,
  ``point_triangle``, ``edge_edge``, ``affine_energy``,
  ``stable_neo_hookean_modified``) and ``examples/dropping_in_container/
  friction_helpers.py`` (all four friction kinds with their lagged
  coordinates, tangent bases and ``lambda_last_h``), executed over
  :class:`TorchAttribute` and differentiated by autograd on seeded inputs.
  Affine bodies compose their positions as the reference scene does
  (``dropping_in_container_mixed/dropping_in_container.py:268-270`` for a
  vertex, ``:288-313`` for a tet)."""
  import torch
  torch.set_default_dtype(torch.float64)
  A = TorchAttribute
  rng = np.random.default_rng(2024)
  hp = _helpers(os.path.join(ref, "examples/dropping_in_container_mixed/helpers.py"),
                ("inertia", "point_point", "point_edge", "point_triangle", "edge_edge", "affine_energy",
                 "stable_neo_hookean_modified"))
  fp = _helpers(os.path.join(ref, "examples/dropping_in_container/friction_helpers.py"),
                {n for n in ("normalize", "scalar_zero", "lambda_last_h_rank2", "smooth_friction_phi",
                             "friction_energy_from_rel_dx")} |
                {f"{p}_{k}" for k in ("pp", "pe", "pt", "ee") for p in (
                    "closest_point_coord_and_tangent_basis", "distance2", "lambda_last_h", "rel_dx",
                    "friction_energy")} | {f"distance2_{k}_from_coord" for k in ("pp", "pe", "pt", "ee")})
  out = {}
  dhat, kappa = 1e-3, 1e4
  arity = {"pp": 2, "pe": 3, "pt": 4, "ee": 4}
  fname = {"pp": "point_point", "pe": "point_edge", "pt": "point_triangle", "ee": "edge_edge"}
  for k, a in arity.items():
    xs = _contact_configs(rng, k, 4, dhat)
    es, gs, hs = [], [], []
    for x in xs:
      f = lambda v: hp[fname[k]](A(v.reshape(a, 3)), dhat, kappa).v.reshape(())
      e, g, h = _ghess(f, torch.tensor(x.reshape(-1)))
      es.append(e); gs.append(g); hs.append(h)
    out.update({f"barrier_{k}_x": xs, f"barrier_{k}_energy": np.array(es), f"barrier_{k}_grad": np.array(gs),
                f"barrier_{k}_hess": np.array(hs)})
    # lagged friction: coordinates, tangent basis and lambda at x_old, energy at x
    # (tangential moves below and above the smoothing radius sqrt(fDhat) dt)
    fdt, rate = 0.01, 0.3
    es, gs, hs, lags, xn = [], [], [], [], []
    for t, x_old in enumerate(xs):
      step = (1e-6 if t % 2 == 0 else 1e-3) * rng.normal(size=x_old.shape)
      x_new = x_old + step
      old = A(torch.tensor(x_old))
      coord, basis = fp[f"closest_point_coord_and_tangent_basis_{k}"](old)
      lam = fp[f"lambda_last_h_{k}"](old, coord, A(dhat), kappa)
      coord, basis, lam = A(coord.v.detach()), A(basis.v.detach()), A(lam.v.detach())
      f = lambda v: fp[f"friction_energy_{k}"](A(v.reshape(a, 3)), old, A(dhat), fdt, rate, coord,
                                               basis.row(0), basis.row(1), lam).v.reshape(())
      e, g, h = _ghess(f, torch.tensor(x_new.reshape(-1)))
      es.append(e); gs.append(g); hs.append(h); xn.append(x_new)
      lags.append(np.concatenate([coord.v.reshape(-1).numpy(), basis.v.reshape(-1).numpy(), lam.v.reshape(-1).numpy()]))
    out.update({f"friction_{k}_x_old": xs, f"friction_{k}_x": np.array(xn), f"friction_{k}_energy": np.array(es),
                f"friction_{k}_grad": np.array(gs), f"friction_{k}_hess": np.array(hs),
                f"friction_{k}_lagged": np.array(lags)})
  out.update(barrier_params=np.array([dhat, kappa]), friction_params=np.array([dhat, 0.01, 0.3]))
  # affine bodies: q = (A row-major, t)
  qs = []
  for _ in range(4):
    rot, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    qs.append(np.concatenate([(rot @ (np.eye(3) + 0.05 * rng.normal(size=(3, 3)))).reshape(-1), rng.normal(size=3)]))
  qs = np.asarray(qs)
  ortho = [_ghess(lambda q: hp["affine_energy"](A(q[:9].reshape(3, 3))).v.reshape(()), torch.tensor(q)) for q in qs]
  xbar, xb, vel = rng.normal(size=(4, 3)), rng.normal(size=(4, 3)), rng.normal(size=(4, 3))
  mass, dt = 0.37, 0.01

  def inertia_q(q, i):
    pos = A(q[:9].reshape(3, 3)) * A(torch.tensor(xbar[i]).reshape(3, 1)) + A(q[9:12].reshape(3, 1))
    return hp["inertia"](A(torch.tensor(xb[i]).reshape(3, 1)), A(torch.tensor(vel[i]).reshape(3, 1)), dt, pos,
                         mass).v.reshape(())
  inert = [_ghess(lambda q: inertia_q(q, i), torch.tensor(qs[i])) for i in range(4)]
  rest = np.array([[0, 0, 0], [1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]]) * 0.2 + rng.normal(size=(4, 4, 3)) * 0.02
  mu, lam_ = 2000.0, 1000.0

  def snh_q(q, i):
    r = A(torch.tensor(rest[i]))
    t = q[9:12]
    pos = r * A(q[:9].reshape(3, 3)).transpose() + A(torch.stack([t] * 4))

    def edges(p):
      x0, x1, x2 = p.row(1) - p.row(0), p.row(2) - p.row(0), p.row(3) - p.row(0)
      return A.to_array([x0[0], x0[1], x0[2], x1[0], x1[1], x1[2], x2[0], x2[1], x2[2]], rows=3, cols=3)
    return hp["stable_neo_hookean_modified"](edges(pos), edges(r), mu, lam_, dt).v.reshape(())
  snh = [_ghess(lambda q: snh_q(q, i), torch.tensor(qs[i])) for i in range(4)]
  for name, res in (("orthogonality", ortho), ("inertia", inert), ("snh", snh)):
    out[f"affine_{name}_energy"] = np.array([r[0] for r in res])
    out[f"affine_{name}_grad"] = np.array([r[1] for r in res])
    out[f"affine_{name}_hess"] = np.array([r[2] for r in res])
  out.update(affine_q=qs, affine_xbar=xbar, affine_x_before=xb, affine_velocity=vel,
             affine_inertia_params=np.array([mass, dt, 0.0, -9.8, 0.0]), affine_rest=rest,
             affine_snh_params=np.array([mu, lam_, dt]))
  np.savez(os.path.join(HERE, "helpers_torch.npz"), **out)


def sympy_six_tets(ref):
  path = os.path.join(ref, "tests/energy/check_stable_neo_hookean.py")
  out = runpy.run_path(path, run_name="__golden__")
  np.savez(os.path.join(HERE, "snh_sympy_six_tets.npz"), vols=np.asarray(out["vols"], dtype=np.float64),
           ibs=np.asarray(out["IBS"], dtype=np.float64).reshape(-1, 3, 3),
           tet_positions=np.asarray(out["tet_positions"], dtype=np.float64).reshape(-1, 4, 3),
           indices=np.asarray(out["indices"], dtype=np.int64), mu=2000.0, lam=1000.0,
           energy=float(out["energy_sum"]), grad=np.asarray(out["gradient_sum"], dtype=np.float64),
           hess=np.asarray(out["sum_mat"], dtype=np.float64))


def mas_reference(ref):
  sys.path.insert(0, os.path.join(ref, "yasps/yasps/solver"))
  import mas
  from mas import hierarchy as mas_hierarchy
  from mas import metis as mas_metis
  from mas.matrix_view import BlockSparseMatrixView
  from oracle import energies, pattern, projection

  def chunk_order(graph, target_nodes_per_partition=16):
    if graph.node_count <= 1 or not graph.edges:
      order = np.arange(graph.node_count, dtype=np.int64)
      return mas_metis.OrderingResult(order, (tuple(map(int, order)),), "trivial", 0.0)
    groups = []
    for start in range(0, graph.node_count, target_nodes_per_partition):
      part = list(range(start, min(graph.node_count, start + target_nodes_per_partition)))
      groups.extend(mas_metis._component_bfs_groups(graph, part))
    groups.sort(key=min)
    order = np.asarray([n for g in groups for n in g], dtype=np.int64)
    return mas_metis.OrderingResult(order, tuple(tuple(map(int, g)) for g in groups), "chunk", 0.0)

  mas_hierarchy.metis_order = chunk_order

  # A 6x6x6 Morton-numbered cube, Kuhn six-tet split, SNH + inertia, z=0 pinned.
  from yasps_b200 import scenes
  sc = scenes.fem_cube(6, spacing=0.1, young=1e5, poisson=0.4, noise=0.01, seed=0)
  rhs, pat, values, n = _assemble_oracle(sc, energies, pattern, projection)
  counts = np.asarray(pat.category_counts, dtype=np.int64)
  view = BlockSparseMatrixView(
      rows=n, cols=n, variable_scalar_offsets=np.arange(0, n, 3), variable_dimensions=np.full(n // 3, 3),
      static_values=values, static_positions=pat.positions.astype(np.int64),
      static_category_starts=pat.category_starts[:-1].astype(np.int64), static_category_counts=counts,
      static_block_dimensions=pat.category_dims.astype(np.int64), symmetric_storage=True)
  solver = mas.MASSolver(max_domain_dofs=96, target_nodes_per_partition=32, inverse_backend="cpu_reference")
  iterations = solver.solve(view, rhs, tolerance=1e-12, max_iterations=500)
  h = solver.hierarchy
  np.savez(os.path.join(HERE, "mas_cpu_reference.npz"), rhs=rhs, values=values, positions=pat.positions,
           solution=solver.solution, iterations=iterations,
           relative_residual=solver.statistics.relative_residual,
           domains_per_level=np.asarray(h.domains_per_level), nodes_per_level=np.asarray(h.nodes_per_level),
           level0_domains=np.concatenate([np.asarray(d) for d in h.levels[0].domains]),
           level0_domain_sizes=np.asarray([len(d) for d in h.levels[0].domains]),
           composed_last=h.composed_node_maps[-1])


def _assemble_oracle(sc, energies, pattern, projection):
  """Gradient and upper block storage of the SNH + inertia scene (oracle)."""
  n = sc.free_count * 3
  codes, sizes = sc.snh_slots()
  perm, _, _ = pattern.compress_slots(codes, sizes)
  c1, d1, o1 = pattern.coordinates(codes, sizes, perm)
  icodes, isizes = sc.inertia_slots()
  iperm, _, _ = pattern.compress_slots(icodes, isizes)
  c2, d2, o2 = pattern.coordinates(icodes, isizes, iperm)
  pat = pattern.build_pattern([c1, c2], [d1, d2])
  x = sc.positions_all()[sc.tets]
  _, g, hh = energies.snh_from_rest(x, sc.rest_all()[sc.tets], sc.mu, sc.lam, sc.dt)
  hh = projection.project_spd(hh, 1)
  gl = np.zeros(n)
  values = np.zeros(pat.total_values)
  diag = np.zeros(n * 3)
  pattern.scatter_term(codes, sizes, perm, pat.lookups[0], o1, g, hh, gl, values, diag, [0, n], [0, 3 * n])
  _, gi, hi = energies.inertia_local(sc.free_positions(), sc.x_tilde(), sc.mass)
  pattern.scatter_term(icodes, isizes, iperm, pat.lookups[1], o2, gi, hi, gl, values, diag, [0, n], [0, 3 * n])
  return gl, pat, values, n


if __name__ == "__main__":
  ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("YASPS_REFERENCE", "")
  if not ref or not os.path.isdir(ref):
    raise SystemExit("usage: make_golden.py <reference checkout>")
  which = sys.argv[2:] or ["torch", "mas", "sympy", "cloth", "helpers"]
  if "torch" in which:
    torch_single_tet(ref)
  if "mas" in which:
    mas_reference(ref)
  if "sympy" in which:
    sympy_six_tets(ref)
  if "cloth" in which:
    torch_cloth(ref)
  if "helpers" in which:
    helper_energies(ref)
