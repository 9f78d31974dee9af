"""The oracle against the reference's own outputs (committed fixtures).

The fixtures were produced by ``tests/golden/make_golden.py`` from the
reference's PyTorch SNH formulation, its SymPy check script and its NumPy MAS
solver; these tests pin the CPU restatement the GPU parity tests rely on.
"""

import os

import numpy as np
import pytest

from oracle import energies, mas, pattern, projection, solvers

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
  return np.load(os.path.join(GOLDEN, name))


def test_snh_matches_reference_torch_single_tet():
  d = _load("snh_torch_single_tet.npz")
  e, g, h = energies.snh_from_rest(d["current"][None], d["rest"][None], d["mu"], d["lam"], 1.0)
  assert abs(e[0] - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))
  assert np.abs(g[0] - d["grad"]).max() <= 1e-12 * np.abs(d["grad"]).max()
  assert np.abs(h[0] - d["hess"]).max() <= 1e-12 * np.abs(d["hess"]).max()
  ib, vol = energies.snh_rest_invariants(d["rest"][None])
  np.testing.assert_allclose(ib[0], d["ib"], rtol=1e-13, atol=1e-13)
  assert abs(vol[0] - float(d["vol"])) <= 1e-14


def test_snh_matches_reference_sympy_six_tet_cube():
  d = _load("snh_sympy_six_tets.npz")
  e, g, h = energies.snh_local(d["tet_positions"], d["ibs"], d["vols"], d["mu"], d["lam"], 1.0)
  G, Hd = np.zeros(24), np.zeros((24, 24))
  for t, idx in enumerate(d["indices"]):
    dof = (3 * idx[:, None] + np.arange(3)).ravel()
    G[dof] += g[t]
    Hd[np.ix_(dof, dof)] += h[t]
  assert np.abs(G - d["grad"]).max() <= 1e-12 * np.abs(d["grad"]).max()
  assert np.abs(Hd - d["hess"]).max() <= 1e-12 * np.abs(d["hess"]).max()


def test_mas_matches_reference_cpu_solver():
  d = _load("mas_cpu_reference.npz")
  pos, vals, rhs = d["positions"], d["values"], d["rhs"]
  pat = pattern.build_pattern([pos], [np.full_like(pos, 3)])
  assert np.array_equal(pat.positions, pos)
  edges = [(r // 3, c // 3) for r, c in pos if r != c]
  h = mas.build_hierarchy(np.full(rhs.size // 3, 3), edges)
  assert [len(l.domains) for l in h.levels] == d["domains_per_level"].tolist()
  assert [l.dims.size for l in h.levels] == d["nodes_per_level"].tolist()
  assert np.array_equal(np.concatenate([np.asarray(x) for x in h.levels[0].domains]), d["level0_domains"])
  assert np.array_equal(h.composed[-1], d["composed_last"])
  blocks = [(r // 3, c // 3, vals[o:o + 9].reshape(3, 3)) for (r, c), o in zip(pat.positions, pat.value_offsets)]
  pre = mas.MASPreconditioner(h, mas.level_local_matrices(h, blocks))
  res = solvers.mas_pcg(lambda v: pattern.spmv(pat, vals, v), rhs, pre.apply, 1e-12, 500)
  assert res.iterations == int(d["iterations"])
  assert np.abs(res.solution - d["solution"]).max() <= 1e-10 * np.abs(d["solution"]).max()


def test_psd_test_rule_on_known_matrices():
  a = np.diag([3.0, 2.0, 0.0, 1.0])
  assert projection.is_psd_reference(a)
  b = a.copy()
  b[2, 2] = -1e-3
  assert not projection.is_psd_reference(b)
  # within the 1e-10 * scale tolerance counts as PSD
  c = a.copy()
  c[2, 2] = -1e-11
  assert projection.is_psd_reference(c)
  # a zero pivot with a nonzero remaining column is not PSD
  d = np.array([[0.0, 1.0], [1.0, 1.0]])
  assert not projection.is_psd_reference(d)


@pytest.mark.parametrize("method", [1, 2])
def test_projection_matches_eigen_rule(method):
  rng = np.random.default_rng(3)
  q, _ = np.linalg.qr(rng.normal(size=(12, 12)))
  w = np.linspace(-2.0, 3.0, 12)
  a = (q * w) @ q.T
  p = projection.project_spd(a, method)
  wp = np.abs(w) if method == 1 else np.maximum(w, 0.0)
  np.testing.assert_allclose(p, (q * wp) @ q.T, atol=1e-12)


def test_diagonal_pseudo_inverse_rule():
  q, _ = np.linalg.qr(np.random.default_rng(1).normal(size=(3, 3)))
  w = np.array([2.0, -4.0, 1e-8])
  blk = (q * w) @ q.T
  inv = projection.diagonal_block_pseudo_inverse(blk[None])[0]
  np.testing.assert_allclose(inv, (q * np.array([0.5, 0.25, 1e-8])) @ q.T, atol=1e-12)


def _close(a, b, tol=1e-12):
  a, b = np.asarray(a), np.asarray(b)
  return float(np.abs(a - b).max()) <= tol * max(float(np.abs(b).max()), 1e-300)


BARRIERS = {"pp": 1, "pe": 2, "pt": 3, "ee": 4}
FRICTIONS = {"pt": 8, "pe": 9, "ee": 10, "pp": 11}


@pytest.mark.parametrize("kind", sorted(BARRIERS))
def test_barriers_match_reference_helpers(kind):
  """``point_point`` / ``point_edge`` / ``point_triangle`` / ``edge_edge`` of
  ``examples/dropping_in_container_mixed/helpers.py`` (fixtures from the
  reference's code over a float64 stand-in of its ``attribute`` class)."""
  from oracle import vertex_energies as ve
  d = _load("helpers_torch.npz")
  x = d[f"barrier_{kind}_x"]
  e, g, h = ve.energy_grad_hess(BARRIERS[kind], x, None, tuple(d["barrier_params"]))
  assert _close(e, d[f"barrier_{kind}_energy"])
  assert _close(g, d[f"barrier_{kind}_grad"])
  assert _close(h, d[f"barrier_{kind}_hess"])


@pytest.mark.parametrize("kind", sorted(FRICTIONS))
def test_lagged_friction_matches_reference_helpers(kind):
  """The lagged coordinates, tangent basis and lambda at the last positions
  and the friction energy at the current ones, for the four kinds of
  ``examples/dropping_in_container/friction_helpers.py``; half of the cases
  move less than the smoothing radius, half more."""
  from oracle import vertex_energies as ve
  d = _load("helpers_torch.npz")
  dhat, kappa = d["barrier_params"]
  x_old, x = d[f"friction_{kind}_x_old"], d[f"friction_{kind}_x"]
  k = FRICTIONS[kind]
  lagged = np.stack([ve.LAGGED[k](xo, dhat, kappa) for xo in x_old])
  assert _close(lagged, d[f"friction_{kind}_lagged"])
  e, g, h = ve.energy_grad_hess(k, x, x_old, tuple(d["friction_params"]), lagged)
  assert _close(e, d[f"friction_{kind}_energy"])
  assert _close(g, d[f"friction_{kind}_grad"])
  assert _close(h, d[f"friction_{kind}_hess"])


def test_affine_terms_match_reference_helpers():
  """``affine_energy``, ``inertia`` of ``A xbar + t`` and
  ``stable_neo_hookean_modified`` of a tet at ``xbar A^T + t`` (the
  reference scene's compositions), differentiated in the body coordinates."""
  from oracle import affine_energies as ae
  d = _load("helpers_torch.npz")
  q = d["affine_q"]
  e, g, h = ae.grad_hess(ae.orthogonality, q, np.zeros((len(q), 1)), 1.0)
  assert _close(e, d["affine_orthogonality_energy"]) and _close(g, d["affine_orthogonality_grad"])
  assert _close(h, d["affine_orthogonality_hess"])
  mass, dt, *grav = d["affine_inertia_params"]
  data = np.concatenate([d["affine_xbar"], d["affine_x_before"], d["affine_velocity"],
                         np.full((len(q), 1), mass)], axis=1)
  e, g, h = ae.grad_hess(ae.inertia, q, data, (dt, *grav))
  assert _close(e, d["affine_inertia_energy"]) and _close(g, d["affine_inertia_grad"])
  assert _close(h, d["affine_inertia_hess"])
  e, g, h = ae.grad_hess(ae.snh, q, d["affine_rest"].reshape(len(q), 12), tuple(d["affine_snh_params"]))
  assert _close(e, d["affine_snh_energy"]) and _close(g, d["affine_snh_grad"])
  assert _close(h, d["affine_snh_hess"])
