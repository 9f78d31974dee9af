"""Known-answer tests of the assembly semantics, ported from the reference's
``tests/differentiator/test_hessian_sparsity_permutation_gpu.py``.

The reference builds its energies symbolically (quadratic energies of linear
boundary maps, ``:17-50``) and checks the assembled blocks, gradient,
diagonal blocks, SpMV and solves against small dense NumPy expectations at
3e-11 (solves at 2e-8).  Here the same seeded local Hessians and gradients
(``J^T P(H_in) J``, ``J^T (H_in (J x + o) + l)``) are scattered with the
oracle's restatement of the reference scatter (slot codes, local
compression, coordinates, pattern, NoProject merge) and compared with the
same dense expectations.  Ported: the interlaced / connected / zero-axes
permutation cases with repeated vertices (``:105-190``) and the mixed target
dimensions with global offsets (``:193-227``).  Not ported (they exercise the
reference's symbolic separate-Jacobian mode and its nonlinear fallback,
outside the fixed-energy path): ``:230-319``.
"""

import numpy as np
import pytest

from oracle import pattern, solvers

TOL = 3e-11


def inner_matrix(size):
  rng = np.random.default_rng(209 + size)
  basis, _ = np.linalg.qr(rng.normal(size=(size, size)))
  return (basis * np.linspace(-1.7, 3.1, size)) @ basis.T


def project(m, method):
  if method < 1:
    return m
  w, v = np.linalg.eigh(m)
  w = np.abs(w) if method == 1 else np.maximum(w, 0.0)
  return (v * w) @ v.T


def permutation_case(kind, method):
  """Local data of the reference's permutation test (2-DoF vertices, 4 per instance)."""
  values = np.sin(np.arange(134) * 0.17).reshape(-1, 2)
  if kind != "connected":
    jac = np.array([[0.3, 0, 0, -0.7, 0, 0, 1.1, 0], [0, 0.6, 0, 0, 0.8, 0, 0, -0.4], [0, 0, 1.2, 0, 0, -0.9, 0, 0],
                    [-0.8, 0, 0, 0.4, 0, 0, 0.5, 0], [0, 1.1, 0, 0, -0.2, 0, 0, 0.7]])
    if kind == "zero_axes":
      jac[4, :] = 0.0
      jac[:, 7] = 0.0
  else:
    jac = np.arange(32, dtype=np.float64).reshape(4, 8) / 41.0 + 0.13
  offset = np.zeros(len(jac))
  if kind == "zero_axes":
    offset[4] = 0.15
  h_in = inner_matrix(len(jac))
  lin = np.linspace(-0.3, 0.4, len(jac))
  conn = np.array([[3, 1, 5, 0], [1, 1, 2, 0], [0, 2, 0, 2], [5, 5, 5, 5]] +
                  [[i, (i + 1) % 67, (i + 9) % 67, (i + 3) % 67] for i in range(67)], dtype=np.int64)
  local_h = jac.T @ project(h_in, method) @ jac
  hs, gs = [], []
  exp_h = np.zeros((values.size, values.size))
  exp_g = np.zeros(values.size)
  for c in conn:
    idx = (2 * c[:, None] + np.arange(2)).ravel()
    b = jac @ values[c].ravel() + offset
    g = jac.T @ (h_in @ b + lin)
    np.add.at(exp_h, (idx[:, None], idx[None, :]), local_h)
    np.add.at(exp_g, idx, g)
    hs.append(local_h)
    gs.append(g)
  codes = 2 + 2 * conn
  sizes = np.full_like(codes, 2)
  return codes, sizes, np.asarray(gs), np.asarray(hs), exp_h, exp_g, values.size, [(len(values), 2)]


def mixed_dims_case(restrict):
  """The reference's mixed target dimensions case: attributes b (3) then a (2)."""
  a = np.linspace(-0.7, 0.6, 14).reshape(-1, 2)
  b = np.linspace(0.5, -0.4, 21).reshape(-1, 3)
  jac = np.array([[0.2, 0, -0.4, 0, 0], [0, 0.7, 0, -0.3, 0.6], [0.9, 0, 0.8, 0, 0], [0, -0.2, 0, 0.5, 0.4]])
  h_in = inner_matrix(4)
  lin = np.linspace(0.1, -0.2, 4)
  exp_h = np.zeros((35, 35))
  exp_g = np.zeros(35)
  codes, hs, gs = [], [], []
  # reference local order [a0, b0, b1, a1, b2] -> slot order [a (2), b (3)]
  order = np.array([0, 3, 1, 2, 4])
  for t in range(7):
    i = 6 - t  # the terms connect to the vertices in reverse order
    idx = np.array([21 + 2 * i, 3 * i, 3 * i + 1, 21 + 2 * i + 1, 3 * i + 2])
    local = np.array([a[i, 0], b[i, 0], b[i, 1], a[i, 1], b[i, 2]])
    d = jac.copy()
    if restrict:
      d[:, [1, 2, 4]] = 0.0
    lh = d.T @ project(h_in, 1) @ d
    lg = d.T @ (h_in @ (jac @ local) + lin)
    np.add.at(exp_h, (idx[:, None], idx[None, :]), lh)
    np.add.at(exp_g, idx, lg)
    codes.append([2 + 21 + 2 * i, 1 if restrict else 2 + 3 * i])
    hs.append(lh[np.ix_(order, order)])
    gs.append(lg[order])
  codes = np.asarray(codes)
  sizes = np.tile([2, 3], (7, 1))
  return codes, sizes, np.asarray(gs), np.asarray(hs), exp_h, exp_g, 35, [(7, 3), (7, 2)]


def oracle_assemble(codes, sizes, gs, hs, n, shapes):
  perm, _, _ = pattern.compress_slots(codes, sizes)
  c, d, o = pattern.coordinates(codes, sizes, perm)
  pat = pattern.build_pattern([c], [d])
  grad = np.zeros(n)
  values = np.zeros(pat.total_values)
  seg = np.cumsum([0] + [cnt * s for cnt, s in shapes])
  dstart = np.cumsum([0] + [cnt * s * s for cnt, s in shapes])
  diag = np.zeros(dstart[-1])
  pattern.scatter_term(codes, sizes, perm, pat.lookups[0], o, gs, hs, grad, values, diag, seg, dstart)
  return pat, values, grad, diag


def expected_diag(exp_h, shapes):
  out, off = [], 0
  for cnt, s in shapes:
    for i in range(cnt):
      st = off + i * s
      out.extend(exp_h[st:st + s, st:st + s].ravel())
    off += cnt * s
  return np.asarray(out)


CASES = [("perm", k, m) for k, m in (("interlaced", -1), ("interlaced", 1), ("interlaced", 2), ("connected", 1),
                                     ("zero_axes", 1))] + [("mixed", r, None) for r in (False, True)]


def build(case):
  if case[0] == "perm":
    return permutation_case(case[1], case[2])
  return mixed_dims_case(case[1])


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-{c[1]}-{c[2]}" for c in CASES])
def test_assembly_matches_reference_dense(case):
  codes, sizes, gs, hs, exp_h, exp_g, n, shapes = build(case)
  pat, values, grad, diag = oracle_assemble(codes, sizes, gs, hs, n, shapes)
  dense = pattern.dense_from_blocks(pat, values, n)
  assert np.allclose(dense, exp_h, rtol=TOL, atol=TOL)
  assert np.allclose(grad, exp_g, rtol=TOL, atol=TOL)
  assert np.allclose(diag, expected_diag(exp_h, shapes), rtol=TOL, atol=TOL)
  x = np.linspace(-0.8, 0.9, n)
  assert np.allclose(pattern.spmv(pat, values, x), exp_h @ x, rtol=TOL, atol=TOL)


def test_regularised_solves_match_dense_solution():
  """The projection-1 case plus 0.25 |x|^2 per vertex, solved by the oracle's
  block-Jacobi PCG to the reference's squared tolerance 1e-18 (``:170-190``)."""
  codes, sizes, gs, hs, exp_h, exp_g, n, shapes = permutation_case("interlaced", 1)
  pat, values, grad, _ = oracle_assemble(codes, sizes, gs, hs, n, shapes)
  reg = 0.5 * np.eye(n)
  matvec = lambda v: pattern.spmv(pat, values, v) + 0.5 * v
  full = exp_h + reg
  rhs = np.cos(np.arange(n) * 0.23)
  blocks = np.stack([full[2 * i:2 * i + 2, 2 * i:2 * i + 2] for i in range(n // 2)]).ravel()
  inv = solvers.diagonal_inverse(blocks, [n // 2], [2])
  res = solvers.jacobi_pcg(matvec, rhs, inv, [n // 2], [2], 1e-18, 1000)
  exact = np.linalg.solve(full, rhs)
  assert res.status >= 0
  assert np.allclose(res.solution, exact, rtol=2e-8, atol=2e-8)
  assert np.linalg.norm(full @ res.solution - rhs) / np.linalg.norm(rhs) < 2e-8
