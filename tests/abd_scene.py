"""Oracle assembly of the soft-cube + affine-bodies scene (test helper).

``yasps_b200.scenes.affine_scene`` builds the scene through the public API;
``oracle_assembly`` assembles the same terms with the oracle in the
reference's layout: the affine matrix of a body is ONE slot of size 9 (its
pattern has 9x9 / 9x3 / 3x3 blocks), the translation a slot of size 3.  The
device splits A into three 3-DoF rows, so the two are compared as dense
matrices, gradients and per-variable diagonal blocks.
"""

import numpy as np

from oracle import affine_energies as ae
from oracle import energies as oe
from oracle import pattern, projection


def oracle_assembly(cube, bodies, projection_method=1):
  """(dense H, gradient, diagonal blocks, energy total, [attribute segment starts])."""
  nf, nb = cube.free_count, bodies.num_bodies
  start_a = 3 * nf
  start_t = start_a + 9 * nb
  n = start_t + 3 * nb
  terms = []  # (codes, sizes, local g, local H)
  # soft SNH (union path [pinned, free], 12x12 projected) and inertia
  codes, sizes = cube.snh_slots()
  e_snh, g, h = oe.snh_from_rest(cube.positions_all()[cube.tets.astype(np.int64)],
                                 cube.rest_all()[cube.tets.astype(np.int64)], cube.mu, cube.lam, cube.dt)
  if projection_method >= 1:
    h = projection.project_spd(h, projection_method)
  terms.append((codes, sizes, g, h))
  e_in, gi, hi = oe.inertia_local(cube.free_position, cube.x_tilde(), cube.mass)
  terms.append((*cube.inertia_slots(), gi, hi))
  # affine bodies: coordinates q = [A row-major (9), t (3)] per body
  q = np.concatenate([bodies.affine, bodies.translation], axis=1)
  vb = bodies.vertex_body.astype(np.int64)
  tb = vb[bodies.tets.astype(np.int64)[:, 0]]
  body_codes = lambda b: np.stack([start_a + 9 * b + 2, start_t + 3 * b + 2], axis=1)
  body_sizes = lambda m: np.tile(np.array([9, 3]), (m, 1))
  rest_t = bodies.rest[bodies.tets.astype(np.int64)].reshape(-1, 12)
  e_as, g, h = ae.snh_projected(q[tb], rest_t, (bodies.mu, bodies.lam, cube.dt), projection_method)
  terms.append((body_codes(tb), body_sizes(tb.size), g, h))
  x_before = bodies.positions()
  data = np.concatenate([bodies.rest, x_before, bodies.velocity, bodies.mass[:, None]], axis=1)
  e_ai, g, h = ae.grad_hess(ae.inertia, q[vb], data, (cube.dt, *bodies.gravity))
  terms.append((body_codes(vb), body_sizes(vb.size), g, h))
  e_ao, g, h = ae.grad_hess(ae.orthogonality, q[:, :9], np.zeros((nb, 1)), bodies.stiffness, size=9)
  h = projection.project_spd(h, 2)
  bi = np.arange(nb)
  terms.append(((start_a + 9 * bi + 2)[:, None], np.full((nb, 1), 9), g, h))
  coords, dims, per = [], [], []
  for codes, sizes, g, h in terms:
    perm, _, _ = pattern.compress_slots(codes, sizes)
    c, d, o = pattern.coordinates(codes, sizes, perm)
    coords.append(c)
    dims.append(d)
    per.append((codes, sizes, perm, o, g, h))
  pat = pattern.build_pattern(coords, dims)
  seg = [0, start_a, start_t, n]
  dstart = [0, 9 * nf, 9 * nf + 81 * nb, 9 * nf + 81 * nb + 9 * nb]
  grad, values, diag = np.zeros(n), np.zeros(pat.total_values), np.zeros(dstart[-1])
  for k, (codes, sizes, perm, o, g, h) in enumerate(per):
    pattern.scatter_term(codes, sizes, perm, pat.lookups[k], o, g, h, grad, values, diag, seg, dstart)
  dense = pattern.dense_from_blocks(pat, values, n)
  energy = sum(float(np.sum(e)) for e in (e_snh, e_in, e_as, e_ai, e_ao))
  return dense, grad, diag, energy, pat
