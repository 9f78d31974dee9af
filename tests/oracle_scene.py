"""Oracle assembly of a FEM cube (test helper; the CPU checker of the GPU path)."""

import numpy as np

from oracle import energies, pattern, projection


class OracleCube:
  """Gradient, pattern, block values and diagonal blocks of the SNH + inertia
  cube, assembled by the oracle in the reference's term order (SNH, inertia)."""

  def __init__(self, c, projection_method=1):
    n = c.dofs
    self.n = n
    codes, sizes = c.snh_slots()
    perm, _, _ = pattern.compress_slots(codes, sizes)
    c1, d1, o1 = pattern.coordinates(codes, sizes, perm)
    icodes, isizes = c.inertia_slots()
    iperm, _, _ = pattern.compress_slots(icodes, isizes)
    c2, d2, o2 = pattern.coordinates(icodes, isizes, iperm)
    self.coords = [c1, c2]
    self.pattern = pattern.build_pattern([c1, c2], [d1, d2])
    x = c.positions_all()[c.tets.astype(np.int64)]
    r = c.rest_all()[c.tets.astype(np.int64)]
    self.energy_snh, g, h = energies.snh_from_rest(x, r, c.mu, c.lam, c.dt)
    self.raw_hess = h
    h = projection.project_spd(h, projection_method) if projection_method >= 1 else h
    self.gradient = np.zeros(n)
    self.values = np.zeros(self.pattern.total_values)
    self.diag_blocks = np.zeros(3 * n)
    pattern.scatter_term(codes, sizes, perm, self.pattern.lookups[0], o1, g, h, self.gradient, self.values,
                         self.diag_blocks, [0, n], [0, 3 * n])
    self.energy_inertia, gi, hi = energies.inertia_local(c.free_position, c.x_tilde(), c.mass)
    pattern.scatter_term(icodes, isizes, iperm, self.pattern.lookups[1], o2, gi, hi, self.gradient, self.values,
                         self.diag_blocks, [0, n], [0, 3 * n])
    self.psd = projection.is_psd_reference(self.raw_hess)

  def matvec(self, x):
    return pattern.spmv(self.pattern, self.values, x)

  def dense(self):
    return pattern.dense_from_blocks(self.pattern, self.values, self.n)
