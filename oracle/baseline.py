"""Timed CPU restatement of one Newton step (oracle; bench baseline only).

TEST AND CPU-BASELINE INFRASTRUCTURE ONLY -- used by ``bench.py``'s ``cpu_baseline``
and ``--impl reference`` legs.  It restates, vectorised with NumPy/SciPy,
the reference's CPU path for the step: SNH gradient/Hessian with the
reference's PSD-test + eigen projection rule, block assembly, the MAS
numeric update (dense domain matrices + FP64 inverse,
``PKG/solver/mas/numeric_assembly.py``, ``local_inverse.py:40-78``) and
MAS-preconditioned CG (``mas/pcg.py``, ``mas/preconditioner.py``) with the
chunk ordering of ``oracle/mas.py``.
"""

from __future__ import annotations

import os
import time

import numpy as np
import scipy.sparse as sp

from . import energies, projection


def system_from_cube(cube, tet_slice=slice(None)):
  """Vectorised oracle gradient + sparse Hessian (free DoFs) of the cube."""
  tets = cube.tets.astype(np.int64)[tet_slice]
  x = cube.positions_all()[tets]
  r = cube.rest_all()[tets]
  _, g, h = energies.snh_from_rest(x, r, cube.mu, cube.lam, cube.dt)
  h = projection.project_spd(h, 1)
  npin, n = cube.pinned_count, cube.dofs
  free = tets >= npin
  dof = np.where(free[:, :, None], 3 * (tets[:, :, None] - npin) + np.arange(3), -1).reshape(len(tets), 12)
  grad = np.zeros(n)
  m = dof >= 0
  np.add.at(grad, dof[m], g[m])
  rows = np.broadcast_to(dof[:, :, None], h.shape)
  cols = np.broadcast_to(dof[:, None, :], h.shape)
  keep = (rows >= 0) & (cols >= 0)
  H = sp.coo_matrix((h[keep], (rows[keep], cols[keep])), shape=(n, n)).tocsr()
  _, gi, hi = energies.inertia_local(cube.free_position, cube.x_tilde(), cube.mass)
  grad += gi.ravel()
  H = H + sp.diags(np.repeat(cube.mass, 3))
  return grad, H.tocsr()


class CpuMas:
  """MAS over chunk-ordered 32-node domains, assembled from a CSR matrix."""

  def __init__(self, H, nv, target=32, coarsest_weight=2.5, max_levels=6, max_dofs=96):
    from . import mas
    B = abs(H)
    B = sp.csr_matrix((np.ones(B.nnz), B.indices, B.indptr), shape=B.shape)
    node = sp.csr_matrix((np.ones(3 * nv), (np.arange(3 * nv), np.repeat(np.arange(nv), 3))), shape=(3 * nv, nv))
    G = (node.T @ B @ node).tocoo()
    edges = np.stack([G.row, G.col], axis=1)
    edges = edges[edges[:, 0] < edges[:, 1]]
    self.h = mas.build_hierarchy(np.full(nv, 3), [tuple(e) for e in edges], max_domain_dofs=max_dofs,
                                 max_levels=max_levels, target_nodes=target)
    L = len(self.h.levels)
    self.weights = (1.0,) * (L - 1) + (coarsest_weight,)
    self.nv = nv
    self.maps = []
    for lvl, cm in zip(self.h.levels, self.h.composed):
      P = sp.csr_matrix((np.ones(3 * nv), (np.arange(3 * nv), (3 * cm[:, None] + np.arange(3)).ravel())),
                        shape=(3 * nv, 3 * lvl.dims.size))
      self.maps.append(P)
    self.update(H)

  def update(self, H, domain_fraction=1.0):
    """Dense domain matrices + FP64 Cholesky inverses.

    With ``domain_fraction < 1`` only that fraction of the level-0 domains is
    processed; returns ``(seconds of the sampled level-0 domain work, seconds
    of everything else)`` so a caller can scale the former alone.
    """
    self.inverses = []
    t_sampled = t_rest = 0.0
    for li, (lvl, P) in enumerate(zip(self.h.levels, self.maps)):
      t0 = time.perf_counter()
      A = H if li == 0 else (P.T @ H @ P).tocsr()
      doms = lvl.domains
      if li == 0 and domain_fraction < 1.0:
        doms = doms[:max(1, int(len(doms) * domain_fraction))]
      t1 = time.perf_counter()
      invs = []
      for dom in doms:
        idx = (3 * np.asarray(dom)[:, None] + np.arange(3)).ravel()
        M = A[idx][:, idx].toarray()
        Lc = np.linalg.cholesky(0.5 * (M + M.T))
        Li = np.linalg.inv(Lc)
        invs.append((idx, Li.T @ Li))
      self.inverses.append(invs)
      t2 = time.perf_counter()
      if li == 0:
        t_sampled += t2 - t1
        t_rest += t1 - t0
      else:
        t_rest += t2 - t0
    return t_sampled, t_rest

  def apply(self, r):
    out = np.zeros_like(r)
    for li, (P, invs) in enumerate(zip(self.maps, self.inverses)):
      rl = P.T @ r
      zl = np.zeros_like(rl)
      for idx, inv in invs:
        zl[idx] = inv @ rl[idx]
      out += self.weights[li] * (P @ zl)
    return out


def pcg(H, g, M, tol, maxit):
  x = np.zeros_like(g)
  r = g.copy()
  z = M.apply(r)
  p = z.copy()
  rz = r @ z
  gn = np.linalg.norm(g)
  for it in range(1, maxit + 1):
    q = H @ p
    a = rz / (p @ q)
    x += a * p
    r -= a * q
    if np.linalg.norm(r) <= tol * gn:
      return x, it
    z = M.apply(r)
    rz2 = r @ z
    p = z + (rz2 / rz) * p
    rz = rz2
  return x, maxit


def assemble_chunked(cube, chunk=200_000):
  """Full CPU gradient + Hessian, element work in chunks (bounded memory)."""
  nt = cube.tet_count
  g, H = None, None
  for s in range(0, nt, chunk):
    gi, Hi = system_from_cube(cube, slice(s, min(nt, s + chunk)))
    g = gi if g is None else g + gi
    H = Hi if H is None else H + Hi
  # the inertia term was added once per chunk: keep one copy
  k = (nt + chunk - 1) // chunk
  if k > 1:
    _, gi, _ = energies.inertia_local(cube.free_position, cube.x_tilde(), cube.mass)
    g -= (k - 1) * gi.ravel()
    H = H - (k - 1) * sp.diags(np.repeat(cube.mass, 3))
  return g, H.tocsr()


_POOL_CUBE = None


def _pool_init(cube):
  global _POOL_CUBE
  _POOL_CUBE = cube


def _pool_chunk(bounds):
  return system_from_cube(_POOL_CUBE, slice(*bounds))


class ElementPool:
  """Worker processes (spawned: safe next to a CUDA context) that evaluate
  the element terms of the cube in chunks, so the CPU step uses every host
  core; created once, reused by every step."""

  def __init__(self, cube, workers=None):
    import concurrent.futures as cf
    import multiprocessing as mp
    self.workers = max(1, int(workers or os.cpu_count() or 1))
    self.cube = cube
    self.ex = cf.ProcessPoolExecutor(self.workers, mp_context=mp.get_context("spawn"), initializer=_pool_init,
                                     initargs=(cube,))
    # start and import in every worker (bounded: a worker that cannot start
    # raises instead of waiting forever)
    list(self.ex.map(_pool_chunk, [(0, 1)] * self.workers, timeout=300))

  def assemble(self):
    """Gradient + Hessian of the whole cube (chunks spread over the workers)."""
    nt = self.cube.tet_count
    step = max(1, (nt + 4 * self.workers - 1) // (4 * self.workers))
    chunks = [(s, min(nt, s + step)) for s in range(0, nt, step)]
    g, H = None, None
    for gi, Hi in self.ex.map(_pool_chunk, chunks, timeout=1800):
      g = gi if g is None else g + gi
      H = Hi if H is None else H + Hi
    k = len(chunks)
    if k > 1:  # the inertia term is in every chunk: keep one copy
      _, gi, _ = energies.inertia_local(self.cube.free_position, self.cube.x_tilde(), self.cube.mass)
      g -= (k - 1) * gi.ravel()
      H = H - (k - 1) * sp.diags(np.repeat(self.cube.mass, 3))
    return g, H.tocsr()

  def close(self):
    self.ex.shutdown()


def cpu_newton_step(cube, mas, tol=1e-6, maxit=1000, pool=None):
  """One whole, unsampled CPU Newton step of the cube (element evaluation,
  projection and assembly of every tetrahedron, the MAS numeric update of
  every domain, MAS-PCG to ``||g - H x|| <= tol ||g||``), timed phase by
  phase; the element phase runs on ``pool`` (an :class:`ElementPool`) when
  given.  ``mas`` carries the hierarchy (built once per structure, as the
  reference caches it) and is updated in place.  Returns
  ``(g, H, x, iterations, seconds_by_phase)``."""
  t0 = time.perf_counter()
  g, H = pool.assemble() if pool is not None else assemble_chunked(cube)
  t1 = time.perf_counter()
  mas.update(H)
  t2 = time.perf_counter()
  x, its = pcg(H, g, mas, tol, maxit)
  t3 = time.perf_counter()
  return g, H, x, its, dict(element_s=t1 - t0, mas_update_s=t2 - t1, pcg_s=t3 - t2, total_s=t3 - t0)


def prepare(cube, tol=1e-6, maxit=1000):
  """Untimed setup: the full CPU system, its MAS and the PCG iteration count."""
  g, H = assemble_chunked(cube)
  mas = CpuMas(H, cube.free_count)
  _, its = pcg(H, g, mas, tol, maxit)
  return g, H, mas, its


def timed_sample(cube, H, g, mas, iterations, sample_fraction=1.0 / 128, pcg_iterations=3):
  """Seconds of one CPU Newton step, measured on a bounded sample.

  Element evaluation (SNH + projection + assembly) on ``sample_fraction`` of
  the tetrahedra and the MAS numeric update on the same fraction of the
  level-0 domains are scaled up by that fraction; ``pcg_iterations`` full
  MAS-PCG iterations are scaled to ``iterations`` (the count a full CPU solve
  to the target residual takes, measured once by :func:`prepare`).
  """
  nt = cube.tet_count
  k = max(1, int(nt * sample_fraction))
  t0 = time.perf_counter()
  system_from_cube(cube, slice(0, k))
  t_elem = (time.perf_counter() - t0) * nt / k
  nd = len(mas.h.levels[0].domains)
  frac = max(1.0 / nd, sample_fraction)
  saved = mas.inverses
  t_sampled, t_rest = mas.update(H, domain_fraction=frac)
  t_mas = t_sampled / frac + t_rest
  mas.inverses = saved
  t0 = time.perf_counter()
  pcg(H, g, mas, 0.0, pcg_iterations)
  t_it = (time.perf_counter() - t0) / pcg_iterations
  total = t_elem + t_mas + t_it * iterations
  return total, dict(element_s=t_elem, mas_update_s=t_mas, pcg_iteration_s=t_it, iterations=int(iterations),
                     sample_fraction=sample_fraction)


def times_from_cube(cube, v, tet_slice=slice(None)):
  """Gradient and Hessian product ``H v`` (free DoFs) of the cube's SNH
  elements in ``tet_slice``, matrix-free (the same element terms and
  projection as :func:`system_from_cube`; inertia excluded)."""
  tets = cube.tets.astype(np.int64)[tet_slice]
  x = cube.positions_all()[tets]
  r = cube.rest_all()[tets]
  _, g, h = energies.snh_from_rest(x, r, cube.mu, cube.lam, cube.dt)
  h = projection.project_spd(h, 1)
  npin, n = cube.pinned_count, cube.dofs
  dof = np.where((tets >= npin)[:, :, None], 3 * (tets[:, :, None] - npin) + np.arange(3), -1).reshape(len(tets), 12)
  m = dof >= 0
  vl = np.where(m, np.asarray(v)[np.maximum(dof, 0)], 0.0)
  hv = np.einsum("tij,tj->ti", h, vl)
  grad, prod = np.zeros(n), np.zeros(n)
  np.add.at(grad, dof[m], g[m])
  np.add.at(prod, dof[m], hv[m])
  return grad, prod


_POOL_V = None


def _times_init(cube, v):
  global _POOL_CUBE, _POOL_V
  _POOL_CUBE, _POOL_V = cube, v


def _times_chunk(bounds):
  return times_from_cube(_POOL_CUBE, _POOL_V, slice(*bounds))


def relative_residual_pooled(cube, v, workers=None, chunk=250_000):
  """``||g - H v|| / ||g||`` of the cube's Newton system at ``v``, element
  terms matrix-free on spawned worker processes (safe next to a CUDA
  context), the inertia term added once."""
  import concurrent.futures as cf
  import multiprocessing as mp
  workers = max(1, int(workers or os.cpu_count() or 1))
  v = np.asarray(v, dtype=np.float64)
  nt = cube.tet_count
  chunks = [(s, min(nt, s + chunk)) for s in range(0, nt, chunk)]
  g, hv = np.zeros(cube.dofs), np.zeros(cube.dofs)
  with cf.ProcessPoolExecutor(min(workers, len(chunks)), mp_context=mp.get_context("spawn"),
                              initializer=_times_init, initargs=(cube, v)) as ex:
    for gi, hi in ex.map(_times_chunk, chunks, timeout=1800):
      g += gi
      hv += hi
  _, gi, _ = energies.inertia_local(cube.free_position, cube.x_tilde(), cube.mass)
  g += gi.ravel()
  hv += np.repeat(cube.mass, 3) * v
  return float(np.linalg.norm(g - hv) / np.linalg.norm(g))
