"""Multilevel additive Schwarz (MAS) preconditioner, FP64 NumPy (oracle only).

Restates the reference's CPU MAS path (``PKG/solver/mas``): hierarchy
construction (``hierarchy.py:150-271``), domain packing (``partition.py:41-73``),
compatible-node collapse (``hierarchy.py:105-147``), numeric assembly
(``numeric_assembly.py:64-83``), the FP64 Cholesky inverse oracle
(``local_inverse.py:40-78``) and the level-weighted application
(``preconditioner.py:26-154``).

Ordering: the reference orders every level with pymetis recursive
partitioning (``metis.py:42-90``; pymetis is an un-vendored dependency,
``yasps/setup.py:75-78``).  This oracle replaces only the partitioner by
*consecutive chunks of ``target_nodes`` node ids*; the reference's own
post-processing (split every part into BFS-connected components, order the
components by their smallest node) is kept.  With vertices numbered in
Morton order this yields the 32-vertex Morton domains the workloads ask for.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def _adjacency(node_count, edges):
  nbr = [[] for _ in range(node_count)]
  for i, j in edges:
    nbr[i].append(j)
    nbr[j].append(i)
  return [sorted(set(r)) for r in nbr]


def _edges_from_pairs(node_count, pairs):
  clean = {(min(int(i), int(j)), max(int(i), int(j))) for i, j in pairs if int(i) != int(j)}
  return sorted(clean)


def chunk_order_groups(node_count, edges, target_nodes):
  """Chunk partition + BFS component split (``metis.py:65-90`` post-processing)."""
  if node_count <= 1 or not edges:
    return [list(range(node_count))]
  adj = _adjacency(node_count, edges)
  groups = []
  for start in range(0, node_count, target_nodes):
    part = list(range(start, min(node_count, start + target_nodes)))
    allowed = set(part)
    remaining = set(part)
    while remaining:
      s = min(remaining)
      queue = [s]
      remaining.remove(s)
      cur = 0
      while cur < len(queue):
        node = queue[cur]
        cur += 1
        for nb in adj[node]:
          if nb in allowed and nb in remaining:
            remaining.remove(nb)
            queue.append(nb)
      groups.append(queue)
  groups.sort(key=min)
  return groups


def pack_domain_groups(groups, dims, max_dofs):
  """Greedy capacity packing inside each group (``partition.py:41-73``)."""
  domains = []
  for group in groups:
    cur, cur_dofs = [], 0
    for node in group:
      d = int(dims[node])
      if cur and cur_dofs + d > max_dofs:
        domains.append(cur)
        cur, cur_dofs = [], 0
      cur.append(node)
      cur_dofs += d
      if d > max_dofs:
        domains.append(cur)
        cur, cur_dofs = [], 0
    if cur:
      domains.append(cur)
  return domains


def collapse_compatible(node_count, edges, domains, dims, types):
  """Union-find collapse of equal-dimension neighbours in one domain (``hierarchy.py:105-147``)."""
  parent = np.arange(node_count)

  def find(n):
    while parent[n] != n:
      parent[n] = parent[parent[n]]
      n = int(parent[n])
    return n

  node_domain = np.full(node_count, -1)
  for d, dom in enumerate(domains):
    node_domain[dom] = d
  for a, b in edges:
    same_type = types is None or types[a] == types[b]
    if node_domain[a] == node_domain[b] and dims[a] == dims[b] and same_type:
      ra, rb = find(a), find(b)
      if ra != rb:
        parent[max(ra, rb)] = min(ra, rb)
  roots = [find(n) for n in range(node_count)]
  compact = {}
  mapping = np.empty(node_count, dtype=np.int64)
  for n, r in enumerate(roots):
    mapping[n] = compact.setdefault(r, len(compact))
  rep = np.empty(len(compact), dtype=np.int64)
  for r, c in compact.items():
    rep[c] = r
  return mapping, dims[rep].copy(), None if types is None else types[rep].copy()


@dataclass
class Level:
  dims: np.ndarray
  offsets: np.ndarray
  domains: list
  domain_offsets: list
  domain_sizes: np.ndarray
  order: list


@dataclass
class Hierarchy:
  levels: list
  composed: list


def _prefix(d):
  d = np.asarray(d, dtype=np.int64)
  return np.concatenate([[0], np.cumsum(d)[:-1]]).astype(np.int64)


def build_hierarchy(node_dims, edge_pairs, types=None, max_domain_dofs=96, max_levels=6, target_nodes=32,
                    global_coarse_domain=True) -> Hierarchy:
  """``build_hierarchy`` of ``hierarchy.py:150-271`` with the chunk ordering."""
  dims = np.asarray(node_dims, dtype=np.int64).copy()
  types = None if types is None else np.asarray(types).copy()
  node_count = dims.size
  edges = _edges_from_pairs(node_count, edge_pairs)
  levels, composed, seen = [], [np.arange(node_count, dtype=np.int64)], set()
  while len(levels) < max_levels:
    sig = (tuple(dims.tolist()), tuple(edges))
    if sig in seen:
      break
    seen.add(sig)
    groups = chunk_order_groups(node_count, edges, target_nodes)
    domains = pack_domain_groups(groups, dims, max_domain_dofs)
    doffs = [_prefix(dims[np.asarray(d)]) for d in domains]
    dsz = np.asarray([int(dims[np.asarray(d)].sum()) for d in domains], dtype=np.int64)
    levels.append(Level(dims.copy(), _prefix(dims), domains, doffs, dsz, [n for g in groups for n in g]))
    if len(levels) >= max_levels or node_count <= 1 or not edges:
      break
    mapping, cdims, ctypes = collapse_compatible(node_count, edges, domains, dims, types)
    if cdims.size == node_count:
      break
    composed.append(mapping[composed[-1]])
    cedges = _edges_from_pairs(cdims.size, ((mapping[a], mapping[b]) for a, b in edges))
    if (tuple(cdims.tolist()), tuple(cedges)) == sig:
      break
    dims, types, edges, node_count = cdims, ctypes, cedges, cdims.size
  last = levels[-1]
  if global_coarse_domain and int(last.dims.sum()) <= max_domain_dofs and len(last.domains) > 1:
    order = list(last.order)
    last.domains = [order]
    last.domain_offsets = [_prefix(last.dims[np.asarray(order)])]
    last.domain_sizes = np.asarray([int(last.dims.sum())], dtype=np.int64)
  return Hierarchy(levels, composed[:len(levels)])


def level_local_matrices(h: Hierarchy, fine_blocks):
  """Dense domain matrices of every level (``numeric_assembly.py:14-83``).

  ``fine_blocks`` yields ``(row_node, col_node, block)`` of the upper storage;
  off-diagonal blocks also contribute their transpose.
  """
  out = []
  for li, (lvl, cmap) in enumerate(zip(h.levels, h.composed)):
    node_dom = np.full(lvl.dims.size, -1)
    node_loc = np.zeros(lvl.dims.size, dtype=np.int64)
    for d, (dom, offs) in enumerate(zip(lvl.domains, lvl.domain_offsets)):
      node_dom[dom] = d
      node_loc[dom] = offs
    mats = [np.zeros((s, s)) for s in lvl.domain_sizes]
    for rn, cn, b in fine_blocks:
      for (a, c, blk) in ((rn, cn, b), (cn, rn, b.T)) if rn != cn else ((rn, cn, b),):
        pa, pc = cmap[a], cmap[c]
        if node_dom[pa] == node_dom[pc]:
          d = node_dom[pa]
          r0, c0 = node_loc[pa], node_loc[pc]
          mats[d][r0:r0 + blk.shape[0], c0:c0 + blk.shape[1]] += blk
    out.append(mats)
  return out


def cholesky_inverse(m: np.ndarray, pivot_tolerance=1e-12) -> np.ndarray:
  """FP64 inverse oracle (``local_inverse.py:40-78``, ``require_spd``)."""
  sym = 0.5 * (m + m.T)
  scale = max(1.0, float(np.linalg.norm(sym, ord=np.inf)))
  if not np.allclose(m, m.T, rtol=1e-12, atol=pivot_tolerance * scale):
    raise np.linalg.LinAlgError("domain is not symmetric")
  l = np.linalg.cholesky(sym)
  if np.min(np.diag(l)) ** 2 <= pivot_tolerance * scale:
    raise np.linalg.LinAlgError("numerically zero Cholesky pivot")
  eye = np.eye(m.shape[0])
  return np.linalg.solve(l.T, np.linalg.solve(l, eye))


class MASPreconditioner:
  """Level-weighted additive Schwarz application (``preconditioner.py:26-154``)."""

  def __init__(self, h: Hierarchy, local_matrices, coarsest_level_weight=2.5, level_weights=None):
    self.h = h
    nl = len(h.levels)
    self.weights = ((1.0,) * max(0, nl - 1) + (float(coarsest_level_weight),)
                    if level_weights is None else tuple(level_weights))
    self.inverses = [[cholesky_inverse(m) for m in mats] for mats in local_matrices]
    fine = h.levels[0]
    self.scalar_maps = []
    for lvl, cmap in zip(h.levels, h.composed):
      smap = np.empty(int(fine.dims.sum()), dtype=np.int64)
      for node, parent in enumerate(cmap):
        d = int(fine.dims[node])
        smap[fine.offsets[node]:fine.offsets[node] + d] = lvl.offsets[parent] + np.arange(d)
      self.scalar_maps.append(smap)

  def apply(self, r: np.ndarray) -> np.ndarray:
    r = np.asarray(r, dtype=np.float64)
    out = np.zeros_like(r)
    for li, (lvl, smap, invs) in enumerate(zip(self.h.levels, self.scalar_maps, self.inverses)):
      n = int(lvl.dims.sum())
      rl = r if li == 0 else np.bincount(smap, weights=r, minlength=n)
      corr = np.zeros(n)
      for dom, offs, inv in zip(lvl.domains, lvl.domain_offsets, invs):
        idx = np.concatenate([lvl.offsets[node] + np.arange(lvl.dims[node]) for node in dom])
        corr[idx] = inv @ rl[idx]
      out += self.weights[li] * (corr if li == 0 else corr[smap])
    return out
