"""MAS hierarchy construction (host, once per static structure).

Restates ``build_hierarchy`` of the reference (``PKG/solver/mas/hierarchy.py:150-271``)
with vectorised NumPy / SciPy graph routines:

* ordering: the reference partitions every level with pymetis
  (``mas/metis.py:42-90``, an un-vendored dependency).  Here the partition
  is *consecutive chunks of* ``target_nodes`` *node ids*, followed by the
  reference's own post-processing: every part is split into its connected
  components and the components are ordered by their smallest node.  With
  vertices numbered in Morton order the parts are 32-vertex Morton domains.
* packing (``mas/partition.py:41-73``), compatible-node collapse
  (``mas/hierarchy.py:105-147``) and the global coarse domain
  (``hierarchy.py:252-269``) follow the reference.

It also produces the device tables of :class:`MasTables`: composed maps,
child lists, domain layouts, the Galerkin source lists of every coarse
block and the dense-assembly entries of every domain.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy.sparse import coo_matrix
from scipy.sparse.csgraph import connected_components


def _unique_edges(i, j):
  i = np.asarray(i, dtype=np.int64)
  j = np.asarray(j, dtype=np.int64)
  keep = i != j
  a, b = np.minimum(i[keep], j[keep]), np.maximum(i[keep], j[keep])
  if a.size == 0:
    return np.zeros((0, 2), dtype=np.int64)
  key = np.unique(a * (1 << 32) + b)
  return np.stack([key >> 32, key & 0xFFFFFFFF], axis=1)


def _components(n, edges, mask):
  e = edges[mask]
  g = coo_matrix((np.ones(len(e)), (e[:, 0], e[:, 1])), shape=(n, n))
  _, labels = connected_components(g, directed=False)
  return labels


def chunk_groups(n, edges, target):
  """Groups (lists of node ids) of one level: chunks split into components,
  ordered by their smallest node.  Within a group nodes are in id order."""
  if n <= 1 or len(edges) == 0:
    return [np.arange(n, dtype=np.int64)]
  chunk = np.arange(n) // target
  labels = _components(n, edges, chunk[edges[:, 0]] == chunk[edges[:, 1]])
  order = np.lexsort((np.arange(n), labels))
  lab_sorted = labels[order]
  splits = np.flatnonzero(np.diff(lab_sorted)) + 1
  groups = np.split(order, splits)
  groups.sort(key=lambda g: int(g[0]))
  return groups


def pack_domain_groups(groups, dims, max_dofs):
  """Greedy capacity packing inside every group (``mas/partition.py:41-73``)."""
  domains = []
  for g in groups:
    d = dims[g]
    if int(d.sum()) <= max_dofs:
      domains.append(g)
      continue
    cur, cur_dofs = [], 0
    for node, nd in zip(g.tolist(), d.tolist()):
      if cur and cur_dofs + nd > max_dofs:
        domains.append(np.asarray(cur))
        cur, cur_dofs = [], 0
      cur.append(node)
      cur_dofs += nd
      if nd > max_dofs:
        domains.append(np.asarray(cur))
        cur, cur_dofs = [], 0
    if cur:
      domains.append(np.asarray(cur))
  return domains


def collapse(n, edges, domains, dims):
  """Compatible-node collapse; compact ids in order of first appearance."""
  node_dom = np.empty(n, dtype=np.int64)
  for d, dom in enumerate(domains):
    node_dom[dom] = d
  same = (node_dom[edges[:, 0]] == node_dom[edges[:, 1]]) & (dims[edges[:, 0]] == dims[edges[:, 1]])
  labels = _components(n, edges, same)
  _, first = np.unique(labels, return_index=True)
  rank = np.empty(first.size, dtype=np.int64)
  rank[np.argsort(first, kind="stable")] = np.arange(first.size)
  mapping = rank[labels]
  coarse_dims = np.empty(first.size, dtype=np.int64)
  coarse_dims[mapping] = dims
  return mapping, coarse_dims


@dataclass
class Level:
  dims: np.ndarray
  edges: np.ndarray
  domains: list
  order: np.ndarray


@dataclass
class Hierarchy:
  levels: list
  composed: list        # composed[l][fine] = node of level l
  signature: tuple = field(default=())

  @property
  def domains_per_level(self):
    return [len(l.domains) for l in self.levels]

  @property
  def nodes_per_level(self):
    return [int(l.dims.size) for l in self.levels]


def build_hierarchy(node_dims, edges, max_domain_dofs=96, max_levels=6, target_nodes=32,
                    global_coarse_domain=True) -> Hierarchy:
  """``build_hierarchy`` (``PKG/solver/mas/hierarchy.py:150-271``) with chunk ordering."""
  dims = np.asarray(node_dims, dtype=np.int64).copy()
  edges = _unique_edges(edges[:, 0], edges[:, 1]) if len(edges) else np.zeros((0, 2), np.int64)
  n = dims.size
  levels, composed, seen = [], [np.arange(n, dtype=np.int64)], set()
  while len(levels) < max_levels:
    sig = (dims.tobytes(), edges.tobytes())
    if sig in seen:
      break
    seen.add(sig)
    groups = chunk_groups(n, edges, target_nodes)
    domains = pack_domain_groups(groups, dims, max_domain_dofs)
    levels.append(Level(dims.copy(), edges.copy(), domains, np.concatenate(groups)))
    if len(levels) >= max_levels or n <= 1 or len(edges) == 0:
      break
    mapping, cdims = collapse(n, edges, domains, dims)
    if cdims.size == n:
      break
    composed.append(mapping[composed[-1]])
    cedges = _unique_edges(mapping[edges[:, 0]], mapping[edges[:, 1]])
    if cdims.size == dims.size and np.array_equal(cedges, edges):
      break
    dims, edges, n = cdims, cedges, cdims.size
  last = levels[-1]
  if global_coarse_domain and int(last.dims.sum()) <= max_domain_dofs and len(last.domains) > 1:
    last.domains = [last.order.copy()]
  return Hierarchy(levels, composed[:len(levels)])


@dataclass
class MasTables:
  """Host arrays of the device description (``ys_mas_desc``)."""

  num_fine_vars: int
  level_node_offset: np.ndarray
  cmap: np.ndarray
  child_ptr: np.ndarray
  child_fine: np.ndarray
  dom_node_ptr: np.ndarray
  dom_nodes: np.ndarray
  inv_offset: np.ndarray
  dom_entry_ptr: np.ndarray
  dom_entry: np.ndarray
  fine_blocks: int
  cb_src_ptr: np.ndarray
  cb_src: np.ndarray
  cb_level_begin: np.ndarray
  max_domain_dofs: int
  inverse_floats: int


def inverse_floats(dofs: int) -> int:
  """FP32 floats of one domain's tiled inverse: the upper 4x4 tiles of the
  inverse padded to T = ceil(dofs / 4) (rounded up to even) tile rows,
  16 floats a tile (``ys_mas_inverse_floats``)."""
  t = (dofs + 3) // 4
  t += t & 1
  return 8 * t * (t + 1)


def _step_map(h: Hierarchy, l: int, counts, nv) -> np.ndarray:
  """Map of level l-1 node ids to level l node ids (composed[l] = step o composed[l-1])."""
  if l == 1:
    return h.composed[1]
  rep = np.zeros(counts[l - 1], dtype=np.int64)
  rep[h.composed[l - 1]] = np.arange(nv)
  return h.composed[l][rep]


def build_tables(h: Hierarchy, fine_positions: np.ndarray) -> MasTables:
  """Device tables for 3-DoF variables and one 3x3 upper block set.

  ``fine_positions`` are the (row, col) scalar offsets of the fine blocks in
  storage order (block b has values at 9*b).
  """
  nv = h.levels[0].dims.size
  if not all(np.all(l.dims == 3) for l in h.levels):
    raise ValueError("the device MAS supports 3-DoF variables")
  L = len(h.levels)
  counts = [l.dims.size for l in h.levels]
  offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
  cmap = np.stack([offs[l] + h.composed[l] for l in range(L)]).astype(np.uint32)
  # children of coarse packed nodes: the packed ids of their nodes one level
  # below, ascending (the restriction runs level by level)
  child_ptr, child_fine, base = [0], [], 0
  for l in range(1, L):
    step = _step_map(h, l, counts, nv)
    order = np.argsort(step, kind="stable")
    cnt = np.bincount(step, minlength=counts[l])
    child_fine.append(offs[l - 1] + order)
    child_ptr.extend((base + np.cumsum(cnt)).tolist())
    base += int(cnt.sum())
  child_ptr = np.asarray(child_ptr, dtype=np.uint32)
  child_fine = np.concatenate(child_fine).astype(np.uint32) if child_fine else np.zeros(0, np.uint32)
  # domains
  dom_ptr, dom_nodes, inv_off, node_dom, node_loc = [0], [], [], [], []
  cursor = 0
  max_dofs = 0
  for l, lvl in enumerate(h.levels):
    nd = np.full(counts[l], -1, dtype=np.int64)
    nl = np.zeros(counts[l], dtype=np.int64)
    for d, dom in enumerate(lvl.domains):
      dom = np.asarray(dom, dtype=np.int64)
      nd[dom] = len(dom_ptr) - 1
      nl[dom] = np.arange(dom.size)
      dom_nodes.append(offs[l] + dom)
      dom_ptr.append(dom_ptr[-1] + dom.size)
      inv_off.append(cursor)
      k = 3 * dom.size
      cursor += inverse_floats(k)
      max_dofs = max(max_dofs, 3 * dom.size)
    node_dom.append(nd)
    node_loc.append(nl)
  # level blocks and Galerkin sources
  fine = np.asarray(fine_positions, dtype=np.int64).reshape(-1, 2) // 3
  nb0 = fine.shape[0]
  level_pairs = [fine]          # (a, b) node pairs of each level's blocks, a <= b
  level_base = [0]              # global block index of each level's first block
  cb_src_ptr, cb_src, cb_level_begin = [0], [], [0, 0]
  next_index = nb0
  for l in range(1, L):
    prev = level_pairs[-1]
    to_l = _step_map(h, l, counts, nv)
    A, B = to_l[prev[:, 0]], to_l[prev[:, 1]]
    lo, hi = np.minimum(A, B), np.maximum(A, B)
    mode = np.where(A < B, 0, np.where(A > B, 1, np.where(prev[:, 0] == prev[:, 1], 0, 2)))
    key = lo * (1 << 32) + hi
    uniq, inv = np.unique(key, return_inverse=True)
    order = np.lexsort((np.arange(key.size), inv))
    src_idx = level_base[-1] + order
    cb_src.append((src_idx | (mode[order] << 30)).astype(np.uint32))
    cnt = np.bincount(inv, minlength=uniq.size)
    cb_src_ptr.extend((cb_src_ptr[-1] + np.cumsum(cnt)).tolist())
    level_pairs.append(np.stack([uniq >> 32, uniq & 0xFFFFFFFF], axis=1))
    level_base.append(next_index)
    next_index += uniq.size
    cb_level_begin.append(cb_level_begin[-1] + uniq.size)
  while len(cb_level_begin) < L + 1:
    cb_level_begin.append(cb_level_begin[-1])
  cb_level_begin = np.asarray(cb_level_begin[:L + 1], dtype=np.uint32)
  # dense-assembly entries per domain
  ent_dom, ent = [], []
  for l in range(L):
    pairs = level_pairs[l]
    da, db = node_dom[l][pairs[:, 0]], node_dom[l][pairs[:, 1]]
    sel = np.flatnonzero(da == db)
    ent_dom.append(da[sel])
    ent.append(np.stack([node_loc[l][pairs[sel, 0]], node_loc[l][pairs[sel, 1]], level_base[l] + sel], axis=1))
  ent_dom = np.concatenate(ent_dom)
  ent = np.concatenate(ent)
  order = np.argsort(ent_dom, kind="stable")
  ndom = len(dom_ptr) - 1
  dom_entry_ptr = np.concatenate([[0], np.cumsum(np.bincount(ent_dom, minlength=ndom))]).astype(np.uint32)
  return MasTables(
      num_fine_vars=nv, level_node_offset=offs.astype(np.uint32), cmap=cmap.reshape(-1),
      child_ptr=child_ptr, child_fine=child_fine, dom_node_ptr=np.asarray(dom_ptr, dtype=np.uint32),
      dom_nodes=np.concatenate(dom_nodes).astype(np.uint32), inv_offset=np.asarray(inv_off, dtype=np.uint64),
      dom_entry_ptr=dom_entry_ptr, dom_entry=ent[order].astype(np.uint32).reshape(-1), fine_blocks=nb0,
      cb_src_ptr=np.asarray(cb_src_ptr, dtype=np.uint32),
      cb_src=np.concatenate(cb_src) if cb_src else np.zeros(0, np.uint32), cb_level_begin=cb_level_begin,
      max_domain_dofs=max(max_dofs, 3), inverse_floats=cursor)
