"""DoF maps, local compression, sparsity pattern and assembly (oracle only).

A *term* is one energy applied to ``n`` instances.  Per instance it has ``K``
index slots with a code and a size, exactly as produced by the reference's
generated ``<energy>_get_indices`` kernel
(``PKG/kernel/Coordinate/gradientIndicesKernel.pyx:546-600,689-846``):

* ``code == 0``   reserved union space (padding, or an argument with no
  differentiated leaf); its size still advances the local layout;
* ``code == 1``   a DATA leaf that is not a minimisation target: it is part
  of the local (projected) Hessian but is not scattered;
* ``code >= 2``   a target leaf at global scalar DoF ``code - 2``.

The local gradient / Hessian of an instance is laid out slot by slot in slot
order, every slot occupying ``size`` rows.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def compress_slots(codes: np.ndarray, sizes: np.ndarray):
  """Local permutation of one term (``computePermutation``).

  Restates ``gradientIndicesKernel.pyx:62-123``: padding slots are skipped;
  a target slot whose code already appeared gets ``-perm`` of that first
  occurrence; every other slot gets ``offset + 1`` and advances the
  compressed offset.  Returns ``(perm, compressed_size, n_unique_targets)``.
  """
  codes = np.asarray(codes, dtype=np.int64)
  sizes = np.asarray(sizes, dtype=np.int64)
  n, k = codes.shape
  perm = np.zeros((n, k), dtype=np.int64)
  total = np.zeros(n, dtype=np.int64)
  uniq = np.zeros(n, dtype=np.int64)
  for t in range(n):
    off = 0
    for i in range(k):
      c = codes[t, i]
      if c == 0:
        continue
      found = False
      if c >= 2:
        for j in range(i):
          if codes[t, j] == c:
            perm[t, i] = -perm[t, j]
            found = True
            break
      if not found:
        perm[t, i] = off + 1
        off += sizes[t, i]
        total[t] += sizes[t, i]
        if c >= 2:
          uniq[t] += 1
  return perm, total, uniq


def coordinates(codes, sizes, perm):
  """Upper-triangle block coordinates in slot order (``computeCoordinates``).

  ``gradientIndicesKernel.pyx:234-274``: for slots ``i <= j`` that are first
  occurrences of targets, emit ``(min dof, max dof)`` with the matching
  block dimensions.  Returns ``(coords (m,2), dims (m,2), outer (n+1,))``.
  """
  codes = np.asarray(codes, dtype=np.int64)
  sizes = np.asarray(sizes, dtype=np.int64)
  n, k = codes.shape
  coords, dims, outer = [], [], [0]
  for t in range(n):
    valid = [i for i in range(k) if perm[t, i] > 0 and codes[t, i] >= 2]
    for a, i in enumerate(valid):
      for j in valid[a:]:
        ci, cj = codes[t, i], codes[t, j]
        if ci < cj:
          coords.append((ci - 2, cj - 2))
          dims.append((sizes[t, i], sizes[t, j]))
        else:
          coords.append((cj - 2, ci - 2))
          dims.append((sizes[t, j], sizes[t, i]))
    outer.append(len(coords))
  return (np.asarray(coords, dtype=np.int64).reshape(-1, 2), np.asarray(dims, dtype=np.int64).reshape(-1, 2),
          np.asarray(outer, dtype=np.int64))


@dataclass
class Pattern:
  """Unique upper block pattern of one block set (static or dynamic)."""

  positions: np.ndarray          # (nb, 2) scalar (row, col), sorted by (h, w, row, col)
  dims: np.ndarray               # (nb, 2) block (h, w)
  value_offsets: np.ndarray      # (nb,) start of each block in the flat values
  category_dims: np.ndarray      # (ncat, 2)
  category_counts: np.ndarray    # (ncat,)
  category_starts: np.ndarray    # (ncat + 1,) value offsets
  lookups: list = field(default_factory=list)  # per term, value offset of each coordinate

  @property
  def total_values(self) -> int:
    return int(self.category_starts[-1]) if self.category_starts.size else 0


def build_pattern(term_coords, term_dims) -> Pattern:
  """Global unique sort of all occurrences (``get_unique_coords``).

  ``PKG/kernel/Coordinate/coordinateCompressionKernel.pyx:34-53,92-144,264-419``:
  occurrences are ordered by ``(h, w, row, col)``, duplicates collapse, the
  value offset of a unique block is the exclusive scan of ``h*w`` in that
  order, and ``lookup[occurrence]`` is the value offset of its block.
  """
  all_c = np.concatenate([c for c in term_coords if len(c)] or [np.zeros((0, 2), np.int64)])
  all_d = np.concatenate([d for d in term_dims if len(d)] or [np.zeros((0, 2), np.int64)])
  if all_c.shape[0] == 0:
    return Pattern(np.zeros((0, 2), np.int64), np.zeros((0, 2), np.int64), np.zeros(0, np.int64),
                   np.zeros((0, 2), np.int64), np.zeros(0, np.int64), np.zeros(1, np.int64),
                   [np.zeros(0, np.int64) for _ in term_coords])
  order = np.lexsort((all_c[:, 1], all_c[:, 0], all_d[:, 1], all_d[:, 0]))
  key = np.stack([all_d[order, 0], all_d[order, 1], all_c[order, 0], all_c[order, 1]], axis=1)
  new_run = np.ones(len(order), dtype=bool)
  new_run[1:] = np.any(key[1:] != key[:-1], axis=1)
  ordinal = np.cumsum(new_run) - 1
  uniq = key[new_run]
  sizes = uniq[:, 0] * uniq[:, 1]
  value_offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
  lookup = np.empty(len(order), dtype=np.int64)
  lookup[order] = value_offsets[ordinal]
  cat_new = np.ones(len(uniq), dtype=bool)
  cat_new[1:] = np.any(uniq[1:, :2] != uniq[:-1, :2], axis=1)
  cat_first = np.flatnonzero(cat_new)
  cat_counts = np.diff(np.concatenate([cat_first, [len(uniq)]]))
  cat_starts = np.concatenate([value_offsets[cat_first], [value_offsets[-1] + sizes[-1]]])
  lookups, pos = [], 0
  for c in term_coords:
    lookups.append(lookup[pos:pos + len(c)])
    pos += len(c)
  return Pattern(uniq[:, 2:].copy(), uniq[:, :2].copy(), value_offsets, uniq[cat_first, :2].copy(), cat_counts,
                 cat_starts, lookups)


def scatter_term(codes, sizes, perm, lookup, outer, local_grad, local_hess, gradient, blocks,
                 diag_blocks, attr_segment_starts, attr_diag_starts):
  """Scatter one term's projected local results (NoProject semantics).

  Restates ``PKG/kernel/Hessian/hessianKernelNoProject.pyx:63-264``: every
  target slot adds its gradient segment; slots sharing a permutation are
  merged by summing their sub-blocks; for unique groups ``i <= j`` of target
  slots the merged block goes to ``lookup`` in row-major order when the row
  DoF is below the column DoF and transposed otherwise; diagonal groups are
  also added to the per-variable diagonal blocks.
  """
  codes = np.asarray(codes, dtype=np.int64)
  sizes = np.asarray(sizes, dtype=np.int64)
  n, k = codes.shape
  seg = np.asarray(attr_segment_starts, dtype=np.int64)
  dstart = np.asarray(attr_diag_starts, dtype=np.int64)
  for t in range(n):
    offs = np.concatenate([[0], np.cumsum(sizes[t])[:-1]])
    for i in range(k):
      if codes[t, i] >= 2:
        d = codes[t, i] - 2
        gradient[d:d + sizes[t, i]] += local_grad[t, offs[i]:offs[i] + sizes[t, i]]
    groups = []  # (first slot, [member slots])
    for i in range(k):
      p = perm[t, i]
      if p == 0:
        continue
      p = abs(p)
      for g in groups:
        if g[0] == p:
          g[2].append(i)
          break
      else:
        groups.append([p, i, [i]])
    m = 0
    for gi in range(len(groups)):
      ci = codes[t, groups[gi][1]]
      if ci < 2:
        continue
      si = sizes[t, groups[gi][1]]
      for gj in range(gi, len(groups)):
        cj = codes[t, groups[gj][1]]
        if cj < 2:
          continue
        sj = sizes[t, groups[gj][1]]
        acc = np.zeros((si, sj))
        for a in groups[gi][2]:
          for b in groups[gj][2]:
            acc += local_hess[t, offs[a]:offs[a] + si, offs[b]:offs[b] + sj]
        place = lookup[outer[t] + m]
        if ci < cj:
          blocks[place:place + si * sj] += acc.ravel()
        else:
          blocks[place:place + si * sj] += acc.T.ravel()
        if gi == gj:
          d = ci - 2
          attr = np.searchsorted(seg[1:], d, side="right")
          inst = (d - seg[attr]) // si
          base = dstart[attr] + inst * si * si
          diag_blocks[base:base + si * si] += acc.T.ravel()
        m += 1


def dense_from_blocks(pattern: Pattern, values: np.ndarray, size: int, symmetric: bool = True) -> np.ndarray:
  """Dense matrix of one block set (mirrors the reference test helper)."""
  dense = np.zeros((size, size))
  for (r, c), (h, w), off in zip(pattern.positions, pattern.dims, pattern.value_offsets):
    b = values[off:off + h * w].reshape(h, w)
    dense[r:r + h, c:c + w] += b
    if symmetric and r != c:
      dense[c:c + w, r:r + h] += b.T
  return dense


def spmv(pattern: Pattern, values: np.ndarray, x: np.ndarray, y: np.ndarray | None = None) -> np.ndarray:
  """``y += H x`` for symmetric upper block storage (``PKG/matrixAndVector/matrix/matrix.pyx:21-63``)."""
  x = np.asarray(x, dtype=np.float64)
  y = np.zeros_like(x) if y is None else y
  for (h, w) in {tuple(d) for d in pattern.dims.tolist()}:
    sel = np.flatnonzero((pattern.dims[:, 0] == h) & (pattern.dims[:, 1] == w))
    if not sel.size:
      continue
    rows, cols = pattern.positions[sel, 0], pattern.positions[sel, 1]
    b = values[pattern.value_offsets[sel][:, None] + np.arange(h * w)[None]].reshape(-1, h, w)
    xc = x[cols[:, None] + np.arange(w)[None]]
    np.add.at(y, rows[:, None] + np.arange(h)[None], np.einsum("bij,bj->bi", b, xc))
    off = rows != cols
    xr = x[rows[off][:, None] + np.arange(h)[None]]
    np.add.at(y, cols[off][:, None] + np.arange(w)[None], np.einsum("bij,bi->bj", b[off], xr))
  return y
