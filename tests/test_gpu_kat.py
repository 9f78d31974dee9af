"""The ported assembly known-answer cases through the device pattern build and
the generic (any block size) deterministic assembly, via the C ABI.

Slot codes -> ``ys_compress_indices`` -> ``ys_compute_coordinates`` ->
``ys_pattern_build``; the per-occurrence records of the local Hessians are
filled on the host with the NoProject merge rules and summed by
``ys_assemble``.  Pattern positions and lookups are compared bit-exact with
the oracle, block values at 1e-12 relative (the oracle itself matches the
reference's dense expectations at 3e-11, tests/test_oracle_kat.py).
"""

import ctypes

import numpy as np
import pytest

from tests.test_oracle_kat import CASES, build, oracle_assemble
from yasps_b200 import _lib as L

pytestmark = pytest.mark.gpu


def occurrence_blocks(codes, sizes, perm, h):
  """Merged upper blocks of one instance in coordinate order."""
  offs = np.concatenate([[0], np.cumsum(sizes)[:-1]])
  groups = []
  for i in range(len(codes)):
    if perm[i] == 0:
      continue
    for g in groups:
      if g[0] == abs(perm[i]):
        g[1].append(i)
        break
    else:
      groups.append([abs(perm[i]), [i]])
  out = []
  tgt = [g[1] for g in groups if codes[g[1][0]] >= 2]
  for a in range(len(tgt)):
    for b in range(a, len(tgt)):
      ga, gb = tgt[a], tgt[b]
      sa, sb = sizes[ga[0]], sizes[gb[0]]
      blk = np.zeros((sa, sb))
      for i in ga:
        for j in gb:
          blk += h[offs[i]:offs[i] + sa, offs[j]:offs[j] + sb]
      out.append(blk if codes[ga[0]] < codes[gb[0]] else blk.T)
  return out


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-{c[1]}-{c[2]}" for c in CASES])
def test_device_pattern_and_assembly(case):
  import torch
  from yasps_b200.hessian import _Pattern
  codes, sizes, gs, hs, exp_h, exp_g, n, shapes = build(case)
  pat, values, _, _ = oracle_assemble(codes, sizes, gs, hs, n, shapes)
  ni, K = codes.shape
  s = L.stream_ptr()
  dc = torch.from_numpy(codes.astype(np.int32).ravel()).cuda()
  ds = torch.from_numpy(sizes.astype(np.int16).ravel()).cuda()
  perm = torch.empty(ni * K, dtype=torch.int16, device="cuda")
  outer = torch.empty(ni + 1, dtype=torch.int32, device="cuda")
  L.call("ys_compress_indices", L.ptr(dc), L.ptr(ds), ni, K, L.ptr(perm), None, L.ptr(outer), s)
  m = int(outer[ni].item())
  coords = torch.empty(2 * m, dtype=torch.int32, device="cuda")
  dims = torch.empty(2 * m, dtype=torch.int16, device="cuda")
  L.call("ys_compute_coordinates", L.ptr(dc), L.ptr(perm), L.ptr(ds), L.ptr(outer), ni, K, L.ptr(coords),
         L.ptr(dims), s)
  p = _Pattern(coords, dims, m)
  pos = p.positions[:2 * p.num_unique].cpu().numpy().astype(np.int64).reshape(-1, 2)
  assert np.array_equal(pos, pat.positions)
  assert np.array_equal(p.lookup[:m].cpu().numpy().astype(np.int64), pat.lookups[0])
  # records at their sorted occurrence slots
  perm_h = perm.cpu().numpy().reshape(ni, K)
  outer_h = outer.cpu().numpy()
  record = p.record[:m].cpu().numpy().astype(np.int64)
  rec = np.zeros(max(p.total_records, 1))
  for t in range(ni):
    for k, blk in enumerate(occurrence_blocks(codes[t], sizes[t], perm_h[t], hs[t])):
      o = record[outer_h[t] + k]
      rec[o:o + blk.size] = blk.ravel()
  drec = torch.from_numpy(rec).cuda()
  vals = torch.zeros(max(p.total_values, 1), dtype=torch.float64, device="cuda")
  L.call("ys_assemble", L.ptr(drec), L.ptr(p.record_begin), L.ptr(p.record_count), L.ptr(p.value_offset),
         L.ptr(p.dims), p.num_unique, L.ptr(vals), None, s)
  got = vals[:values.size].cpu().numpy()
  assert np.abs(got - values).max() <= 1e-12 * np.abs(values).max()
