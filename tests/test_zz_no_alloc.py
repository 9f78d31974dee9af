"""ys_compress_indices_noalloc (no allocation, fixed device scratch) against
ys_compress_indices, both through the C ABI.

The outputs are integers: the tolerance is bit-exact.  Several calls in a row
on inputs of different sizes check that the shared scratch, which keeps the
previous call's contents, does not leak into a later result.  The device's
memory pool (the one cudaMallocAsync draws from) shows that the entry point
really allocates nothing: its used-memory high-water mark stays at zero over
the calls, while the allocating entry point raises it.
"""

import ctypes

import numpy as np
import pytest

from yasps_b200 import _lib as L

pytestmark = pytest.mark.gpu

MAX_INSTANCES = 67_108_864


def make_codes(n, K, seed):
  """Slot codes with padding (0), DATA (1), repeated targets and sizes 1..4."""
  rng = np.random.default_rng(seed)
  codes = rng.integers(2, 2 + max(8, n // 4), size=(n, K), dtype=np.int64)
  codes[rng.random((n, K)) < 0.1] = 0
  codes[rng.random((n, K)) < 0.05] = 1
  dup = rng.random((n, K)) < 0.15
  src = rng.integers(0, K, size=(n, K))
  codes[dup] = codes[np.nonzero(dup)[0], src[dup]]
  sizes = rng.integers(1, 5, size=(n, K), dtype=np.int64)
  return codes.astype(np.int32), sizes.astype(np.int16)


def run(name, codes, sizes):
  import torch
  n, K = codes.shape
  c = torch.from_numpy(codes.reshape(-1)).cuda()
  sz = torch.from_numpy(sizes.reshape(-1)).cuda()
  perm = torch.full((n * K,), 77, dtype=torch.int16, device="cuda")
  total = torch.full((n,), 77, dtype=torch.int16, device="cuda")
  outer = torch.full((n + 1,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
  L.call(name, L.ptr(c), L.ptr(sz), n, K, L.ptr(perm), L.ptr(total), L.ptr(outer), L.stream_ptr())
  torch.cuda.synchronize()
  return perm.cpu().numpy(), total.cpu().numpy(), outer.cpu().numpy()


def test_noalloc_matches_allocating_entry_on_calls_in_a_row():
  # 2.5M instances span 1221 tiles of 2048 (more than one tile sum per thread
  # of the offset scan); then smaller and ragged sizes reuse the scratch.
  cases = [(2_500_000, 4, 0), (5_000, 8, 1), (3 * 2048, 2, 2), (1, 3, 3), (2_500_000, 4, 4)]
  for n, K, seed in cases:
    codes, sizes = make_codes(n, K, seed)
    ref = run("ys_compress_indices", codes, sizes)
    for _ in range(2):
      got = run("ys_compress_indices_noalloc", codes, sizes)
      for a, b in zip(got, ref):
        assert np.array_equal(a, b), (n, K)
    counts = np.diff(ref[2].astype(np.int64))
    assert ref[2][0] == 0 and (counts >= 0).all()


def test_noalloc_rejects_sizes_beyond_its_scratch():
  lib = L.load()
  rc = lib.ys_compress_indices_noalloc(None, None, MAX_INSTANCES + 1, 4, None, None, None, None)
  assert rc == -3  # YS_ERR_CAPACITY
  assert b"67,108,864" in lib.ys_last_error()


CU_MEMPOOL_ATTR_USED_MEM_HIGH = 8


def pool_high_water(fn):
  """Bytes of the current device's memory pool in use at its peak while
  ``fn`` runs (the high-water mark is reset to zero before, read after)."""
  import torch
  cu = ctypes.CDLL("libcuda.so.1")
  dev = ctypes.c_int()
  assert cu.cuCtxGetDevice(ctypes.byref(dev)) == 0
  pool = ctypes.c_void_p()
  assert cu.cuDeviceGetMemPool(ctypes.byref(pool), dev) == 0
  torch.cuda.synchronize()
  zero = ctypes.c_uint64(0)
  assert cu.cuMemPoolSetAttribute(pool, CU_MEMPOOL_ATTR_USED_MEM_HIGH, ctypes.byref(zero)) == 0
  fn()
  torch.cuda.synchronize()
  high = ctypes.c_uint64(1)
  assert cu.cuMemPoolGetAttribute(pool, CU_MEMPOOL_ATTR_USED_MEM_HIGH, ctypes.byref(high)) == 0
  return high.value


def test_noalloc_allocates_nothing():
  import torch
  n, K = 2_500_000, 4
  codes, sizes = make_codes(n, K, 5)
  c = torch.from_numpy(codes.reshape(-1)).cuda()
  sz = torch.from_numpy(sizes.reshape(-1)).cuda()
  perm = torch.empty(n * K, dtype=torch.int16, device="cuda")
  total = torch.empty(n, dtype=torch.int16, device="cuda")
  outer = torch.empty(n + 1, dtype=torch.int32, device="cuda")
  args = (L.ptr(c), L.ptr(sz), n, K, L.ptr(perm), L.ptr(total), L.ptr(outer), L.stream_ptr())
  L.call("ys_compress_indices_noalloc", *args)  # the first call on the device does the set-up
  assert pool_high_water(lambda: [L.call("ys_compress_indices_noalloc", *args) for _ in range(2)]) == 0
  # the check sees allocations: the allocating entry point's scan storage
  assert pool_high_water(lambda: L.call("ys_compress_indices", *args)) > 0
