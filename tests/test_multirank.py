"""The multi-rank path of bench.py on host-only ranks: world size 2 over the
gloo backend (127.0.0.1).  Each rank is an independent replica; the job's
time is the max over ranks and its throughput counts every rank's steps."""

import os
import socket

import pytest


def _free_port():
  with socket.socket() as s:
    s.bind(("127.0.0.1", 0))
    return s.getsockname()[1]


def _rank(rank, world, port, out):
  os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                    MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
  import bench
  r, w, _, pg = bench.dist_setup(None)
  assert (r, w) == (rank, world) and pg is not None and pg.get_backend() == "gloo"
  bench.barrier(pg)
  ms = bench.max_over_ranks(100.0 + 50.0 * rank, pg)
  out.put((rank, ms, bench.replica_value(w, 30, ms)))
  bench.barrier(pg)
  pg.destroy_process_group()


def test_two_gloo_ranks_time_as_the_slowest_replica():
  import torch.multiprocessing as mp
  ctx = mp.get_context("spawn")
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
  for p in procs:
    p.start()
  for p in procs:
    p.join(timeout=120)
    assert p.exitcode == 0
  got = sorted(q.get(timeout=10) for _ in range(2))
  assert [g[1] for g in got] == [150.0, 150.0]
  assert all(g[2] == pytest.approx(2 * 30 / 0.150) for g in got)
