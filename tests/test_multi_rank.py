"""Multi-rank plumbing of bench.py on the CPU: two gloo ranks reduce their counters (sum)
and elapsed times (max) the way the GPU ranks do over NCCL; the weak-scaling shards differ
per rank. No GPU needed."""

from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
  with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
    s.bind(("127.0.0.1", 0))
    return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
  import datetime

  import torch.distributed as dist

  sys.path.insert(0, ROOT)
  import bench

  os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
  dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
  try:
    units, elapsed = bench.aggregate(10.0 * (rank + 1), 0.5 + rank, world)
    out.put((rank, units, elapsed))
  finally:
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_sum_units_and_max_time():
  import torch.multiprocessing as tmp

  ctx = tmp.get_context("spawn")
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
  for p in procs:
    p.start()
  results = sorted(q.get(timeout=120) for _ in procs)
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  assert [(r, u, e) for r, u, e in results] == [(0, 30.0, 1.5), (1, 30.0, 1.5)]


def test_single_process_aggregate_is_identity():
  sys.path.insert(0, ROOT)
  import bench

  assert bench.aggregate(7.0, 0.25, 1) == (7.0, 0.25)


def test_weak_scaling_shards_differ_per_rank():
  from tsp_gpu_clean_b200 import instances

  sys.path.insert(0, ROOT)
  import bench

  a = instances.uneven_batch(8, bench.UNEVEN_SEED)
  b = instances.uneven_batch(8, bench.UNEVEN_SEED + 7919)
  assert [len(x) for x in a] != [len(x) for x in b] or any(not np.array_equal(x, y) for x, y in zip(a, b))
  t0 = instances.random_tours(50, 4, instances.TWO_OPT_TOUR_SEED)
  t1 = instances.random_tours(50, 4, instances.TWO_OPT_TOUR_SEED + 1000)
  assert not np.array_equal(t0, t1)
