"""Sharding plumbing on the CPU: LPT partition and tour ranges, and the final gather of
best tours and costs across two gloo ranks (each rank solves only its share with a fake
solver). No GPU needed."""

from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from tsp_gpu_clean_b200 import sharding  # noqa: E402


def test_lpt_partition_covers_everything_and_balances():
  rng = np.random.default_rng(5)
  ns = [int(round(np.exp(rng.uniform(np.log(50), np.log(5000))))) for _ in range(256)]
  work = sharding.instance_work(ns, 64)
  for world in (1, 2, 3, 8):
    parts = sharding.lpt_partition(work, world)
    assert sorted(i for p in parts for i in p) == list(range(256))
    assert parts == sharding.lpt_partition(work, world)  # same plan on every rank
    loads = [sum(work[i] for i in p) for p in parts]
    assert max(loads) <= sum(work) / world + max(work)  # LPT bound
  # 0 (5) -> r0, 2 (4) -> r1, 4 (3) -> r1, 3 (2) -> r0, 1 (1) -> r0 (tie at 7: lower rank)
  assert sharding.lpt_partition([5, 1, 4, 2, 3], 2) == [[0, 1, 3], [2, 4]]
  with pytest.raises(ValueError):
    sharding.lpt_partition([1.0], 0)


def test_tour_ranges_are_contiguous_and_even():
  for total, world in ((1024, 8), (1000, 3), (5, 8), (0, 2)):
    ranges = [sharding.tour_range(total, world, r) for r in range(world)]
    assert ranges[0][0] == 0 and ranges[-1][1] == total
    assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    sizes = [hi - lo for lo, hi in ranges]
    assert max(sizes) - min(sizes) <= 1


def test_gather_without_a_process_group_reorders():
  t, c = sharding.gather_best([2, 0], [np.array([1, 0]), np.array([0, 1, 2])], [5.0, 7.0], 3)
  assert np.array_equal(t[0], [0, 1, 2]) and t[1] is None and np.array_equal(t[2], [1, 0])
  assert c[0] == 7.0 and np.isnan(c[1]) and c[2] == 5.0


class _Ctx:
  def __init__(self, n, seed):
    self.dimension, self.seed = n, seed


def _expected(ctx):
  return np.roll(np.arange(ctx.dimension, dtype=np.int32), ctx.seed % ctx.dimension), float(ctx.seed * 3 + ctx.dimension)


class _FakeSolver:
  def __init__(self, log):
    self.log = log

  def evolve(self, contexts, G, patience=None, optimal_cost=None):
    self.log.extend(c.seed for c in contexts)
    out = []
    for c in contexts:
      tour, cost = _expected(c)
      out.append((tour, {"best_fitness": cost, "generations_completed": G}))
    return out


def _free_port() -> int:
  with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
    s.bind(("127.0.0.1", 0))
    return s.getsockname()[1]


def _contexts(count=23):
  rng = np.random.default_rng(9)
  return [_Ctx(int(n), s) for s, n in enumerate(rng.integers(5, 400, count))]


def _rank_main(rank: int, world: int, port: int, out, count=23):
  import datetime

  import torch.distributed as dist

  sys.path.insert(0, ROOT)
  from tsp_gpu_clean_b200 import sharding as sh

  os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
  dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
  try:
    log = []
    solver = sh.ShardedBatchSolver(lambda: _FakeSolver(log), population_size=64)
    res = solver.evolve(_contexts(count), 10)
    out.put((rank, [(t.tolist(), c) for t, c in res], sorted(log), sorted(solver.local_stats)))
  finally:
    dist.destroy_process_group()


@pytest.mark.timeout(180)
@pytest.mark.parametrize("count", [23, 1])
def test_two_gloo_ranks_solve_their_share_and_gather_every_run(count):
  """23 runs split across two ranks, and a single run (the second rank has none)."""
  import torch.multiprocessing as tmp

  ctx = tmp.get_context("spawn")
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q, count)) for r in range(2)]
  for p in procs:
    p.start()
  results = sorted(q.get(timeout=120) for _ in procs)
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  contexts = _contexts(count)
  want = [(_expected(c)[0].tolist(), _expected(c)[1]) for c in contexts]
  (_, res0, log0, own0), (_, res1, log1, own1) = results
  assert res0 == want and res1 == want  # every rank holds every run's result
  assert sorted(log0 + log1) == list(range(len(contexts)))  # each run solved exactly once
  assert log0 and (log1 if count > 1 else not log1)
  plan = sharding.lpt_partition(sharding.instance_work([c.dimension for c in contexts], 64), 2)
  assert own0 == plan[0] and own1 == plan[1]
