"""Multi-GPU sharding of the GA and 2-opt work: one process per GPU, no collective inside
the generation loop, one gather at the end.

GA runs and tours are independent units, so ranks split them and never exchange data while
they run:
- `lpt_partition` assigns whole instances to ranks by longest-processing-time bin packing on
  an estimate of each run's work (n^2 * population);
- `tour_range` splits a batch of tours into contiguous ranges.

`gather_best` is the only exchange: every rank's best tours and costs go to every rank with
two `all_gather` calls. The first carries the sizes; the second carries the padded tours and
costs. Over NCCL they travel NVLink / NVSwitch; over gloo (tests) the host network.
`ShardedBatchSolver` combines the two: each rank solves its share on a `FusedBatchSolver`,
then every rank holds every run's best tour and cost in the caller's order.
"""

from __future__ import annotations

from typing import Any, Callable, Sequence

import numpy as np


def instance_work(ns: Sequence[int], population: int) -> list[float]:
  """Work estimate of one GA run per instance: n^2 * population."""
  return [float(n) * float(n) * float(population) for n in ns]


def lpt_partition(work: Sequence[float], world: int) -> list[list[int]]:
  """Indices of `work` per rank. Largest first, each to the rank with the least work so far
  (ties: the lower index first, then the lower rank), so every rank computes the same plan."""
  if world < 1:
    raise ValueError("world must be >= 1")
  loads = [0.0] * world
  parts: list[list[int]] = [[] for _ in range(world)]
  for i in sorted(range(len(work)), key=lambda j: (-float(work[j]), j)):
    r = min(range(world), key=lambda q: (loads[q], q))
    parts[r].append(i)
    loads[r] += float(work[i])
  return [sorted(p) for p in parts]


def tour_range(num_tours: int, world: int, rank: int) -> tuple[int, int]:
  """[lo, hi) of rank's contiguous share of `num_tours` (sizes differ by at most one)."""
  if not 0 <= rank < world:
    raise ValueError("rank outside [0, world)")
  base, extra = divmod(num_tours, world)
  lo = rank * base + min(rank, extra)
  return lo, lo + base + (1 if rank < extra else 0)


def _dist():
  import torch.distributed as dist

  return dist if dist.is_available() and dist.is_initialized() else None


def gather_best(indices: Sequence[int], tours: Sequence[np.ndarray], costs: Sequence[float], total: int,
                device: str | None = None) -> tuple[list[np.ndarray | None], np.ndarray]:
  """Every rank's (global index, best tour, best cost) triples on every rank.

  `indices` are this rank's global run indices and `tours` / `costs` their results. Returns
  the tours in global order (None for an index no rank reported) and the costs (NaN there).
  Without an initialised process group this only reorders the local results.
  """
  import torch

  dist = _dist()
  out_t: list[np.ndarray | None] = [None] * total
  out_c = np.full(total, np.nan)
  if dist is None or dist.get_world_size() == 1:
    for i, t, c in zip(indices, tours, costs):
      out_t[int(i)] = np.asarray(t, dtype=np.int32)
      out_c[int(i)] = float(c)
    return out_t, out_c
  world = dist.get_world_size()
  if device is None:
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
  # 1) sizes: runs and tour elements per rank
  lens = [int(np.asarray(t).shape[0]) for t in tours]
  size = torch.tensor([len(indices), int(sum(lens))], dtype=torch.int64, device=device)
  sizes = [torch.zeros_like(size) for _ in range(world)]
  dist.all_gather(sizes, size)
  sizes = [s.cpu().numpy() for s in sizes]
  max_runs = max(int(s[0]) for s in sizes)
  max_elems = max(int(s[1]) for s in sizes)
  # 2) one padded buffer per rank: [index, length] per run, the costs, then the tours
  head = np.zeros((max_runs, 2), dtype=np.int64)
  head[: len(indices), 0] = np.asarray(indices, dtype=np.int64)
  head[: len(indices), 1] = np.asarray(lens, dtype=np.int64)
  cost = np.zeros(max_runs, dtype=np.float64)
  cost[: len(costs)] = np.asarray(costs, dtype=np.float64)
  body = np.zeros(max(max_elems, 1), dtype=np.int64)
  if lens:
    body[: sum(lens)] = np.concatenate([np.asarray(t, dtype=np.int64) for t in tours])
  flat = np.concatenate([head.ravel(), cost.view(np.int64), body])
  mine = torch.from_numpy(flat).to(device)
  bufs = [torch.empty_like(mine) for _ in range(world)]
  dist.all_gather(bufs, mine)
  for r, buf in enumerate(bufs):
    b = buf.cpu().numpy()
    nr = int(sizes[r][0])
    h = b[: 2 * max_runs].reshape(max_runs, 2)
    c = b[2 * max_runs: 3 * max_runs].view(np.float64)
    body = b[3 * max_runs:]
    off = 0
    for q in range(nr):
      idx, ln = int(h[q, 0]), int(h[q, 1])
      out_t[idx] = body[off: off + ln].astype(np.int32)
      out_c[idx] = float(c[q])
      off += ln
  return out_t, out_c


class ShardedBatchSolver:
  """The runs of `evolve` split across the ranks of the current process group (LPT on
  n^2 * population), each rank's share on its own `FusedBatchSolver`, then `gather_best`.

  `make_solver()` returns the rank's solver (a `FusedBatchSolver` or any object with the
  same `evolve(contexts, G, patience=..., optimal_cost=...)`). Every rank passes the same
  contexts in the same order and gets every run's `(best_tour, best_cost)`. This rank's own
  runs keep their full statistics in `local_stats` (global index -> stats dict).
  """

  def __init__(self, make_solver: Callable[[], Any], population_size: int) -> None:
    self.make_solver = make_solver
    self.population_size = int(population_size)
    self.local_stats: dict[int, dict] = {}
    self.plan: list[list[int]] = []

  def evolve(self, contexts: Sequence[Any], max_generations: int, patience: Any = None,
             optimal_cost: Any = None) -> list[tuple[np.ndarray, float]]:
    dist = _dist()
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    ns = [int(c.dimension) for c in contexts]
    self.plan = lpt_partition(instance_work(ns, self.population_size), world)
    mine = self.plan[rank]

    def pick(v):
      if isinstance(v, (list, tuple, np.ndarray)):
        return [v[i] for i in mine]
      return v

    tours, costs = [], []
    self.local_stats = {}
    if mine:
      solver = self.make_solver()
      res = solver.evolve([contexts[i] for i in mine], max_generations, patience=pick(patience),
                          optimal_cost=pick(optimal_cost))
      for i, (best, stats) in zip(mine, res):
        tours.append(np.asarray(best, dtype=np.int32))
        costs.append(float(stats["best_fitness"]))
        self.local_stats[i] = stats
    all_t, all_c = gather_best(mine, tours, costs, len(contexts))
    return [(t, float(c)) for t, c in zip(all_t, all_c)]
