"""B200 population operators: evaluation, tournament selection, PMX crossover, inversion mutation.

Each class keeps the constructor and method shapes of the reference's CPU strategy and
produces bit-identical results for the same inputs and the same random draws:

- `EvaluationB200Cost`      <- `EvaluationCPUCost` (`cost_evaluation.py:46-162`, TSP branch;
                               `evaluate_tour_cpu`, `tour_cost.py:17-29`)
- `SelectionB200Tournament` <- `SelectionCPUTournament` (`tournament_selection.py:29-128`)
- `CrossoverB200PermPartiallyMapped` <- `CrossoverCPUPermPartiallyMapped` (`pmx_crossover.py:36-171`)
- `MutationB200PermInversion` <- `MutationCPUPermInversion` (`inversion_mutation.py:36-99`)
- `CrossoverB200PermOrder`  <- `CrossoverCPUPermOrder` (`order_crossover.py:36-168`)
- `MutationB200PermSwap`    <- `MutationCPUPermSwap` (`swap_mutation.py:36-99`)

Random draws are taken on the host from `context.rng` (falling back to the strategy's
own generator) with the same calls, shapes and order as the reference, then uploaded;
the kernels consume them. Host arrays in give host arrays out; CUDA tensors in give
CUDA tensors out. There is no CPU fallback.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from .. import native
from ..device import (
  PinnedStager,
  candidate_list,
  device_tensor,
  is_device_array,
  operands_for,
  ptr,
  require_gpu,
  stream_handle,
  torch,
)
from ..errors import NotPermutationError
from ..phase_timer import time_strategy
from ..problem import resolve_rng
from ..routes import ensure_routes_batch, resolve_route_bounds, restore_shape, sample_distinct_pairs
from .base import StrategyBase, tour_assessment


def _to_device(batch: Any, stager: PinnedStager | None = None) -> tuple["torch.Tensor", bool]:
  if is_device_array(batch):
    return batch.to(torch.int32).contiguous(), True
  host = np.ascontiguousarray(batch, dtype=np.int32)
  if stager is not None:
    return stager.upload(host, torch.int32), False
  return torch.from_numpy(host).to("cuda"), False


def _to_host(t: "torch.Tensor", stager: PinnedStager | None = None) -> np.ndarray:
  if stager is not None:
    return stager.download(t)
  return t.cpu().numpy()


class EvaluationB200Cost(StrategyBase):
  """Closed-tour cost of every route, float64 (exact: integer sums below 2^53)."""

  def __init__(self, max_matrix_dimension: int | None = None, return_gpu: bool = False) -> None:
    super().__init__()
    self.max_matrix_dimension = max_matrix_dimension
    self.return_gpu = return_gpu
    self._stager = PinnedStager()

  def _costs_device(self, d_routes: "torch.Tensor", context: Any) -> "torch.Tensor":
    num, n = int(d_routes.shape[0]), int(d_routes.shape[1])
    costs = torch.empty(num, dtype=torch.float64, device="cuda")
    if num == 0:
      return costs
    ops = operands_for(context)
    before = ops.h2d_bytes
    dist, stride, coords = ops.distance_args(max(n, int(context.dimension)), self.max_matrix_dimension)
    self.h2d_bytes += ops.h2d_bytes - before
    native.call("tspb_tour_cost", ptr(d_routes), num, n, ptr(dist), stride, ptr(coords),
                1 if bool(getattr(context, "return_to_depot", True)) else 0, ptr(costs), stream_handle())
    self.kernel_launches += 1
    return costs

  def _warmup_impl(self, context: Any) -> None:
    self.evaluate_batch(self._warmup_batch(context, rows=1), context)

  def evaluate(self, route: Any, context: Any) -> float:
    return float(np.asarray(self.evaluate_batch(route, context)).reshape(-1)[0])

  @time_strategy
  def evaluate_batch(self, routes: Any, context: Any, return_gpu: bool = False) -> Any:
    require_gpu()
    batch, _ = ensure_routes_batch(routes)
    d_routes, on_dev = _to_device(batch, None if is_device_array(batch) else self._stager)
    if not on_dev:
      self.h2d_bytes += d_routes.numel() * 4
    costs = self._costs_device(d_routes, context)
    if on_dev or return_gpu:
      return costs
    out = _to_host(costs)
    self.d2h_bytes += out.nbytes
    return out

  def assess_batch(self, routes: Any, context: Any, return_gpu: bool = False):
    return tour_assessment(self.evaluate_batch(routes, context, return_gpu=return_gpu))


class SelectionB200Tournament(StrategyBase):
  """k-way tournament with replacement; the first minimum wins (strict `<`)."""

  def __init__(self, k: int = 3, seed: Any = None) -> None:
    if k < 1:
      raise ValueError(f"Tournament size k must be >= 1, got {k}")
    super().__init__(seed)
    self.k = k

  def select(self, population: Any, fitness: Any, context: Any = None) -> Any:
    pop, _ = ensure_routes_batch(population)
    fit = fitness.cpu().numpy() if is_device_array(fitness) else np.asarray(fitness, dtype=np.float64)
    host = pop.cpu().numpy() if is_device_array(pop) else np.asarray(pop)
    rng = resolve_rng(context, self.rng)
    k_eff = min(self.k, len(host))
    idx = rng.choice(len(host), size=k_eff, replace=False)
    return host[int(idx[int(np.argmin(fit[idx]))])].copy()

  @time_strategy
  def select_batch(self, routes: Any, fitness: Any, num_parents: int | None = None, context: Any = None) -> Any:
    require_gpu()
    pop, _ = ensure_routes_batch(routes)
    pop_size = int(pop.shape[0])
    n_select = pop_size if num_parents is None else int(num_parents)
    rng = resolve_rng(context, self.rng)
    cand = rng.integers(0, pop_size, size=(n_select, self.k), dtype=np.int32)
    d_pop, on_dev = _to_device(pop)
    if is_device_array(fitness):
      d_fit = fitness.to(torch.float64).contiguous()
    else:
      d_fit = device_tensor(np.asarray(fitness, dtype=np.float64), torch.float64)
      self.h2d_bytes += d_fit.numel() * 8
    d_cand = device_tensor(cand, torch.int32)
    self.h2d_bytes += cand.nbytes + (0 if on_dev else d_pop.numel() * 4)
    winners = torch.empty(n_select, dtype=torch.int32, device="cuda")
    native.call("tspb_tournament", ptr(d_fit), pop_size, ptr(d_cand), n_select, self.k, ptr(winners), stream_handle())
    out = torch.empty((n_select, int(pop.shape[1])), dtype=torch.int32, device="cuda")
    native.call("tspb_gather_rows", ptr(d_pop), pop_size, int(pop.shape[1]), ptr(winners), n_select, ptr(out), stream_handle())
    self.kernel_launches += 2
    if on_dev:
      return out
    host = out.cpu().numpy()
    self.d2h_bytes += host.nbytes
    return host


class CrossoverB200PermPartiallyMapped(StrategyBase):
  """PMX on pairs (2q, 2q+1) sharing cut points; the odd tail row is copied."""

  _entry = "tspb_pmx"

  def __init__(self, seed: Any = None) -> None:
    super().__init__(seed)

  def _warmup_impl(self, context: Any) -> None:
    self.crossover_batch(self._warmup_batch(context, rows=2), context)

  def crossover(self, parent1: Any, parent2: Any, context: Any = None) -> Any:
    p1 = np.asarray(parent1.cpu() if is_device_array(parent1) else parent1, dtype=np.int32)
    p2 = np.asarray(parent2.cpu() if is_device_array(parent2) else parent2, dtype=np.int32)
    n = len(p1)
    if n <= 1:
      return p1.copy()
    rng = resolve_rng(context, self.rng)
    low, high = resolve_route_bounds(n, context=context, route_sample=p1)
    if high - low < 2:
      return p1.copy()
    if (low, high) != (0, n):
      raise NotImplementedError(f"{type(self).__name__} covers open permutations only")
    cuts = sample_distinct_pairs(rng, 1, low, high)
    pair = np.stack([p1, p2])
    out = self._pmx_device(pair, cuts)
    return out[0]

  def _pmx_device(self, batch: np.ndarray | "torch.Tensor", pairs: np.ndarray):
    d_in, on_dev = _to_device(batch)
    num, n = int(d_in.shape[0]), int(d_in.shape[1])
    first = device_tensor(np.ascontiguousarray(pairs[:, 0]), torch.int32)
    second = device_tensor(np.ascontiguousarray(pairs[:, 1]), torch.int32)
    out = torch.empty_like(d_in)
    status = torch.empty(num, dtype=torch.int32, device="cuda")
    native.call(self._entry, ptr(d_in), num, n, ptr(first), ptr(second), ptr(out), ptr(status), stream_handle())
    self.kernel_launches += 1
    if int(status.max().item()) != 0:
      raise NotPermutationError("crossover_batch: a parent is not a permutation of 0..n-1")
    if on_dev:
      return out
    host = out.cpu().numpy()
    self.d2h_bytes += host.nbytes
    return host

  @time_strategy
  def crossover_batch(self, routes: Any, context: Any = None) -> Any:
    require_gpu()
    batch, was_1d = ensure_routes_batch(routes)
    if was_1d or int(batch.shape[0]) < 2:
      return restore_shape(batch.clone() if is_device_array(batch) else np.array(batch, dtype=np.int32), was_1d)
    num, n = int(batch.shape[0]), int(batch.shape[1])
    sample = None if is_device_array(batch) else batch[0]
    low, high = resolve_route_bounds(n, context=context, route_sample=sample)
    if n <= 1 or high - low < 2:
      return batch.clone() if is_device_array(batch) else np.array(batch, dtype=np.int32)
    if (low, high) != (0, n):
      raise NotImplementedError(f"{type(self).__name__} covers open permutations only")
    rng = resolve_rng(context, self.rng)
    pairs = sample_distinct_pairs(rng, num // 2, low, high)
    if num // 2 == 0:
      return batch.clone() if is_device_array(batch) else np.array(batch, dtype=np.int32)
    if not is_device_array(batch):
      self.h2d_bytes += batch.size * 4
    return self._pmx_device(batch, pairs)


class CrossoverB200PermOrder(CrossoverB200PermPartiallyMapped):
  """Order Crossover on pairs (2q, 2q+1) sharing cut points; the odd tail row is copied.

  The child keeps `p1[c1..c2]`; positions `c2+1, ..., n-1, 0, ..., c1-1` take the genes of
  `p2` not in that segment, in the order met reading `p2` from `c2+1` with wrap-around
  (`CrossoverCPUPermOrder._apply_ox`, `order_crossover.py:52-83`). Draws are those of the
  reference: one `sample_distinct_pairs(rng, N // 2, low, high)` per batch
  (`order_crossover.py:148-150`), one pair per single `crossover` call. Depot-bounded
  (closed) tours raise NotImplementedError.
  """

  _entry = "tspb_ox"


class MutationB200PermInversion(StrategyBase):
  """Reverse `[min(p1,p2), max(p1,p2)]` of every row whose `u < mutation_rate`."""

  _entry = "tspb_inversion"

  def __init__(self, seed: Any = None, candidate_k: int | None = None) -> None:
    super().__init__(seed)
    self.candidate_k = candidate_k

  def mutate(self, individual: Any, mutation_rate: float, context: Any = None) -> Any:
    return self.mutate_batch(individual, mutation_rate, context=context)

  @time_strategy
  def mutate_batch(self, routes: Any, mutation_rate: float, context: Any = None) -> Any:
    require_gpu()
    batch, was_1d = ensure_routes_batch(routes)
    num, n = int(batch.shape[0]), int(batch.shape[1])
    sample = None if is_device_array(batch) else batch[0]
    low, high = resolve_route_bounds(n, context=context, route_sample=sample)
    if high - low < 2:
      out = batch.clone() if is_device_array(batch) else np.array(batch, dtype=np.int32)
      return restore_shape(out, was_1d)
    rng = resolve_rng(context, self.rng)
    probs = rng.random(num)
    if self.candidate_k is not None and self.candidate_k > 0 and context is not None:
      pos1, pos2 = self._candidate_positions(rng, batch, low, high, context)
    else:
      pairs = sample_distinct_pairs(rng, num, low, high)
      pos1, pos2 = pairs[:, 0].copy(), pairs[:, 1].copy()
    d_routes, on_dev = _to_device(batch)
    d_routes = d_routes.clone() if on_dev else d_routes
    if not on_dev:
      self.h2d_bytes += d_routes.numel() * 4
    u = device_tensor(probs, torch.float64)
    d1 = device_tensor(pos1.astype(np.int32), torch.int32)
    d2 = device_tensor(pos2.astype(np.int32), torch.int32)
    native.call(self._entry, ptr(d_routes), num, n, ptr(u), float(mutation_rate), ptr(d1), ptr(d2), stream_handle())
    self.kernel_launches += 1
    if on_dev:
      return restore_shape(d_routes, was_1d)
    host = d_routes.cpu().numpy()
    self.d2h_bytes += host.nbytes
    return restore_shape(host, was_1d)

  def _candidate_positions(self, rng, batch, low, high, context):
    """Second cut from a k-NN neighbour of the first city (`route_helpers.py:183-231`)."""
    cand = candidate_list(context, self.candidate_k)
    host = batch.cpu().numpy() if is_device_array(batch) else np.asarray(batch)
    num = host.shape[0]
    pos1 = np.zeros(num, dtype=np.int32)
    pos2 = np.zeros(num, dtype=np.int32)
    for i in range(num):
      row = np.asarray(host[i], dtype=np.int32)
      first = int(rng.integers(low, high))
      pos1[i] = first
      pos2[i] = _proximity_index(row, first, low, high, cand, rng)
    return pos1, pos2


class MutationB200PermSwap(MutationB200PermInversion):
  """Exchange positions `pos1`, `pos2` of every row whose `u < mutation_rate`.

  Draws follow `MutationCPUPermSwap.mutate_batch` (`swap_mutation.py:65-99`): `rng.random(N)`,
  then the positions of `sample_mutation_positions` (`route_helpers.py:183-231`), uniform
  distinct pairs or, with `candidate_k`, a k-NN neighbour's position for the second one.
  """

  _entry = "tspb_swap"


def _proximity_index(route, anchor, low, high, cand, rng) -> int:
  """`select_proximity_index` (`route_helpers.py:134-180`)."""
  if cand is not None and cand.ndim == 2 and cand.shape[0] > 0:
    node = int(route[anchor])
    if 0 <= node < cand.shape[0]:
      size = max(int(route.size), int(route.max()) + 1)
      positions = np.full(size, -1, dtype=np.int32)
      positions[route] = np.arange(route.size, dtype=np.int32)
      for order in rng.permutation(int(cand.shape[1])):
        nb = int(cand[node, int(order)])
        if nb < 0 or nb >= positions.size:
          continue
        idx = int(positions[nb])
        if idx != anchor and low <= idx < high:
          return idx
  pool = np.array([i for i in range(low, high) if i != anchor], dtype=np.int64)
  if pool.size == 0:
    if low >= high:
      raise ValueError(f"Invalid mutable range [low, high): [{low}, {high}) is empty or degenerate")
    return anchor if low <= anchor < high else low
  return int(rng.choice(pool))
