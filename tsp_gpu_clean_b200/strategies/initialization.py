"""B200 initial populations (drop-ins for the reference's initializers).

- `InitializationB200TourNearestNeighbor(k, seed, return_gpu)` mirrors
  `InitializationCPUTourNearestNeighbor` / `InitializationGPUTourNearestNeighbor`
  (`src/algorithms/strategies/initialization/nearest_neighbor_init.py:102-238`): one thread
  per row builds the GRASP tour on the GPU.
- `InitializationB200PermRandom(seed, return_gpu)` mirrors `InitializationCPUPermRandom` /
  `InitializationGPUPermRandom` (`src/algorithms/strategies/initialization/random_init.py:24-120`):
  one CTA per row shuffles the customer list on the GPU.

Both draw their row seeds on the host from `context.rng` exactly as `draw_row_seeds` does
(`src/utils/splitmix64.py:21-25`); each row then follows its own SplitMix64 stream.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from .. import native
from ..device import candidate_list, device_tensor, ptr, require_gpu, stream_handle, torch
from ..phase_timer import time_strategy
from ..problem import resolve_rng
from .base import StrategyBase


def draw_row_seeds(rng: np.random.Generator, population_size: int) -> np.ndarray:
  if population_size <= 0:
    return np.empty(0, dtype=np.uint64)
  return rng.integers(0, np.iinfo(np.int64).max, size=population_size, dtype=np.int64).view(np.uint64)


class InitializationB200TourNearestNeighbor(StrategyBase):
  def __init__(self, k: int = 20, seed: Any = None, return_gpu: bool = False) -> None:
    if isinstance(k, bool) or not isinstance(k, int) or k < 1:
      raise ValueError(f"Candidate-list width k must be >= 1, got {k!r}")
    super().__init__(seed)
    self.k = k
    self.return_gpu = return_gpu
    self._ws = None

  def _warmup_impl(self, context: Any) -> None:
    if context.dimension > 1:
      self.initialize(list(range(context.dimension)), 2, context)

  @time_strategy
  def initialize(self, customers: Any, population_size: int, context: Any = None) -> Any:
    if context is None:
      raise ValueError("InitializationB200TourNearestNeighbor requires a ProblemContext to read the k-NN candidate list")
    if population_size < 0:
      raise ValueError(f"population_size must be >= 0, got {population_size}")
    require_gpu()
    cust = np.ascontiguousarray(customers, dtype=np.int32)
    n = int(cust.size)
    seeds = draw_row_seeds(resolve_rng(context, self.rng), population_size)
    if population_size == 0 or n == 0:
      empty = torch.empty((population_size, n), dtype=torch.int32, device="cuda")
      return empty if self.return_gpu else np.empty((population_size, n), dtype=np.int32)
    cand = np.ascontiguousarray(candidate_list(context, self.k), dtype=np.int32)
    rows, kk = (cand.shape[0], cand.shape[1]) if cand.ndim == 2 else (0, 0)
    max_node = int(cust.max())
    d_cust = device_tensor(cust, torch.int32)
    d_cand = device_tensor(cand if cand.size else np.zeros(1, np.int32), torch.int32)
    d_seeds = torch.from_numpy(seeds.view(np.int64).copy()).to("cuda")
    self.h2d_bytes += cust.nbytes + cand.nbytes + seeds.nbytes
    need = population_size * (n + max_node + 1 + kk) * 4
    if self._ws is None or self._ws.numel() * 4 < need:
      self._ws = torch.empty(max(need // 4, 1), dtype=torch.int32, device="cuda")
    out = torch.empty((population_size, n), dtype=torch.int32, device="cuda")
    native.call("tspb_nn_init", ptr(d_cust), n, ptr(d_cand), rows, kk, ptr(d_seeds), population_size, max_node,
                ptr(self._ws), need, ptr(out), stream_handle())
    self.kernel_launches += 1
    if self.return_gpu:
      return out
    host = out.cpu().numpy()
    self.d2h_bytes += host.nbytes
    return host


class InitializationB200PermRandom(StrategyBase):
  """Uniform random permutations of `customers`, bit-identical to `InitializationCPUPermRandom`
  (Fisher-Yates from the last position down, SplitMix64 bounded draws per row)."""

  def __init__(self, seed: Any = None, return_gpu: bool = False) -> None:
    super().__init__(seed)
    self.return_gpu = return_gpu

  def _warmup_impl(self, context: Any) -> None:
    self.initialize(list(range(max(1, context.dimension))), 2, context)

  @time_strategy
  def initialize(self, customers: Any, population_size: int, context: Any = None) -> Any:
    if population_size < 0:
      raise ValueError(f"population_size must be >= 0, got {population_size}")
    require_gpu()
    cust = np.ascontiguousarray(customers, dtype=np.int32)
    n = int(cust.size)
    seeds = draw_row_seeds(resolve_rng(context, self.rng), population_size)
    if population_size == 0 or n == 0:
      empty = torch.empty((population_size, n), dtype=torch.int32, device="cuda")
      return empty if self.return_gpu else np.empty((population_size, n), dtype=np.int32)
    d_cust = device_tensor(cust, torch.int32)
    d_seeds = torch.from_numpy(seeds.view(np.int64).copy()).to("cuda")
    self.h2d_bytes += cust.nbytes + seeds.nbytes
    out = torch.empty((population_size, n), dtype=torch.int32, device="cuda")
    native.call("tspb_random_init", ptr(d_seeds), population_size, n, ptr(d_cust), ptr(out), stream_handle())
    self.kernel_launches += 1
    if self.return_gpu:
      return out
    host = out.cpu().numpy()
    self.d2h_bytes += host.nbytes
    return host
