"""Strategy base class and the route assessment record.

`StrategyBase` mirrors `src/algorithms/strategies/base.py:37-155` of the reference:
per-instance telemetry counters (`h2d_bytes`, `d2h_bytes`, `kernel_launches`, the
`@time_strategy` timers) and a `warmup` template that restores every counter and
both RNG states afterwards. `RouteAssessment` mirrors the record of
`src/protocols/vrp_strategies.py` (feasible, zero-violation rows for TSP tours).
"""

from __future__ import annotations

import copy
from dataclasses import dataclass
from typing import Any

import numpy as np

from ..problem import make_rng


@dataclass
class RouteAssessment:
  objectives: Any
  travel_costs: Any
  is_feasible: Any
  violations: Any
  normalized_violations: Any
  raw_violation_components: Any = None
  num_vehicles: Any = None


def tour_assessment(costs: Any) -> RouteAssessment:
  """Feasible assessment of Hamiltonian tours (`tour_cost.py:68-82`)."""
  from ..device import is_device_array, torch

  if is_device_array(costs):
    c = costs.to(torch.float64)
    m = c.shape[0]
    z = torch.zeros(m, dtype=torch.float64, device=c.device)
    return RouteAssessment(c, c, torch.ones(m, dtype=torch.bool, device=c.device), z, z.clone(),
                           torch.zeros((m, 3), dtype=torch.float64, device=c.device),
                           torch.ones(m, dtype=torch.int32, device=c.device))
  c = np.asarray(costs, dtype=np.float64)
  m = c.shape[0]
  z = np.zeros(m, dtype=np.float64)
  return RouteAssessment(c, c, np.ones(m, dtype=bool), z, z.copy(), np.zeros((m, 3)), np.ones(m, dtype=np.int32))


class StrategyBase:
  def __init__(self, seed: Any = None) -> None:
    self.seed = seed
    self.rng = make_rng(seed)
    self.h2d_bytes = 0
    self.d2h_bytes = 0
    self.kernel_launches = 0
    self.last_elapsed_ms = 0.0
    self.total_elapsed_ms = 0.0
    self.call_count = 0

  def reset_metrics(self) -> None:
    self.h2d_bytes = 0
    self.d2h_bytes = 0
    self.kernel_launches = 0

  def warmup(self, context: Any) -> None:
    """Run `_warmup_impl` and restore telemetry and RNG state (`base.py:83-118`)."""
    saved = (self.h2d_bytes, self.d2h_bytes, self.kernel_launches, self.last_elapsed_ms, self.total_elapsed_ms,
             self.call_count)
    self_rng = copy.deepcopy(self.rng.bit_generator.state)
    ctx_rng = getattr(context, "rng", None)
    ctx_state = copy.deepcopy(ctx_rng.bit_generator.state) if ctx_rng is not None else None
    ctx_h2d = getattr(context, "h2d_bytes", None)
    try:
      self._warmup_impl(context)
    finally:
      (self.h2d_bytes, self.d2h_bytes, self.kernel_launches, self.last_elapsed_ms, self.total_elapsed_ms,
       self.call_count) = saved
      self.rng.bit_generator.state = self_rng
      if ctx_state is not None:
        ctx_rng.bit_generator.state = ctx_state
      if ctx_h2d is not None:
        context.h2d_bytes = ctx_h2d

  def _warmup_impl(self, context: Any) -> None:
    del context

  def canonicalize_route(self, route: Any, context: Any) -> np.ndarray:
    from ..device import is_device_array

    if is_device_array(route):
      return route.detach().cpu().numpy().astype(np.int32, copy=True)
    return np.asarray(route, dtype=np.int32).copy()

  @staticmethod
  def _warmup_batch(context: Any, rows: int = 2) -> np.ndarray:
    return np.tile(np.arange(context.dimension, dtype=np.int32), (rows, 1))
