"""Per-phase wall-clock accounting, mirroring `src/utils/phase_timer.py` of the reference.

`PhaseTimer.measure(name, fn, *args)` accumulates host milliseconds per phase and
`summary()` returns `{phase: {"total_ms", "calls", "mean_ms"}}`; `time_strategy`
records `last_elapsed_ms` / `total_elapsed_ms` / `call_count` on a strategy.
"""

from __future__ import annotations

import functools
import time
from collections import defaultdict
from typing import Any, Callable


class PhaseTimer:
  def __init__(self, enabled: bool = True) -> None:
    self.enabled = enabled
    self._total: dict[str, float] = defaultdict(float)
    self._calls: dict[str, int] = defaultdict(int)

  def reset(self) -> None:
    self._total.clear()
    self._calls.clear()

  def measure(self, name: str, fn: Callable[..., Any], *args: Any, **kwargs: Any) -> Any:
    if not self.enabled:
      return fn(*args, **kwargs)
    t0 = time.perf_counter()
    try:
      return fn(*args, **kwargs)
    finally:
      self._total[name] += (time.perf_counter() - t0) * 1e3
      self._calls[name] += 1

  def summary(self) -> dict[str, dict[str, float | int]]:
    return {
      k: {"total_ms": v, "calls": self._calls[k], "mean_ms": v / max(1, self._calls[k])} for k, v in self._total.items()
    }


def time_strategy(fn: Callable[..., Any]) -> Callable[..., Any]:
  @functools.wraps(fn)
  def wrapper(self, *args, **kwargs):
    t0 = time.perf_counter()
    try:
      return fn(self, *args, **kwargs)
    finally:
      ms = (time.perf_counter() - t0) * 1e3
      self.last_elapsed_ms = ms
      self.total_elapsed_ms = getattr(self, "total_elapsed_ms", 0.0) + ms
      self.call_count = getattr(self, "call_count", 0) + 1

  return wrapper
