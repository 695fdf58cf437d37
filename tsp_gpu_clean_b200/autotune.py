"""Launch-shape autotuner for the uneven batch, with a JSON cache.

A shape key names what the best launch depends on: the device, the kernel, the size
bucket, the distance source, the 2-opt mode/k/passes and the number of work units
(rounded up to a power of two). `choose` measures every candidate once per key with the
caller's probe (CUDA-event time of a representative launch) and caches the winner;
later runs with the same key reuse it without measuring. The cache lives in memory and,
when a path is given (or TSPB_TUNE_CACHE is set), in a JSON file.
"""

from __future__ import annotations

import json
import os
import threading
from typing import Callable, Sequence


def _pow2_ceil(v: int) -> int:
  v = max(int(v), 1)
  return 1 << (v - 1).bit_length()


class BatchAutotuner:
  def __init__(self, cache_path: str | None = None, enabled: bool = True) -> None:
    self.cache_path = cache_path if cache_path is not None else os.environ.get("TSPB_TUNE_CACHE")
    self.enabled = enabled
    self._lock = threading.Lock()
    self.entries: dict[str, dict] = {}
    self.measured = 0
    if self.cache_path and os.path.exists(self.cache_path):
      try:
        with open(self.cache_path) as f:
          data = json.load(f)
        if isinstance(data, dict):
          self.entries.update({k: v for k, v in data.items() if isinstance(v, dict) and "choice" in v})
      except (OSError, ValueError):
        pass

  @staticmethod
  def key(device: str, kernel: str, **shape) -> str:
    if "units" in shape:
      shape = dict(shape, units=_pow2_ceil(shape["units"]))
    parts = [device, kernel] + [f"{k}={shape[k]}" for k in sorted(shape)]
    return "|".join(str(p) for p in parts)

  def choose(self, key: str, candidates: Sequence[int], probe: Callable[[int], float]) -> int:
    """The cached choice for `key`, else the candidate with the smallest probe time."""
    cands = list(candidates)
    if not cands:
      raise ValueError("no launch candidates to choose from")
    with self._lock:
      hit = self.entries.get(key)
    if hit is not None and hit["choice"] in cands:
      return int(hit["choice"])
    if not self.enabled or len(cands) == 1:
      return int(cands[0]) if len(cands) == 1 else int(cands[len(cands) // 2])
    times = {}
    for c in cands:
      times[c] = float(probe(c))
      self.measured += 1
    best = min(cands, key=lambda c: (times[c], c))
    with self._lock:
      self.entries[key] = {"choice": int(best), "ms": {str(c): round(t, 4) for c, t in times.items()}}
    self.save()
    return int(best)

  def save(self) -> None:
    if not self.cache_path:
      return
    with self._lock:
      data = dict(self.entries)
    d = os.path.dirname(os.path.abspath(self.cache_path))
    os.makedirs(d, exist_ok=True)
    tmp = f"{self.cache_path}.tmp{os.getpid()}"
    with open(tmp, "w") as f:
      json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, self.cache_path)
