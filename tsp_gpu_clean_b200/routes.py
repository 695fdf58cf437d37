"""Route batch helpers and the host-side random draws shared by every strategy.

Mirrors `src/utils/route_helpers.py` of the reference for the TSP path:
`ensure_routes_batch` (:234-258), `resolve_route_bounds` (:30-71),
`sample_distinct_pairs` (:74-108). Host arrays are NumPy; device arrays are CUDA
torch tensors (the reference's CuPy arrays play that role there).
"""

from __future__ import annotations

from typing import Any

import numpy as np

from .device import is_device_array, torch


def ensure_routes_batch(routes: Any) -> tuple[Any, bool]:
  if is_device_array(routes):
    if routes.ndim == 1:
      return routes.reshape(1, -1), True
    if routes.ndim == 2:
      return routes, False
    raise ValueError(f"Expected 1D route or 2D routes batch, got array with ndim={routes.ndim}")
  if not hasattr(routes, "ndim"):
    routes = np.asarray(routes, dtype=np.int32)
  if routes.ndim == 1:
    return routes.reshape(1, -1), True
  if routes.ndim == 2:
    return routes, False
  raise ValueError(f"Expected 1D route or 2D routes batch, got array with ndim={routes.ndim}")


def restore_shape(batch: Any, was_1d: bool) -> Any:
  return batch[0] if was_1d else batch


def to_device_routes(batch: Any) -> tuple["torch.Tensor", bool]:
  """`(contiguous int32 CUDA tensor, was_on_device)`; host arrays are copied H2D."""
  if is_device_array(batch):
    t = batch if batch.dtype == torch.int32 else batch.to(torch.int32)
    return t.contiguous(), True
  host = np.ascontiguousarray(batch, dtype=np.int32)
  return torch.from_numpy(host).to("cuda"), False


def resolve_route_bounds(n: int, context: Any = None, route_sample: Any = None) -> tuple[int, int]:
  """Mutable slice `[low, high)`: `(0, n)` for open permutations, `(1, n-1)` for depot-bounded."""
  if route_sample is not None and n > 2 and not is_device_array(route_sample):
    sample = np.asarray(route_sample)
    if sample.size == n and int(sample[0]) == int(sample[-1]):
      return 1, n - 1
  if context is not None:
    closed = bool(getattr(context, "is_closed", False))
    if n == int(getattr(context, "dimension", -1)) - 1 and closed:
      return 0, n
    return (1, n - 1) if closed else (0, n)
  if route_sample is not None:
    if is_device_array(route_sample):
      closed = n > 2 and int(route_sample[0]) == int(route_sample[-1])
      return (1, n - 1) if closed else (0, n)
    return 0, n
  return 1, n - 1


def sample_distinct_pairs(rng: np.random.Generator, num_pairs: int, low: int, high: int) -> np.ndarray:
  """`num_pairs` ordered distinct pairs from `[low, high)`: `v = v' + (v' >= u)`."""
  if high - low < 2:
    raise ValueError(f"Need at least two distinct integers in [{low}, {high})")
  if num_pairs <= 0:
    return np.empty((0, 2), dtype=np.int32)
  first = rng.integers(low, high, size=num_pairs, dtype=np.int32)
  shifted = rng.integers(low, high - 1, size=num_pairs, dtype=np.int32)
  second = shifted + (shifted >= first).astype(np.int32)
  return np.stack((first, second), axis=1).astype(np.int32, copy=False)
