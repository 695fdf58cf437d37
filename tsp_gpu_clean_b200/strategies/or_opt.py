"""B200 Or-opt local search (a new operator beside the 2-opt and 3-opt strategies).

The reference has no Or-opt strategy. `LocalSearchB200OrOpt` gives the segment-relocation
neighbourhood the reference's `LocalSearchStrategy` shape (`improve` / `improve_batch`,
`src/protocols/algorithm_strategies.py:145-172`) and the conventions of its candidate
2-opt (`src/algorithms/strategies/local_search/two_opt.py:97-149, 347-367`): the
context's k-NN table (`candidate_k`), open cyclic tours with position 0 fixed, exact
integer deltas, best improvement with the first move in scan order on ties, and up to
`max_iterations` passes. A move takes one to `max_segment` consecutive cities and
re-inserts them, forward or reversed, after a k-NN candidate of the segment's first
(forward) or last (reversed) city; `tspb_or_opt` in `include/tspb.h` states the scan key.

Host arrays in, host arrays out; CUDA tensors in, CUDA tensors out. Inputs are never
modified. No CPU fallback.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from .. import native
from ..device import PinnedStager, candidate_list, operands_for, ptr, require_gpu, stream_handle, torch
from ..errors import NotPermutationError
from ..phase_timer import time_strategy
from ..routes import ensure_routes_batch, restore_shape
from .base import StrategyBase
from .local_search import _topology


class LocalSearchB200OrOpt(StrategyBase):
  """Candidate-list Or-opt (segments of 1..max_segment cities), one CTA per tour."""

  def __init__(self, max_iterations: int = 10, candidate_k: int = 20, max_segment: int = 3,
               threads_per_block: int = 128, max_matrix_dimension: int | None = None) -> None:
    super().__init__()
    if max_iterations < 0:
      raise ValueError(f"max_iterations must be >= 0, got {max_iterations}")
    if candidate_k is None or candidate_k < 1:
      raise ValueError(f"candidate_k must be >= 1, got {candidate_k}")
    if not 1 <= max_segment <= 8:
      raise ValueError(f"max_segment must be in 1..8, got {max_segment}")
    if threads_per_block <= 0:
      raise ValueError(f"threads_per_block must be > 0, got {threads_per_block}")
    self.max_iterations = max_iterations
    self.candidate_k = candidate_k
    self.max_segment = max_segment
    self.threads_per_block = threads_per_block
    self.max_matrix_dimension = max_matrix_dimension
    self.last_stats: np.ndarray | None = None
    self._stager = PinnedStager()

  def _warmup_impl(self, context: Any) -> None:
    self.improve_batch(self._warmup_batch(context, rows=1), context)

  def improve(self, route: Any, context: Any) -> Any:
    return self.improve_batch(route, context)

  @time_strategy
  def improve_batch(self, routes: Any, context: Any) -> Any:
    require_gpu()
    batch, was_1d = ensure_routes_batch(routes)
    num, n = int(batch.shape[0]), int(batch.shape[1])
    on_device = not isinstance(batch, np.ndarray)
    if n < 3 or self.max_iterations <= 0 or num == 0:
      self.last_stats = np.zeros((num, 3), dtype=np.int64)
      out = batch.clone() if on_device else np.array(batch, dtype=np.int32, copy=True)
      return restore_shape(out, was_1d)
    is_closed, is_cyclic = _topology(context)
    if is_closed or not is_cyclic:
      raise NotImplementedError("LocalSearchB200OrOpt covers open (cyclic TSP) tours only")
    if n != int(context.dimension):
      raise ValueError("Or-opt tours must visit every city of the problem")
    lib = native.load_library()
    if n > int(lib.tspb_or_opt_max_n()):
      raise ValueError(f"Or-opt keeps a tour in shared memory: n={n} exceeds {int(lib.tspb_or_opt_max_n())}")
    ops = operands_for(context)
    before = ops.h2d_bytes
    dist, stride, coords = ops.distance_args(n, self.max_matrix_dimension)
    tabs = ops.candidates(int(self.candidate_k), candidate_list(context, int(self.candidate_k)), n,
                          self.max_matrix_dimension)
    self.h2d_bytes += ops.h2d_bytes - before
    if on_device:
      d_tours = batch.to(torch.int32).contiguous().clone()
    else:
      host = np.ascontiguousarray(batch, dtype=np.int32)
      d_tours = self._stager.upload(host, torch.int32)
      self.h2d_bytes += host.nbytes
    # 128 is fastest on the 1024-tour, n = 1000 workload (27.9 ms vs 32.3 ms at 256, 30.3 at 512)
    threads = 512 if self.threads_per_block >= 512 else (256 if self.threads_per_block >= 256 else 128)
    stats = torch.empty((num, 3), dtype=torch.int64, device="cuda")
    status = torch.empty(num, dtype=torch.int32, device="cuda")
    native.call("tspb_or_opt", ptr(d_tours), num, n, ptr(dist), stride, ptr(coords), ptr(tabs.cand),
                ptr(tabs.cand_dist), ptr(tabs.packed), int(tabs.k), int(self.max_segment), int(self.max_iterations),
                threads, ptr(status), ptr(stats), stream_handle())
    self.kernel_launches += 1
    code = int(status.max().item())
    if code == native.TSPB_ERR_NOT_PERMUTATION:
      raise NotPermutationError("improve_batch: a route is not a permutation of 0..n-1")
    if code != 0:
      raise RuntimeError(f"Or-opt kernel reported {native.status_text(code)}")
    self.last_stats = stats.cpu().numpy()
    if on_device:
      return restore_shape(d_tours, was_1d)
    out = self._stager.download(d_tours)
    self.d2h_bytes += out.nbytes
    return restore_shape(out, was_1d)
