"""B200 3-opt local search (drop-in for the reference's experimental 3-opt strategy).

`LocalSearchB200ThreeOpt` keeps the constructor and call shape of `LocalSearchGPUThreeOpt`
(`benchmark_scripts/experiments-and-examples/experiment-comparing-3opt-and-2opt/gpu_three_opt.py:280-340`):

- exhaustive `"batch"` / `"naive"` (`candidate_k=None`): exactly what the reference's CPU
  3-opt computes (`cpu_three_opt_refine`, `:256-277`), up to `max_iterations` passes,
  each applying the steepest of all 3-opt moves (seven reconnection cases, first in scan
  order on ties);
- `candidate_k > 0` (any mode) and exhaustive `"multi_move"`: the moves of the
  reference's grid kernels (`three_opt_batch.cu`, `three_opt_multi_move.cu` with
  `three_opt_common.cuh`), which alone define these parts: the candidate-pruned scan with
  `candidate_k` / `inner_candidate_k`, and the greedy disjoint multi_move, both as the
  reference launches them with `threads_per_block` threads per tour (`_improve_grid`,
  `:452-537`). Refinement stops after a pass that applies nothing, where the reference's
  remaining launches change nothing.

Open cyclic TSP tours only (the candidate scan, like the reference's, needs tours of
every city; otherwise it falls back to the exhaustive scan as `_uses_candidates` does).

Host arrays in, host arrays out; CUDA tensors in, CUDA tensors out. Inputs are never
modified. No CPU fallback.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from .. import native
from ..device import PinnedStager, Workspace, operands_for, ptr, require_gpu, stream_handle, torch
from ..errors import NotPermutationError
from ..phase_timer import time_strategy
from ..routes import ensure_routes_batch, restore_shape
from .base import StrategyBase
from .local_search import _topology

MODES = frozenset({"batch", "multi_move", "naive"})
#: Tours above this size keep their tour-ordered matrix in HBM: CTAs per launch then are
#: bounded by this many per SM (each holds n*n int32 of workspace).
_HBM_CTAS_PER_SM = 2


class LocalSearchB200ThreeOpt(StrategyBase):
  """Exhaustive steepest-descent 3-opt, one CTA per tour, every pass on the device."""

  def __init__(self, max_iterations: int = 10, mode: str = "batch", threads_per_block: int = 256,
               max_matrix_dimension: int | None = None, max_shared_tour_cities: int = 4096,
               candidate_k: int | None = None, inner_candidate_k: int | None = None) -> None:
    super().__init__()
    if mode not in MODES:
      raise ValueError(f"Invalid 3-opt mode {mode!r}; expected one of {sorted(MODES)}")
    if max_iterations < 0:
      raise ValueError(f"max_iterations must be >= 0, got {max_iterations}")
    if threads_per_block <= 0:
      raise ValueError(f"threads_per_block must be > 0, got {threads_per_block}")
    if max_shared_tour_cities < 0:
      raise ValueError(f"max_shared_tour_cities must be >= 0, got {max_shared_tour_cities}")
    if inner_candidate_k is not None and inner_candidate_k < 0:
      raise ValueError(f"inner_candidate_k must be >= 0 or None, got {inner_candidate_k}")
    self.mode = mode
    self.max_iterations = max_iterations
    self.threads_per_block = threads_per_block
    self.max_matrix_dimension = max_matrix_dimension
    self.max_shared_tour_cities = max_shared_tour_cities
    self.candidate_k = candidate_k
    self.inner_candidate_k = inner_candidate_k
    self.last_stats: np.ndarray | None = None
    self._workspace = Workspace()
    self._stager = PinnedStager()

  def _warmup_impl(self, context: Any) -> None:
    self.improve_batch(self._warmup_batch(context, rows=1), context)

  def improve(self, route: Any, context: Any) -> Any:
    return self.improve_batch(route, context)

  def _uses_candidates(self, context: Any, n: int) -> bool:
    """`_uses_candidates` of the reference (`gpu_three_opt.py:367-373`) for open tours."""
    if self.candidate_k is None or self.candidate_k <= 0:
      return False
    if str(context.problem.problem_type) in {"CVRP", "OVRP", "DCVRP"}:
      return False
    return n >= int(context.dimension)

  @time_strategy
  def improve_batch(self, routes: Any, context: Any) -> Any:
    require_gpu()
    batch, was_1d = ensure_routes_batch(routes)
    num, n = int(batch.shape[0]), int(batch.shape[1])
    on_device = not isinstance(batch, np.ndarray)
    if n < 4 or self.max_iterations <= 0 or num == 0:
      self.last_stats = np.zeros((num, 3), dtype=np.int64)
      out = batch.clone() if on_device else np.array(batch, dtype=np.int32, copy=True)
      return restore_shape(out, was_1d)
    is_closed, is_cyclic = _topology(context)
    if is_closed or not is_cyclic:
      raise NotImplementedError("LocalSearchB200ThreeOpt covers open (cyclic TSP) tours only")
    if n != int(context.dimension):
      raise ValueError("3-opt tours must visit every city of the problem")
    ops = operands_for(context)
    before = ops.h2d_bytes
    dist, stride, coords = ops.distance_args(n, self.max_matrix_dimension)
    self.h2d_bytes += ops.h2d_bytes - before
    if on_device:
      d_tours = batch.to(torch.int32).contiguous().clone()
    else:
      host = np.ascontiguousarray(batch, dtype=np.int32)
      d_tours = self._stager.upload(host, torch.int32)
      self.h2d_bytes += host.nbytes
    bad = torch.empty(num, dtype=torch.int32, device="cuda")
    native.call("tspb_validate_perm", ptr(d_tours), num, n, ptr(bad), stream_handle())
    self.kernel_launches += 1
    if int(bad.max().item()) != 0:
      raise NotPermutationError("improve_batch: a route is not a permutation of 0..n-1")
    use_cand = self._uses_candidates(context, n)
    if use_cand or self.mode == "multi_move":
      return self._improve_grid(d_tours, num, n, dist, stride, coords, use_cand, context, on_device, was_1d)
    threads = 512 if self.threads_per_block >= 512 else (256 if self.threads_per_block >= 256 else 128)
    import ctypes

    ctas = min(num, _HBM_CTAS_PER_SM * torch.cuda.get_device_properties(0).multi_processor_count)
    need = ctypes.c_size_t(0)
    native.call("tspb_three_opt_workspace_bytes", n, ctas, ctypes.byref(need))
    ws = self._workspace.get(int(need.value)) if need.value else None
    stats = torch.empty((num, 3), dtype=torch.int64, device="cuda")
    status = torch.empty(num, dtype=torch.int32, device="cuda")
    native.call("tspb_three_opt", ptr(d_tours), num, n, ptr(dist), stride, ptr(coords), int(self.max_iterations),
                threads, ptr(ws), int(need.value), ptr(status), ptr(stats), stream_handle())
    self.kernel_launches += 1
    code = int(status.max().item())
    if code != 0:
      raise RuntimeError(f"3-opt kernel reported {native.status_text(code)}")
    return self._finish(d_tours, stats, on_device, was_1d)

  def _improve_grid(self, d_tours, num, n, dist, stride, coords, use_cand, context, on_device, was_1d):
    """Candidate-pruned scan or multi_move with the reference's grid-kernel rules."""
    from ..device import candidate_list

    cand = cand_dist = None
    k = inner = 0
    if use_cand:
      ops = operands_for(context)
      before = ops.h2d_bytes
      tabs = ops.candidates(int(self.candidate_k), candidate_list(context, int(self.candidate_k)), n,
                            self.max_matrix_dimension)
      self.h2d_bytes += ops.h2d_bytes - before
      cand, cand_dist, k = tabs.cand, tabs.cand_dist, int(tabs.k)
      inner = int(self.inner_candidate_k) if self.inner_candidate_k else 0
    stats = torch.empty((num, 3), dtype=torch.int64, device="cuda")
    status = torch.empty(num, dtype=torch.int32, device="cuda")
    native.call("tspb_three_opt_grid", ptr(d_tours), num, n, ptr(dist), stride, ptr(coords), ptr(cand),
                ptr(cand_dist), k, inner, 1 if self.mode == "multi_move" else 0, int(self.threads_per_block),
                int(self.max_iterations), ptr(status), ptr(stats), stream_handle())
    self.kernel_launches += 1
    code = int(status.max().item())
    if code != 0:
      raise RuntimeError(f"3-opt kernel reported {native.status_text(code)}")
    return self._finish(d_tours, stats, on_device, was_1d)

  def _finish(self, d_tours, stats, on_device, was_1d):
    self.last_stats = stats.cpu().numpy()
    if on_device:
      return restore_shape(d_tours, was_1d)
    out = self._stager.download(d_tours)
    self.d2h_bytes += out.nbytes
    return restore_shape(out, was_1d)
