"""B200 2-opt local search strategy (drop-in for the reference's 2-opt strategies).

`LocalSearchB200TourTwoOpt` keeps the constructor and call shape of
`LocalSearchCPUTourTwoOpt` / `LocalSearchGPUTourTwoOpt`
(`src/algorithms/strategies/local_search/two_opt.py:279-301, 656-697`) and the
results of the CPU acceptance rules bit for bit: `mode` is `"best"`, `"first"`,
`"multi_move"` or `"batch"` (the reference's GPU name for the best-improvement
kernel), `max_iterations` bounds the passes, and `candidate_k` restricts the
second break point to the k nearest neighbours of the first city.

Host arrays in, host arrays out (H2D, one kernel launch for every pass of every
tour, D2H); CUDA tensors in, CUDA tensors out without host copies. Inputs are
never modified. Without a CUDA device the call raises `GPUUnavailableError`
(`two_opt.py:746-754`); there is no CPU fallback.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from .. import native
from ..device import (
  PinnedStager,
  Workspace,
  auto_threads,
  candidate_list,
  operands_for,
  ptr,
  require_gpu,
  stream_handle,
  torch,
)
from ..errors import NotPermutationError
from ..phase_timer import time_strategy
from ..routes import ensure_routes_batch, restore_shape
from .base import StrategyBase

MODES = frozenset({"best", "first", "multi_move", "batch"})


def _topology(context: Any) -> tuple[bool, bool]:
  """`(is_closed, is_cyclic)` as in `_resolve_topology` (`two_opt.py:97-114`)."""
  is_closed = bool(getattr(context, "is_closed", False))
  if is_closed:
    return True, False
  return False, bool(getattr(context, "return_to_depot", True))


class LocalSearchB200TourTwoOpt(StrategyBase):
  """2-opt on B200: persistent CTA per tour, all passes on device."""

  def __init__(
    self,
    max_iterations: int = 10,
    mode: str = "best",
    candidate_k: int | None = None,
    threads_per_block: int | None = None,
    max_matrix_dimension: int | None = None,
  ) -> None:
    super().__init__()
    if mode not in MODES:
      raise ValueError(f"Invalid 2-opt B200 mode {mode!r}; expected one of {sorted(MODES)}")
    if max_iterations < 0:
      raise ValueError(f"max_iterations must be >= 0, got {max_iterations}")
    self.mode = mode
    self.max_iterations = max_iterations
    self.candidate_k = candidate_k
    self.threads_per_block = threads_per_block
    self.max_matrix_dimension = max_matrix_dimension
    self.collect_stats = True
    #: candidate best/first kernel: "scan" (full rescan, packed k-NN words), "scan_unpacked"
    #: (same kernel, separate id/distance arrays) or "cached" (exact incremental row keys).
    #: All give identical results; the choice is a performance knob.
    self.kernel = "scan"
    #: first mode on the scan kernel: restart each pass from the entries a move can have
    #: changed and the move's row (same results as rescanning from entry 0).
    self.incremental_first = True
    self.last_stats: np.ndarray | None = None
    self._workspace = Workspace()
    self._stager = PinnedStager()

  def _warmup_impl(self, context: Any) -> None:
    self.improve_batch(self._warmup_batch(context, rows=1), context)

  def _candidate_table(self, context: Any, n: int, host_batch: np.ndarray | None) -> np.ndarray | None:
    """`_resolve_candidates` (`two_opt.py:117-149`) for the cyclic TSP topology."""
    k = self.candidate_k
    if k is None or k <= 0:
      return None
    if n != int(context.dimension):
      return None
    if str(context.problem.problem_type) in {"CVRP", "OVRP", "DCVRP"}:
      return None
    table = candidate_list(context, k)
    if host_batch is not None and host_batch.size and int(host_batch.max()) >= table.shape[0]:
      return None
    return table

  def improve(self, route: Any, context: Any) -> Any:
    return self.improve_batch(route, context)

  @time_strategy
  def improve_batch(self, routes: Any, context: Any) -> Any:
    require_gpu()
    batch, was_1d = ensure_routes_batch(routes)
    num, n = int(batch.shape[0]), int(batch.shape[1])
    on_device = not isinstance(batch, np.ndarray)
    if n < 4 or self.max_iterations <= 0 or num == 0:
      self.last_stats = np.zeros((num, 4), dtype=np.int64)
      out = batch.clone() if on_device else np.array(batch, dtype=np.int32, copy=True)
      return restore_shape(out, was_1d)
    is_closed, is_cyclic = _topology(context)
    if is_closed or not is_cyclic:
      raise NotImplementedError("LocalSearchB200TourTwoOpt covers cyclic TSP tours only")
    host = None if on_device else np.ascontiguousarray(batch, dtype=np.int32)
    table = self._candidate_table(context, n, host)
    ops = operands_for(context)
    before = ops.h2d_bytes
    dist, stride, coords = ops.distance_args(n, self.max_matrix_dimension)
    tabs = None
    k = 0
    if table is not None:
      tabs = ops.candidates(int(self.candidate_k), table, n, self.max_matrix_dimension)
      k = tabs.k
      if k == 0:
        tabs = None
    self.h2d_bytes += ops.h2d_bytes - before

    if on_device:
      d_tours = batch.to(torch.int32).contiguous().clone()
    else:
      d_tours = self._stager.upload(host, torch.int32)
      self.h2d_bytes += host.nbytes
    mode = native.MODE_CODES[self.mode]
    if dist is not None and ops.symmetric:
      mode |= native.TSPB_MODE_SYMMETRIC  # a move's out-edges from the old ones (include/tspb.h)
    threads = int(self.threads_per_block) if self.threads_per_block else auto_threads(num)
    ws_bytes = native.load_library().tspb_two_opt_workspace_bytes(num, n, k, mode, threads)
    ws = self._workspace.get(int(ws_bytes))
    stats = torch.empty((num, 4), dtype=torch.int64, device="cuda") if self.collect_stats else None
    status = torch.empty(num, dtype=torch.int32, device="cuda")
    cand = tabs.cand if tabs is not None else None
    cand_dist = tabs.cand_dist if tabs is not None else None
    cached = tabs is not None and self.kernel == "cached"
    packed = tabs.packed if tabs is not None and self.kernel == "scan" else None
    use_rev = cached or (packed is not None and self.mode == "first" and self.incremental_first)
    rev_off = tabs.rev_off if use_rev else None
    rev_idx = tabs.rev_idx if use_rev else None
    native.call(
      "tspb_two_opt", ptr(d_tours), num, n, ptr(dist), stride, ptr(coords), ptr(cand), ptr(cand_dist), ptr(rev_off),
      ptr(rev_idx), ptr(packed), k, mode,
      int(self.max_iterations), threads, ptr(stats), ptr(status), ptr(ws), int(ws_bytes),
      stream_handle(),
    )
    self.kernel_launches += 1
    bad = int(status.max().item())
    if bad != 0:
      if bad == native.TSPB_ERR_NOT_PERMUTATION:
        raise NotPermutationError("improve_batch: a route is not a permutation of 0..n-1 (candidate mode)")
      raise ValueError(f"improve_batch: kernel rejected a route ({native.status_text(bad)})")
    self.last_stats = stats.cpu().numpy() if stats is not None else None
    if on_device:
      return restore_shape(d_tours, was_1d)
    out = self._stager.download(d_tours)
    self.d2h_bytes += out.nbytes
    return restore_shape(out, was_1d)
