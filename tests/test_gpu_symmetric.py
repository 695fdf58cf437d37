"""TSPB_MODE_SYMMETRIC: after a move the candidate scan takes a reversed window's new
out-edges from the old ones. On symmetric distances that gives the same tours and counts
as reading every edge again; asymmetric matrices keep the exact per-edge path (no flag),
which must still match the oracle's directional edge costs."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import distances as odist
from oracle import two_opt as otwo
from tsp_gpu_clean_b200 import instances

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  from tsp_gpu_clean_b200 import native

  return native.load_library()


def _run(lib, coords, tours, k, mode, threads, flag, incremental, packed=True):
  import torch

  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import operands_for, ptr, stream_handle
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  n = len(coords)
  ctx = ProblemContext(Problem.from_coordinates(coords), seed=0)
  ops = operands_for(ctx)
  dist, stride, _ = ops.distance_args(n, None)
  assert ops.symmetric
  tabs = ops.candidates(k, ctx.get_cpu_candidate_list(k), n)
  t = torch.from_numpy(np.ascontiguousarray(tours, dtype=np.int32)).cuda()
  num = len(tours)
  stats = torch.zeros((num, 4), dtype=torch.int64, device="cuda")
  status = torch.zeros(num, dtype=torch.int32, device="cuda")
  use_rev = incremental and mode == "first"
  code = native.MODE_CODES[mode] | (native.TSPB_MODE_SYMMETRIC if flag else 0)
  native.check("tspb_two_opt", lib.tspb_two_opt(
    ptr(t), num, n, ptr(dist), stride, None, ptr(tabs.cand), ptr(tabs.cand_dist),
    ptr(tabs.rev_off) if use_rev else None, ptr(tabs.rev_idx) if use_rev else None,
    ptr(tabs.packed) if packed else None, tabs.k, code, 10**9, threads, ptr(stats), ptr(status), None, 0,
    stream_handle()))
  torch.cuda.synchronize()
  assert int(status.max().item()) == 0
  return t.cpu().numpy(), stats.cpu().numpy()


@pytest.mark.parametrize("mode,incremental", [("best", False), ("first", False), ("first", True)])
@pytest.mark.parametrize("threads", [64, 128, 256])
def test_flag_gives_the_same_refinement(lib, mode, incremental, threads):
  """Random tours of a 700-city clustered instance: windows from 2 to n positions, some
  reaching the last position (wrap-around successor), many wider than the CTA."""
  coords = instances.clustered_instance(700, 12, 30.0, 801)
  tours = instances.random_tours(700, 24, 802 + threads)
  for k in (8, 20):
    a, sa = _run(lib, coords, tours, k, mode, threads, False, incremental)
    b, sb = _run(lib, coords, tours, k, mode, threads, True, incremental)
    assert np.array_equal(a, b), (k, mode)
    # passes, pairs and moves; the gains computed (column 3) depend on thread timing in
    # first mode, whose threads stop once a lower improving index is published
    assert np.array_equal(sa[:, :3], sb[:, :3]), (k, mode)


def test_flag_matches_the_oracle_on_a_lattice(lib):
  """Tie-heavy integer lattice: equal gains everywhere, both modes, against the oracle."""
  side = 12
  coords = np.array([[10.0 * x, 10.0 * y] for x in range(side) for y in range(side)])
  n = len(coords)
  tours = instances.random_tours(n, 6, 803)
  D = odist.euc2d_matrix(coords)
  cand = odist.candidate_list(10, coords=coords)
  for mode in ("best", "first"):
    got, st = _run(lib, coords, tours, 10, mode, 128, True, mode == "first")
    want, wst = otwo.improve_batch(tours, D, cand, mode, 10**9)
    assert np.array_equal(got, want), mode
    assert np.array_equal(st[:, :3], wst), mode


def test_asymmetric_matrix_keeps_the_per_edge_path(lib):
  """An asymmetric explicit matrix: the operands report it, the strategy leaves the flag
  off, and every mode matches the oracle's directional edge costs."""
  from tsp_gpu_clean_b200.device import operands_for
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext
  from tsp_gpu_clean_b200.strategies.local_search import LocalSearchB200TourTwoOpt

  rng = np.random.default_rng(804)
  n = 90
  D = rng.integers(1, 1000, size=(n, n)).astype(np.int32)
  np.fill_diagonal(D, 0)
  assert not np.array_equal(D, D.T)
  tours = instances.random_tours(n, 5, 805)
  ctx = ProblemContext(Problem.from_matrix(D), seed=0)
  assert operands_for(ctx).symmetric is False
  # a bounded number of passes: with asymmetric costs the reference's gain ignores the
  # reversed segment's direction, so its moves need not shorten the tour or stop
  for k in (None, 12):
    cand = odist.candidate_list(k, distances=D) if k else None
    for mode in ("best", "first", "multi_move"):
      ls = LocalSearchB200TourTwoOpt(max_iterations=40, mode=mode, candidate_k=k)
      got = ls.improve_batch(tours, ctx)
      want, _ = otwo.improve_batch(tours, D, cand, mode, 40)
      assert np.array_equal(got, want), (k, mode)
  sym = ProblemContext(Problem.from_matrix(np.minimum(D, D.T)), seed=0)
  assert operands_for(sym).symmetric is True
