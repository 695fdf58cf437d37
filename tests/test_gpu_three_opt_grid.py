"""3-opt with the reference's grid-kernel rules (candidate-pruned scan, multi_move) on B200.

`tspb_three_opt_grid` must give the moves of the reference's `three_opt_batch_kernel` /
`three_opt_multi_move_batch_kernel` as `LocalSearchGPUThreeOpt._improve_grid` launches
them: against the kernels' own recorded outputs (`three_opt_kernel.npz`), against the
restatement in `oracle/three_opt_kernel.py` on more shapes (threads per tour 1..256,
k-NN widths, inner widths, tie-heavy lattices, the exhaustive multi_move), and with one
thread per tour against the reference's CPU 3-opt (`three_opt.npz`).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import distances as odist
from oracle import three_opt_kernel as tk
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


def _grid(lib, coords, tours, k, inner, tpb, mode, iters, cand=None):
  """Run tspb_three_opt_grid on host tours; returns (tours, stats)."""
  import torch

  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  n = len(coords)
  D = odist.euc2d_matrix(coords).astype(np.int32)
  d_D = torch.from_numpy(D).cuda()
  d_t = torch.from_numpy(np.ascontiguousarray(tours, dtype=np.int32)).cuda()
  num = len(tours)
  d_c = d_cd = None
  if k > 0:
    if cand is None:
      cand = odist.candidate_list(k, coords=coords)
    cand = np.ascontiguousarray(cand, dtype=np.int32)
    d_c = torch.from_numpy(cand).cuda()
    cd = np.take_along_axis(D, cand.astype(np.int64), axis=1).astype(np.int32)
    d_cd = torch.from_numpy(np.ascontiguousarray(cd)).cuda()
    k = cand.shape[1]
  status = torch.zeros(num, dtype=torch.int32, device="cuda")
  stats = torch.zeros((num, 3), dtype=torch.int64, device="cuda")
  rc = lib.tspb_three_opt_grid(ptr(d_t), num, n, ptr(d_D), n, None, ptr(d_c), ptr(d_cd), k, inner,
                               1 if mode == "multi_move" else 0, tpb, iters, ptr(status), ptr(stats), stream_handle())
  native.check("tspb_three_opt_grid", rc)
  torch.cuda.synchronize()
  assert int(status.max().item()) == 0
  return d_t.cpu().numpy(), stats.cpu().numpy()


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "three_opt_kernel.npz")),
                    reason="three_opt_kernel.npz not recorded yet")
def test_matches_the_reference_kernels(lib, golden):
  g = golden("three_opt_kernel.npz")
  for tag in g["tags"]:
    n, k, inner, tpb, multi, iters, B = (int(v) for v in g[f"{tag}_meta"])
    assert lib.tspb_three_opt_grid_threads(tpb, n) == B
    got, _ = _grid(lib, g[f"{tag}_coords"], g[f"{tag}_in"], k, inner, tpb, "multi_move" if multi else "batch", iters,
                   cand=g[f"{tag}_cand"] if k > 0 else None)
    assert np.array_equal(got, g[f"{tag}_out"]), str(tag)


@pytest.mark.parametrize("mode", ["batch", "multi_move"])
@pytest.mark.parametrize("tpb,k,inner", [(256, 8, 0), (64, 10, 3), (32, 20, 0), (8, 6, 0), (1, 5, 2), (128, 12, 12)])
def test_candidate_scan_vs_oracle(lib, mode, tpb, k, inner):
  coords = instances.clustered_instance(90, 6, 30.0, 700 + tpb + k)
  tours = instances.random_tours(90, 5, 701 + tpb)
  D = odist.euc2d_matrix(coords)
  cand = odist.candidate_list(k, coords=coords)
  iters = 25
  got, st = _grid(lib, coords, tours, k, inner, tpb, mode, iters)
  for t in range(len(tours)):
    want, (passes, moves) = tk.refine(tours[t], D, cand, inner, tpb, mode, iters)
    assert np.array_equal(got[t], want), (mode, tpb, k, inner, t)
    assert (int(st[t, 0]), int(st[t, 1])) == (passes, moves)


def test_candidate_scan_on_lattice_ties(lib):
  side = 9
  coords = np.array([[10.0 * x, 10.0 * y] for x in range(side) for y in range(side)])
  tours = instances.random_tours(len(coords), 4, 710)
  D = odist.euc2d_matrix(coords)
  for mode in ("batch", "multi_move"):
    for tpb in (256, 16):
      cand = odist.candidate_list(8, coords=coords)
      got, _ = _grid(lib, coords, tours, 8, 0, tpb, mode, 30)
      for t in range(len(tours)):
        want, _ = tk.refine(tours[t], D, cand, 0, tpb, mode, 30)
        assert np.array_equal(got[t], want), (mode, tpb, t)


@pytest.mark.parametrize("tpb", [256, 32, 4])
def test_exhaustive_multi_move_vs_oracle(lib, tpb):
  coords = instances.uniform_instance(30, 720 + tpb)
  tours = instances.random_tours(30, 4, 721)
  D = odist.euc2d_matrix(coords)
  got, st = _grid(lib, coords, tours, 0, 0, tpb, "multi_move", 8)
  for t in range(len(tours)):
    want, (passes, moves) = tk.refine(tours[t], D, None, 0, tpb, "multi_move", 8)
    assert np.array_equal(got[t], want), t
    assert (int(st[t, 0]), int(st[t, 1])) == (passes, moves)


def test_one_thread_equals_the_cpu_three_opt(lib, golden):
  """One reference thread per tour scans in the CPU 3-opt's order: multi_move then applies
  the CPU's steepest move each pass (recorded in three_opt.npz)."""
  g = golden("three_opt.npz")
  for tag in ("u9", "u16", "lat16", "u40"):
    for iters in (1, 3, 1000):
      got, _ = _grid(lib, g[f"{tag}_coords"], g[f"{tag}_tours"], 0, 0, 1, "multi_move", iters)
      assert np.array_equal(got, g[f"{tag}_refined{iters}"]), (tag, iters)


def test_large_candidate_tours_stay_permutations_and_match_the_oracle_for_two_passes(lib):
  n = 1500
  coords = instances.clustered_instance(n, 30, 30.0, 730)
  tours = instances.random_tours(n, 2, 731)
  D = odist.euc2d_matrix(coords)
  cand = odist.candidate_list(10, coords=coords)
  got, _ = _grid(lib, coords, tours, 10, 0, 256, "multi_move", 2)
  for t in range(2):
    want, _ = tk.refine(tours[t], D, cand, 0, 256, "multi_move", 2)
    assert np.array_equal(got[t], want)
  long_run, st = _grid(lib, coords, tours, 10, 0, 256, "batch", 10**6)
  for t in range(2):
    assert np.array_equal(np.sort(long_run[t]), np.arange(n))
    before = D[tours[t], np.roll(tours[t], -1)].sum()
    after = D[long_run[t], np.roll(long_run[t], -1)].sum()
    assert after < before and st[t, 1] == st[t, 0] - 1  # one move per pass until none improves


def test_strategy_runs_candidate_and_multi_move(lib):
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext
  from tsp_gpu_clean_b200.strategies import LocalSearchB200ThreeOpt

  coords = instances.uniform_instance(70, 740)
  ctx = ProblemContext(Problem.from_coordinates(coords), seed=0)
  tours = instances.random_tours(70, 3, 741)
  D = odist.euc2d_matrix(coords)
  cand = ctx.get_cpu_candidate_list(8)
  for mode in ("batch", "multi_move"):
    ls = LocalSearchB200ThreeOpt(max_iterations=20, mode=mode, candidate_k=8, inner_candidate_k=4)
    got = ls.improve_batch(tours, ctx)
    for t in range(3):
      want, _ = tk.refine(tours[t], D, cand, 4, 256, mode, 20)
      assert np.array_equal(got[t], want), (mode, t)
  ls = LocalSearchB200ThreeOpt(max_iterations=5, mode="multi_move")
  got = ls.improve_batch(tours, ctx)
  for t in range(3):
    want, _ = tk.refine(tours[t], D, None, 0, 256, "multi_move", 5)
    assert np.array_equal(got[t], want)
