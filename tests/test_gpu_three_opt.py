"""Exhaustive 3-opt on the B200 against the reference's CPU 3-opt (`tests/golden/three_opt.npz`)
and the oracle (`oracle/three_opt.py`)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import distances as odist
from oracle import three_opt as o3
from tsp_gpu_clean_b200 import instances

pytestmark = pytest.mark.gpu

TAGS = ["u5", "u6", "u9", "u16", "u40", "lat16", "lat36"]


@pytest.fixture(scope="module")
def torch_mod():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  return torch


def _ctx(coords, **kw):
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  return ProblemContext(Problem.from_coordinates(np.asarray(coords, dtype=np.float64)), seed=0, **kw)


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("resident", [False, True])
def test_three_opt_matches_reference(torch_mod, golden, tag, resident):
  from tsp_gpu_clean_b200.strategies import LocalSearchB200ThreeOpt

  g = golden("three_opt.npz")
  ctx = _ctx(g[f"{tag}_coords"])
  tours = g[f"{tag}_tours"]
  for iters in (1, 3, 1000):
    ls = LocalSearchB200ThreeOpt(max_iterations=iters)
    x = torch_mod.from_numpy(tours.copy()).cuda() if resident else tours.copy()
    out = ls.improve_batch(x, ctx)
    got = out.cpu().numpy() if resident else out
    assert np.array_equal(got, g[f"{tag}_refined{iters}"]), iters
    if not resident:
      assert np.array_equal(x, tours)  # inputs are not modified


def test_three_opt_stats_and_larger_tours_vs_oracle(torch_mod):
  """Smaller tours keep their tour-ordered matrix in shared memory, tours above 220 cities
  in HBM; the distance source is the matrix or FP64 coordinates. Every case equals the
  oracle, and the kernel's pass and move counts equal the oracle refinement's."""
  from tsp_gpu_clean_b200.strategies import LocalSearchB200ThreeOpt

  for n, tours_n, iters, mmd in ((7, 9, 1000, None), (150, 3, 6, None), (221, 2, 3, None), (300, 2, 2, 100)):
    c = instances.clustered_instance(n, 6, 40.0, 300 + n)
    ctx = _ctx(c)
    D = odist.euc2d_matrix(c)
    tours = instances.random_tours(n, tours_n, n)
    ls = LocalSearchB200ThreeOpt(max_iterations=iters, max_matrix_dimension=mmd, threads_per_block=512 if n > 200 else 256)
    got = ls.improve_batch(tours, ctx)
    want, moves = o3.improve_batch(tours, D, iters)
    assert np.array_equal(got, want), n
    assert ls.last_stats[:, 1].tolist() == moves, n
    assert (ls.last_stats[:, 0] >= np.asarray(moves)).all()


def test_three_opt_rejects_what_it_does_not_cover(torch_mod):
  from tsp_gpu_clean_b200.errors import NotPermutationError
  from tsp_gpu_clean_b200.strategies import LocalSearchB200ThreeOpt

  c = instances.uniform_instance(12, 1)
  ctx = _ctx(c)
  t = instances.random_tours(12, 2, 3)
  bad = t.copy()
  bad[1, 3] = bad[1, 4]
  with pytest.raises(NotPermutationError):
    LocalSearchB200ThreeOpt().improve_batch(bad, ctx)
  with pytest.raises(ValueError):
    LocalSearchB200ThreeOpt(mode="oropt")
  short = np.array([[2, 0, 1]], dtype=np.int32)
  assert np.array_equal(LocalSearchB200ThreeOpt().improve_batch(short, _ctx(c[:3])), short)


def test_three_opt_improves_two_opt_local_optima(torch_mod):
  """Tours at a 2-opt local optimum still improve under 3-opt (block moves that 2-opt
  cannot make), and the result equals the oracle's."""
  from tsp_gpu_clean_b200.strategies import LocalSearchB200ThreeOpt, LocalSearchB200TourTwoOpt

  n = 60
  c = instances.uniform_instance(n, 8)
  ctx = _ctx(c)
  D = odist.euc2d_matrix(c)
  tours = instances.random_tours(n, 4, 21)
  two = LocalSearchB200TourTwoOpt(mode="best", max_iterations=10**6).improve_batch(tours, ctx)
  three = LocalSearchB200ThreeOpt(max_iterations=10**6).improve_batch(two, ctx)
  want, _ = o3.improve_batch(two, D, 10**6)
  assert np.array_equal(three, want)
  cost = lambda t: int(D[t, np.roll(t, -1)].sum())  # noqa: E731
  assert sum(cost(t) for t in three) < sum(cost(t) for t in two)
