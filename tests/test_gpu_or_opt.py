"""Or-opt on the B200 (`tspb_or_opt`, `LocalSearchB200OrOpt`) against the oracle
(`oracle/or_opt.py`): tours, pass / move / evaluated counts, edge sizes, lattice ties, both
distance sources, resident and host arrays, and the error paths."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import distances as odist
from oracle import or_opt as oo
from tsp_gpu_clean_b200 import instances

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  return torch


def _ctx(coords):
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  return ProblemContext(Problem.from_coordinates(np.asarray(coords, dtype=np.float64)), seed=0)


def _tours(rng, n, m):
  return np.stack([np.concatenate([[0], 1 + rng.permutation(n - 1)]) for _ in range(m)]).astype(np.int32)


def _check(ls, ctx, coords, tours, k, S, iters):
  from tsp_gpu_clean_b200.device import candidate_list

  out = ls.improve_batch(tours, ctx)
  D = odist.euc2d_matrix(coords)
  cand = candidate_list(ctx, k)
  for t in range(tours.shape[0]):
    want, passes, moves, evaluated = oo.refine(tours[t], D, cand, iters, S)
    assert np.array_equal(out[t], want), t
    assert ls.last_stats[t].tolist() == [passes, moves, evaluated], t
  return out


@pytest.mark.parametrize("n,k,S,iters,threads", [(3, 2, 3, 10, 256), (4, 3, 3, 10, 128), (5, 4, 2, 10, 256),
                                                 (9, 8, 3, 1000, 256), (40, 10, 3, 1000, 128),
                                                 (131, 20, 3, 7, 256), (250, 7, 1, 1000, 512),
                                                 (400, 20, 2, 40, 512)])
def test_or_opt_matches_oracle(torch_mod, n, k, S, iters, threads):
  from tsp_gpu_clean_b200.strategies import LocalSearchB200OrOpt

  rng = np.random.default_rng(n * 7 + S)
  coords = instances.uniform_instance(n, 500 + n)
  ctx = _ctx(coords)
  tours = _tours(rng, n, 5)
  keep = tours.copy()
  ls = LocalSearchB200OrOpt(max_iterations=iters, candidate_k=k, max_segment=S, threads_per_block=threads)
  _check(ls, ctx, coords, tours, min(k, n - 1), S, iters)
  assert np.array_equal(tours, keep)  # inputs are not modified


def test_or_opt_lattice_ties_and_coordinates(torch_mod):
  """Lattice tours tie on many moves (the key order decides); a matrix cap makes the kernel
  rebuild every distance from FP64 coordinates, with the same result."""
  from tsp_gpu_clean_b200.strategies import LocalSearchB200OrOpt

  coords = np.array([[x * 10.0, y * 10.0] for x in range(7) for y in range(8)])
  rng = np.random.default_rng(5)
  tours = _tours(rng, len(coords), 6)
  for mmd in (None, 10):
    ctx = _ctx(coords)
    ls = LocalSearchB200OrOpt(max_iterations=1000, candidate_k=6, max_segment=3, max_matrix_dimension=mmd)
    _check(ls, ctx, coords, tours, 6, 3, 1000)


def test_or_opt_resident_tensors_and_large_tour(torch_mod):
  """CUDA tensors in and out; a 2000-city clustered tour for 25 passes equals the oracle."""
  from tsp_gpu_clean_b200.device import candidate_list
  from tsp_gpu_clean_b200.strategies import LocalSearchB200OrOpt

  coords = instances.clustered_instance(2000, 12, 40.0, 9)
  ctx = _ctx(coords)
  rng = np.random.default_rng(1)
  tours = _tours(rng, 2000, 3)
  ls = LocalSearchB200OrOpt(max_iterations=25, candidate_k=16)
  out = ls.improve_batch(torch_mod.from_numpy(tours.copy()).cuda(), ctx)
  assert out.is_cuda
  D = odist.euc2d_matrix(coords)
  cand = candidate_list(ctx, 16)
  for t in range(3):
    want, passes, moves, evaluated = oo.refine(tours[t], D, cand, 25, 3)
    assert np.array_equal(out[t].cpu().numpy(), want)
    assert ls.last_stats[t].tolist() == [passes, moves, evaluated]
  single = ls.improve(tours[0], ctx)
  assert single.shape == (2000,) and np.array_equal(single, out[0].cpu().numpy())


def test_or_opt_errors(torch_mod):
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.errors import NotPermutationError
  from tsp_gpu_clean_b200.strategies import LocalSearchB200OrOpt

  coords = instances.uniform_instance(30, 3)
  ctx = _ctx(coords)
  bad = np.arange(30, dtype=np.int32)[None, :].repeat(2, axis=0)
  bad[1, 5] = 7
  with pytest.raises(NotPermutationError):
    LocalSearchB200OrOpt().improve_batch(bad, ctx)
  for kw in ({"max_iterations": -1}, {"candidate_k": 0}, {"max_segment": 0}, {"max_segment": 9}):
    with pytest.raises(ValueError):
      LocalSearchB200OrOpt(**kw)
  lib = native.load_library()
  t = torch_mod.zeros((1, 30), dtype=torch_mod.int32, device="cuda")
  st = torch_mod.zeros(1, dtype=torch_mod.int32, device="cuda")
  c = torch_mod.zeros((30, 4), dtype=torch_mod.int32, device="cuda")
  d = torch_mod.zeros((30, 30), dtype=torch_mod.int32, device="cuda")
  p = lambda x: x.data_ptr()  # noqa: E731
  assert lib.tspb_or_opt(p(t), 1, 30, p(d), 30, None, p(c), p(c), None, 4, 3, 10, 200, p(st), None, None) == native.TSPB_ERR_ARG
  assert lib.tspb_or_opt(p(t), 1, 30, p(d), 30, None, p(c), p(c), None, 30, 3, 10, 256, p(st), None, None) == native.TSPB_ERR_ARG
  assert lib.tspb_or_opt(p(t), 1, 30, None, 0, None, p(c), p(c), None, 4, 3, 10, 256, p(st), None, None) == native.TSPB_ERR_ARG
  assert lib.tspb_or_opt(p(t), 1, 2, p(d), 30, None, p(c), p(c), None, 1, 3, 10, 256, p(st), None, None) == native.TSPB_OK
  assert lib.tspb_or_opt_max_n() > 10000


class _OracleOrOpt:
  """Test-only LocalSearchStrategy: the oracle's Or-opt on host arrays."""

  def __init__(self, coords, table, iters, S):
    self.D = odist.euc2d_matrix(coords)
    self.table, self.iters, self.S = table, iters, S

  def improve(self, route, context):
    return self.improve_batch(np.asarray(route)[None, :], context)[0]

  def improve_batch(self, routes, context):
    routes = np.asarray(routes, dtype=np.int32)
    return np.stack([oo.refine(r, self.D, self.table, self.iters, self.S)[0] for r in routes]).astype(np.int32)


def test_or_opt_drops_into_the_ga_pipeline(torch_mod):
  """The reference-shaped GA (post-init and elite local-search steps) with
  LocalSearchB200OrOpt equals the same pipeline whose local search is the oracle."""
  from tsp_gpu_clean_b200.device import candidate_list
  from tsp_gpu_clean_b200.ga import GeneticAlgorithm
  from tsp_gpu_clean_b200.pipeline_steps import EliteOnlyLocalSearchStep, PostInitLocalSearchStep
  from tsp_gpu_clean_b200.strategies import (
    CrossoverB200PermPartiallyMapped,
    EvaluationB200Cost,
    InitializationB200TourNearestNeighbor,
    LocalSearchB200OrOpt,
    MutationB200PermInversion,
    SelectionB200Tournament,
  )

  coords = instances.uniform_instance(90, 31)
  runs = []
  for which in ("b200", "oracle"):
    ctx = _ctx(coords)
    ls = (LocalSearchB200OrOpt(max_iterations=6, candidate_k=10) if which == "b200"
          else _OracleOrOpt(coords, candidate_list(ctx, 10), 6, 3))
    ev = EvaluationB200Cost()
    steps = [PostInitLocalSearchStep(local_search=ls, evaluation=ev),
             EliteOnlyLocalSearchStep(local_search=ls, evaluation=ev, elite_count=6)]
    ga = GeneticAlgorithm(population_size=32, mutation_rate=0.1, seed=42,
                          initialization=InitializationB200TourNearestNeighbor(k=5, seed=42),
                          selection=SelectionB200Tournament(k=5, seed=42),
                          crossover=CrossoverB200PermPartiallyMapped(seed=42),
                          mutation=MutationB200PermInversion(seed=42), local_search=ls, evaluation=ev,
                          pipeline=steps)
    best, stats = ga.evolve(context=ctx, customers=list(range(90)), max_generations=12, patience=10**9)
    runs.append((np.asarray(best), list(stats["convergence_history"])))
  assert np.array_equal(runs[0][0], runs[1][0])
  assert runs[0][1] == runs[1][1]


def test_or_opt_packed_and_plain_tables_agree(torch_mod):
  """k % 4 == 0: the packed words (four per 16-byte load) and the plain id / distance
  tables give the same tours and counts, both equal to the oracle."""
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import candidate_list, operands_for, ptr, stream_handle

  coords = instances.clustered_instance(300, 6, 25.0, 4)
  ctx = _ctx(coords)
  ops = operands_for(ctx)
  dist, stride, _ = ops.distance_args(300)
  tabs = ops.candidates(12, candidate_list(ctx, 12), 300)
  assert tabs.packed is not None and tabs.k == 12
  tours = _tours(np.random.default_rng(8), 300, 6)
  lib = native.load_library()
  outs = []
  for packed in (tabs.packed, None):
    t = torch_mod.from_numpy(tours.copy()).cuda()
    st = torch_mod.zeros(6, dtype=torch_mod.int32, device="cuda")
    stats = torch_mod.zeros((6, 3), dtype=torch_mod.int64, device="cuda")
    native.check("tspb_or_opt", lib.tspb_or_opt(ptr(t), 6, 300, ptr(dist), stride, None, ptr(tabs.cand),
                                                ptr(tabs.cand_dist), ptr(packed), 12, 3, 1000, 128, ptr(st), ptr(stats),
                                                stream_handle()))
    assert int(st.max().item()) == 0
    outs.append((t.cpu().numpy(), stats.cpu().numpy()))
  assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
  D = odist.euc2d_matrix(coords)
  cand = candidate_list(ctx, 12)
  for r in range(6):
    want, passes, moves, evaluated = oo.refine(tours[r], D, cand, 1000, 3)
    assert np.array_equal(outs[0][0][r], want) and outs[0][1][r].tolist() == [passes, moves, evaluated]
