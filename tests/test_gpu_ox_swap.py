"""Order Crossover and swap mutation on the B200 against the reference's golden outputs.

`tests/golden/ox_swap.npz` holds what the reference's CPU strategies produced
(`CrossoverCPUPermOrder`, `MutationCPUPermSwap`) on fixed populations, and two full GA runs
with those operators; the oracle (`oracle/ga_ops.py`) covers random cases.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import ga_ops
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


def _ctx(n, seed):
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  coords = np.random.default_rng(0).uniform(0.0, 1000.0, (n, 2))
  return ProblemContext(Problem.from_coordinates(coords), seed=seed)


@pytest.mark.parametrize("tag", ["a", "b", "c", "d", "e", "f"])
@pytest.mark.parametrize("resident", [False, True])
def test_ox_and_swap_match_reference(torch_mod, golden, tag, resident):
  from tsp_gpu_clean_b200.strategies import CrossoverB200PermOrder, MutationB200PermSwap

  g = golden("ox_swap.npz")
  n, _, seed = (int(v) for v in g[f"{tag}_meta"])
  ctx = _ctx(n, seed)
  pop = g[f"{tag}_pop"]
  x = torch_mod.from_numpy(pop).cuda() if resident else pop.copy()
  ox = CrossoverB200PermOrder(seed=1).crossover_batch(x, ctx)
  sw = MutationB200PermSwap(seed=1).mutate_batch(ox if resident else np.asarray(ox).copy(), float(g[f"{tag}_rate"]),
                                                 ctx)
  host = (lambda t: t.cpu().numpy()) if resident else np.asarray
  assert np.array_equal(host(ox), g[f"{tag}_ox"])
  assert np.array_equal(host(sw), g[f"{tag}_swap"])
  assert ctx.rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"{tag}_rng_state"][0])


def test_ox_and_swap_random_vs_oracle(torch_mod):
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  torch = torch_mod
  rng = np.random.default_rng(11)
  for n in (2, 3, 5, 31, 32, 33, 64, 1000, 4099, 20000):
    for rows in (1, 2, 33):
      pop = instances.random_tours(n, rows, n + rows)
      pairs = ga_ops.sample_distinct_pairs(rng, max(rows // 2, 1), 0, n)
      want = ga_ops.ox_apply(pop, pairs[: rows // 2])
      d = torch.from_numpy(pop).cuda()
      out = torch.empty_like(d)
      st = torch.full((rows,), -7, dtype=torch.int32, device="cuda")
      f = torch.from_numpy(pairs[:, 0].copy()).cuda()
      s = torch.from_numpy(pairs[:, 1].copy()).cuda()
      native.call("tspb_ox", ptr(d), rows, n, ptr(f), ptr(s), ptr(out), ptr(st), stream_handle())
      assert np.array_equal(out.cpu().numpy(), want), (n, rows)
      assert st.cpu().numpy().tolist() == [0] * rows
      u = rng.random(rows)
      u[: rows // 2] = 0.0
      p1 = rng.integers(0, n, rows).astype(np.int32)
      p2 = rng.integers(0, n, rows).astype(np.int32)
      want = ga_ops.swap_apply(pop, 0.5, u, p1, p2)
      d = torch.from_numpy(pop).cuda()
      du, d1, d2 = torch.from_numpy(u).cuda(), torch.from_numpy(p1).cuda(), torch.from_numpy(p2).cuda()
      native.call("tspb_swap", ptr(d), rows, n, ptr(du), 0.5, ptr(d1), ptr(d2), stream_handle())
      assert np.array_equal(d.cpu().numpy(), want), (n, rows)


def test_ox_rejects_non_permutations(torch_mod):
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle
  from tsp_gpu_clean_b200.errors import NotPermutationError
  from tsp_gpu_clean_b200.strategies import CrossoverB200PermOrder

  torch = torch_mod
  pop = instances.random_tours(40, 6, 2)
  pop[1, 3] = pop[1, 4]  # duplicate in the second parent of pair 0
  pop[4, 0] = 40  # out of range in the first parent of pair 2
  d = torch.from_numpy(pop).cuda()
  out = torch.empty_like(d)
  st = torch.zeros(6, dtype=torch.int32, device="cuda")
  cuts = torch.tensor([3, 5, 0], dtype=torch.int32, device="cuda")
  native.call("tspb_ox", ptr(d), 6, 40, ptr(cuts), ptr(cuts), ptr(out), ptr(st), stream_handle())
  status = st.cpu().numpy()
  assert status[0] != 0 and status[1] != 0 and status[4] != 0 and status[5] != 0
  assert status[2] == 0 and status[3] == 0
  with pytest.raises(NotPermutationError):
    CrossoverB200PermOrder(seed=0).crossover_batch(pop, _ctx(40, 0))


def _ga_expect(g, tag):
  pop_size, gens, elite, post_init, patience = (int(v) for v in g[f"ga_{tag}_meta"])
  return pop_size, gens, elite, bool(post_init), (None if patience < 0 else patience)


def _check(g, tag, best, stats, ctx):
  assert stats["generations_completed"] == int(g[f"ga_{tag}_gens"])
  assert np.array_equal(np.asarray(stats["convergence_history"]), g[f"ga_{tag}_history"])
  assert np.array_equal(np.asarray(best), g[f"ga_{tag}_best"])
  assert ctx.rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"ga_{tag}_rng"][0])


@pytest.mark.parametrize("resident", [False, True])
@pytest.mark.parametrize("tag", ["ox1", "ox2"])
def test_strategy_ga_with_ox_and_swap_matches_reference(torch_mod, golden, tag, resident):
  from tsp_gpu_clean_b200.ga import GeneticAlgorithm
  from tsp_gpu_clean_b200.pipeline_steps import EliteOnlyLocalSearchStep, PostInitLocalSearchStep
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext
  from tsp_gpu_clean_b200.strategies import (
    CrossoverB200PermOrder,
    EvaluationB200Cost,
    InitializationB200TourNearestNeighbor,
    LocalSearchB200TourTwoOpt,
    MutationB200PermSwap,
    SelectionB200Tournament,
  )

  g = golden("ox_swap.npz")
  coords = g[f"ga_{tag}_coords"]
  pop_size, gens, elite, post_init, patience = _ga_expect(g, tag)
  ctx = ProblemContext(Problem.from_coordinates(coords), seed=7)
  ls = LocalSearchB200TourTwoOpt(mode="best", max_iterations=10, candidate_k=20)
  ev = EvaluationB200Cost(return_gpu=resident)
  steps = [PostInitLocalSearchStep(local_search=ls, evaluation=ev)] if post_init else []
  steps.append(EliteOnlyLocalSearchStep(local_search=ls, evaluation=ev, elite_count=elite))
  ga = GeneticAlgorithm(population_size=pop_size, mutation_rate=float(g[f"ga_{tag}_rate"]), seed=7,
                        initialization=InitializationB200TourNearestNeighbor(k=5, seed=7, return_gpu=resident),
                        selection=SelectionB200Tournament(k=5, seed=7), crossover=CrossoverB200PermOrder(seed=7),
                        mutation=MutationB200PermSwap(seed=7), local_search=ls, evaluation=ev,
                        local_search_stage="none", pipeline=steps)
  best, stats = ga.evolve(context=ctx, customers=list(range(len(coords))), max_generations=gens, patience=patience)
  _check(g, tag, best, stats, ctx)


@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("tag", ["ox1", "ox2"])
def test_fused_ga_with_ox_and_swap_matches_reference(torch_mod, golden, tag, use_graph):
  from tsp_gpu_clean_b200.fused import FusedMemeticSolver, LocalSearchConfig
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  g = golden("ox_swap.npz")
  coords = g[f"ga_{tag}_coords"]
  pop_size, gens, elite, post_init, patience = _ga_expect(g, tag)
  ctx = ProblemContext(Problem.from_coordinates(coords), seed=7)
  solver = FusedMemeticSolver(population_size=pop_size, mutation_rate=float(g[f"ga_{tag}_rate"]), tournament_k=5,
                              nn_k=5, local_search=LocalSearchConfig("best", 10, 20), elite_count=elite,
                              post_init=post_init, use_graph=use_graph, chunk=5, crossover="ox", mutation="swap")
  best, stats = solver.evolve(ctx, list(range(len(coords))), gens, patience=patience)
  _check(g, tag, best, stats, ctx)


def test_batch_runs_ox_and_swap(torch_mod, golden):
  """Three copies of a reference run in one batch: each equals the reference's run."""
  from tsp_gpu_clean_b200.batch import FusedBatchSolver
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  g = golden("ox_swap.npz")
  tag = "ox2"
  coords = g[f"ga_{tag}_coords"]
  pop_size, gens, elite, post_init, patience = _ga_expect(g, tag)
  ctxs = [ProblemContext(Problem.from_coordinates(coords), seed=7) for _ in range(3)]
  solver = FusedBatchSolver(population_size=pop_size, mutation_rate=float(g[f"ga_{tag}_rate"]), tournament_k=5,
                            nn_k=5, local_search=LocalSearchConfig("best", 10, 20), elite_count=elite,
                            post_init=post_init, chunk=4, crossover="ox", mutation="swap")
  results = solver.evolve(ctxs, gens, patience=patience)
  for (best, stats), ctx in zip(results, ctxs):
    _check(g, tag, best, stats, ctx)


def test_single_engine_refuses_ox():
  from tsp_gpu_clean_b200.fused import FusedMemeticSolver

  with pytest.raises(ValueError):
    FusedMemeticSolver(engine="single", crossover="ox")
  with pytest.raises(ValueError):
    FusedMemeticSolver(mutation="scramble")
