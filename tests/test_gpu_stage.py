"""Random-permutation init and 2-opt on every offspring (`local_search_stage="post_mutation"`)
on the B200, against the reference's recorded runs (`tests/golden/stage.npz`) and the oracle.

Two of the recorded runs use the configuration of the reference's published Chapter-4
benchmarks (random init, tournament 5, OX, swap, 2-opt k=20 x10 on every child); the third
mixes the stage with NN init, PMX, inversion and the post-init and elite steps.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import distances as odist
from oracle import ga as oga
from oracle import ga_ops

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  return torch


def _ctx(coords, seed):
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  return ProblemContext(Problem.from_coordinates(np.asarray(coords, dtype=np.float64)), seed=seed)


@pytest.mark.parametrize("tag", ["r1", "r2", "r3", "r4", "r5"])
@pytest.mark.parametrize("resident", [False, True])
def test_random_init_matches_reference(torch_mod, golden, tag, resident):
  from tsp_gpu_clean_b200.strategies import InitializationB200PermRandom

  g = golden("stage.npz")
  n, pop_size, seed = (int(v) for v in g[f"{tag}_meta"])
  ctx = _ctx(np.random.default_rng(0).uniform(0, 1000, (max(n, 2), 2)), seed)
  out = InitializationB200PermRandom(seed=1, return_gpu=resident).initialize(list(g[f"{tag}_customers"]), pop_size, ctx)
  pop = np.ascontiguousarray(out.cpu().numpy() if resident else out, dtype=np.int32)
  if f"{tag}_pop" in g:
    assert np.array_equal(pop, g[f"{tag}_pop"])
  else:
    assert hashlib.sha256(pop.tobytes()).digest() == g[f"{tag}_digest"].tobytes()
  assert ctx.rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"{tag}_rng_state"][0])


def test_random_init_long_rows_vs_oracle(torch_mod):
  """Rows longer than the shared-memory stage are shuffled in place in global memory."""
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  torch = torch_mod
  for n, rows in ((24 * 1024, 2), (24 * 1024 + 1, 2), (40000, 3)):
    rng = np.random.default_rng(n)
    want = ga_ops.random_init(np.random.default_rng(n), np.arange(n), rows)
    seeds = ga_ops.draw_row_seeds(rng, rows)
    d_seeds = torch.from_numpy(seeds.view(np.int64).copy()).cuda()
    out = torch.empty((rows, n), dtype=torch.int32, device="cuda")
    native.call("tspb_random_init", ptr(d_seeds), rows, n, None, ptr(out), stream_handle())
    assert np.array_equal(out.cpu().numpy(), want), n


def _stage(g, tag):
  pop_size, gens, elite, post_init, patience, chapter4 = (int(v) for v in g[f"ga_{tag}_meta"])
  return dict(pop_size=pop_size, gens=gens, elite=elite, post_init=bool(post_init),
              patience=None if patience < 0 else patience, chapter4=bool(chapter4),
              rate=float(g[f"ga_{tag}_rate"]))


def _check(g, tag, best, stats, ctx):
  assert stats["generations_completed"] == int(g[f"ga_{tag}_gens"])
  assert np.array_equal(np.asarray(stats["convergence_history"]), g[f"ga_{tag}_history"])
  assert np.array_equal(np.asarray(best), g[f"ga_{tag}_best"])
  assert ctx.rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"ga_{tag}_rng"][0])


@pytest.mark.parametrize("resident", [False, True])
@pytest.mark.parametrize("tag", ["s1", "s2", "s3"])
def test_strategy_ga_with_post_mutation_stage_matches_reference(torch_mod, golden, tag, resident):
  from tsp_gpu_clean_b200.ga import GeneticAlgorithm
  from tsp_gpu_clean_b200.pipeline_steps import EliteOnlyLocalSearchStep, PostInitLocalSearchStep
  from tsp_gpu_clean_b200.strategies import (
    CrossoverB200PermOrder,
    CrossoverB200PermPartiallyMapped,
    EvaluationB200Cost,
    InitializationB200PermRandom,
    InitializationB200TourNearestNeighbor,
    LocalSearchB200TourTwoOpt,
    MutationB200PermInversion,
    MutationB200PermSwap,
    SelectionB200Tournament,
  )

  g = golden("stage.npz")
  s = _stage(g, tag)
  coords = g[f"ga_{tag}_coords"]
  ctx = _ctx(coords, 42)
  ls = LocalSearchB200TourTwoOpt(mode="best", max_iterations=10, candidate_k=20)
  ev = EvaluationB200Cost(return_gpu=resident)
  steps = []
  if s["post_init"]:
    steps.append(PostInitLocalSearchStep(local_search=ls, evaluation=ev))
  if s["elite"]:
    steps.append(EliteOnlyLocalSearchStep(local_search=ls, evaluation=ev, elite_count=s["elite"]))
  if s["chapter4"]:
    init = InitializationB200PermRandom(seed=42, return_gpu=resident)
    xo, mut = CrossoverB200PermOrder(seed=42), MutationB200PermSwap(seed=42)
  else:
    init = InitializationB200TourNearestNeighbor(k=5, seed=42, return_gpu=resident)
    xo, mut = CrossoverB200PermPartiallyMapped(seed=42), MutationB200PermInversion(seed=42)
  ga = GeneticAlgorithm(population_size=s["pop_size"], mutation_rate=s["rate"], seed=42, initialization=init,
                        selection=SelectionB200Tournament(k=5, seed=42), crossover=xo, mutation=mut, local_search=ls,
                        evaluation=ev, local_search_stage="post_mutation", pipeline=steps or None)
  best, stats = ga.evolve(context=ctx, customers=list(range(len(coords))), max_generations=s["gens"],
                          patience=s["patience"])
  _check(g, tag, best, stats, ctx)


def _fused_kwargs(s):
  return dict(population_size=s["pop_size"], mutation_rate=s["rate"], tournament_k=5, nn_k=5,
              elite_count=s["elite"], post_init=s["post_init"], local_search_stage="post_mutation",
              crossover="ox" if s["chapter4"] else "pmx", mutation="swap" if s["chapter4"] else "inversion",
              init="random" if s["chapter4"] else "nn")


@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("tag", ["s1", "s2", "s3"])
def test_fused_ga_with_post_mutation_stage_matches_reference(torch_mod, golden, tag, use_graph):
  from tsp_gpu_clean_b200.fused import FusedMemeticSolver, LocalSearchConfig

  g = golden("stage.npz")
  s = _stage(g, tag)
  coords = g[f"ga_{tag}_coords"]
  ctx = _ctx(coords, 42)
  solver = FusedMemeticSolver(local_search=LocalSearchConfig("best", 10, 20), use_graph=use_graph, chunk=6,
                              **_fused_kwargs(s))
  best, stats = solver.evolve(ctx, list(range(len(coords))), s["gens"], patience=s["patience"])
  _check(g, tag, best, stats, ctx)


@pytest.mark.parametrize("skip_converged,incremental", [(True, "on"), (False, "on"), (True, "off")])
def test_batch_chapter4_runs_of_mixed_sizes_match_oracle(torch_mod, skip_converged, incremental):
  """Instances of sizes across several buckets, Chapter-4 configuration, each run equal to
  the oracle GA (random init, OX, swap, 2-opt on every child) with its own seed. With the
  reverse k-NN index (incremental "on") best mode recomputes only the rows a move can
  change; the same runs either way."""
  from tsp_gpu_clean_b200 import instances
  from tsp_gpu_clean_b200.batch import FusedBatchSolver
  from tsp_gpu_clean_b200.fused import LocalSearchConfig

  sizes = [12, 57, 130, 300, 520]
  coords = [instances.uniform_instance(n, 600 + n) for n in sizes]
  ctxs = [_ctx(c, 70 + j) for j, c in enumerate(coords)]
  P, G, rate = 24, 12, 0.2
  solver = FusedBatchSolver(population_size=P, mutation_rate=rate, tournament_k=5, nn_k=5,
                            local_search=LocalSearchConfig("best", 10, 8), elite_count=0, post_init=False,
                            chunk=5, skip_converged=skip_converged, crossover="ox", mutation="swap", init="random",
                            local_search_stage="post_mutation", incremental=incremental)
  results = solver.evolve(ctxs, G, patience=10**9)
  assert all(b.incremental == (incremental == "on") for b in solver.buckets)
  tot = solver.two_opt_totals
  # gains computed: below the pairs scanned either way (an entry whose lower bound cannot
  # improve is settled without its gather); with the reverse index also fewer rows rescanned
  assert 0 < tot["evaluated"] < tot["pairs"]
  for j, ((best, stats), c) in enumerate(zip(results, coords)):
    cache = {}

    def provider(k, c=c):
      if k not in cache:
        cache[k] = odist.candidate_list(k, coords=c)
      return cache[k]

    cfg = oga.GAConfig(population_size=P, mutation_rate=rate, nn_k=5, tournament_k=5,
                       local_search=oga.LocalSearchSpec("best", 10, 8), local_search_stage="post_mutation",
                       post_init=False, elite_count=None, crossover="ox", mutation="swap", init="random")
    rng = np.random.default_rng(70 + j)
    obest, opop, ofit, ostats, _ = oga.OracleGA(odist.euc2d_matrix(c), provider, cfg, rng).evolve(G, patience=10**9)
    assert np.array_equal(np.asarray(stats["convergence_history"]), np.asarray(ostats["convergence_history"])), j
    assert np.array_equal(best, obest), j
    assert np.array_equal(solver.final_population[j].cpu().numpy(), opop), j
    assert np.array_equal(solver.final_fitness[j].cpu().numpy(), ofit), j
    assert ctxs[j].rng.bit_generator.state["state"]["state"] == rng.bit_generator.state["state"]["state"], j


def test_invalid_stage_options():
  from tsp_gpu_clean_b200.batch import FusedBatchSolver
  from tsp_gpu_clean_b200.fused import FusedMemeticSolver

  with pytest.raises(ValueError):
    FusedBatchSolver(local_search_stage="post_crossover")
  with pytest.raises(ValueError):
    FusedBatchSolver(init="greedy")
  with pytest.raises(ValueError):
    FusedBatchSolver(incremental="yes")
  with pytest.raises(ValueError):
    FusedMemeticSolver(engine="single", local_search_stage="post_mutation")
  with pytest.raises(ValueError):
    FusedMemeticSolver(engine="single", init="random")
