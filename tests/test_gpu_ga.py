"""Full GA runs on the B200 strategies against the reference's recorded runs.

Every generation's population digest and fitness vector, the best tour, the convergence
history and the final RNG state must equal what the reference's CPU GA produced
(`tests/golden/ga.npz`), in drop-in mode (host arrays) and device-resident mode.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class Recorder:
  stage_anchor = "post_survival"

  def __init__(self):
    self.digests = []
    self.fitness = []

  def run(self, state, timer):
    pop = state.population
    fit = state.fitness
    pop = pop.cpu().numpy() if hasattr(pop, "is_cuda") else np.asarray(pop)
    fit = fit.cpu().numpy() if hasattr(fit, "is_cuda") else np.asarray(fit)
    self.digests.append(hashlib.sha256(np.ascontiguousarray(pop, dtype=np.int32).tobytes()).hexdigest())
    self.fitness.append(np.asarray(fit, dtype=np.float64).copy())


def run_b200_ga(g, tag, resident: bool):
  from tsp_gpu_clean_b200.ga import GeneticAlgorithm
  from tsp_gpu_clean_b200.pipeline_steps import EliteOnlyLocalSearchStep, PeriodicLocalSearchStep, PostInitLocalSearchStep
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext
  from tsp_gpu_clean_b200.strategies import (
    CrossoverB200PermPartiallyMapped,
    EvaluationB200Cost,
    InitializationB200TourNearestNeighbor,
    LocalSearchB200TourTwoOpt,
    MutationB200PermInversion,
    SelectionB200Tournament,
  )

  coords = g[f"{tag}_coords"]
  pop_size, gens, elite, post_init, ls_iters, seed, per_int, per_tgt = (int(v) for v in g[f"{tag}_meta"])
  stage = str(g[f"{tag}_stage"])
  ctx = ProblemContext(Problem.from_coordinates(coords), seed=seed)
  ls = LocalSearchB200TourTwoOpt(mode="best", max_iterations=ls_iters, candidate_k=20)
  ev = EvaluationB200Cost(return_gpu=resident)
  rec = Recorder()
  steps = []
  if post_init:
    steps.append(PostInitLocalSearchStep(local_search=ls, evaluation=ev))
  if per_int > 0:
    target = "offspring" if per_tgt == 0 else "population"
    steps.append(PeriodicLocalSearchStep(local_search=ls, interval=per_int, target=target,
                                         re_evaluate=ev if target == "population" else None))
  if elite:
    steps.append(EliteOnlyLocalSearchStep(local_search=ls, evaluation=ev, elite_count=elite))
  steps.append(rec)
  ga = GeneticAlgorithm(population_size=pop_size, mutation_rate=float(g[f"{tag}_rate"]), seed=42,
                        initialization=InitializationB200TourNearestNeighbor(k=5, seed=42, return_gpu=resident),
                        selection=SelectionB200Tournament(k=5, seed=42), crossover=CrossoverB200PermPartiallyMapped(seed=42),
                        mutation=MutationB200PermInversion(seed=42), local_search=ls, evaluation=ev,
                        local_search_stage=stage, pipeline=steps)
  patience = None if tag == "c1default" else 10**9
  best, stats = ga.evolve(context=ctx, customers=list(range(len(coords))), max_generations=gens, patience=patience)
  return best, stats, rec, ctx


@pytest.mark.parametrize("resident", [False, True])
@pytest.mark.parametrize("tag", ["c1", "c1default", "pm", "pc", "pe", "px", "pp", "po", "c3"])
def test_ga_matches_reference(golden, tag, resident):
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  g = golden("ga.npz")
  best, stats, rec, ctx = run_b200_ga(g, tag, resident)
  assert rec.digests == [str(d) for d in g[f"{tag}_digests"]]
  assert np.array_equal(np.stack(rec.fitness), g[f"{tag}_fitness"])
  assert np.array_equal(best, g[f"{tag}_best"])
  assert np.array_equal(np.asarray(stats["convergence_history"]), g[f"{tag}_history"])
  assert stats["generations_completed"] == int(g[f"{tag}_gens"])
  assert ctx.rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"{tag}_rng"][0])
