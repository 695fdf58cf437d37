"""NumPy restatement of the reference `GeneticAlgorithm.evolve` loop for TSP.

Follows `src/algorithms/metaheuristics/genetic_algorithm.py`:
- pipeline composition `_steps_*` / `STAGE_SPECS` / `_compose_pipeline` (:313-368, :459-487);
- `evolve` (:789-965): initial raw evaluation, per-generation steps, best tracking with
  the strict `cand < best - 1e-6` rule (:768-783, :876-892), patience early stop
  (:815-816, :906-910), and the `post_evolution` hook (:912-943);
and the extension steps of `src/algorithms/pipeline_steps.py`:
`PostInitLocalSearchStep.run` (:103-125), `EliteOnlyLocalSearchStep.run` (:153-195),
`PeriodicLocalSearchStep.run` (:252-285).

Strategies are the oracle operators in `oracle.ga_ops` and `oracle.two_opt`; every
random draw comes from the one context generator, in the reference's order.
Test infrastructure only (see the package docstring).
"""

from __future__ import annotations

import hashlib
import math
from dataclasses import dataclass, field

import numpy as np

from . import ga_ops, two_opt


@dataclass
class LocalSearchSpec:
  mode: str = "best"
  max_iterations: int = 10
  candidate_k: int | None = 20


@dataclass
class GAConfig:
  population_size: int = 128
  mutation_rate: float = 0.05
  nn_k: int = 5
  tournament_k: int = 5
  local_search: LocalSearchSpec | None = field(default_factory=LocalSearchSpec)
  local_search_stage: str = "none"
  post_init: bool = True
  elite_count: int | None = 16
  periodic: tuple[int, str] | None = None  # (interval, target)
  crossover: str = "pmx"  # "pmx" (CrossoverCPUPermPartiallyMapped) or "ox" (CrossoverCPUPermOrder)
  mutation: str = "inversion"  # "inversion" (MutationCPUPermInversion) or "swap" (MutationCPUPermSwap)
  init: str = "nn"  # "nn" (InitializationCPUTourNearestNeighbor) or "random" (InitializationCPUPermRandom)


def routes_digest(routes: np.ndarray) -> str:
  return hashlib.sha256(np.ascontiguousarray(routes, dtype=np.int32).tobytes()).hexdigest()


class OracleGA:
  """One GA run on a dense int32 matrix `D` and a candidate-table provider."""

  def __init__(self, D: np.ndarray, cand_provider, cfg: GAConfig, rng: np.random.Generator):
    self.D = D
    self.cand_provider = cand_provider  # k -> (n, k_eff) int32 table
    self.cfg = cfg
    self.rng = rng
    self.n = D.shape[0]

  # --- strategies -----------------------------------------------------------------
  def _improve(self, routes):
    ls = self.cfg.local_search
    cand = None
    if ls.candidate_k is not None and ls.candidate_k > 0:
      cand = two_opt.resolve_candidates(self.cand_provider(ls.candidate_k), np.asarray(routes), self.n)
    out, _ = two_opt.improve_batch(routes, self.D, cand, ls.mode, ls.max_iterations)
    return out

  def _cost(self, routes):
    return ga_ops.tour_cost(routes, self.D)

  # --- pipeline -------------------------------------------------------------------
  def _steps(self):
    cfg = self.cfg
    ls = cfg.local_search
    stage = cfg.local_search_stage
    core = ["select", "crossover", "mutate", "eval_offspring", "survive"]
    if ls is not None:
      if stage == "post_crossover":
        core = ["select", "crossover", "ls_offspring", "mutate", "eval_offspring", "survive"]
      elif stage == "post_mutation":
        core = ["select", "crossover", "mutate", "ls_offspring", "eval_offspring", "survive"]
      elif stage == "post_evaluation":
        core = ["select", "crossover", "mutate", "eval_offspring", "survive", "ls_population"]
    pre = ["post_init"] if cfg.post_init else []
    post = []
    if cfg.periodic is not None:
      interval, target = cfg.periodic
      if target == "offspring":
        core.insert(core.index("eval_offspring"), "periodic_offspring")
      else:
        post.append("periodic_population")
    if cfg.elite_count:
      post.append("elite")
    return pre + core + post

  def evolve(self, max_generations: int, patience: int | None = None, record: bool = False):
    cfg = self.cfg
    rng = self.rng
    n = self.n
    if patience is None:
      patience = int(2 * math.sqrt(n))
    customers = np.arange(n, dtype=np.int32)
    if cfg.init == "random":
      pop = ga_ops.random_init(rng, customers, cfg.population_size)
    else:
      pop = ga_ops.nn_init(rng, customers, cfg.population_size, self.cand_provider(cfg.nn_k))
    fit = self._cost(pop)
    best_idx = int(np.argmin(fit))
    best_cost = float(fit[best_idx])
    best_tour = pop[best_idx].copy()
    history = [best_cost]
    records = []
    stall = 0
    gen_done = 0
    stop_reason = "max_generations"
    steps = self._steps()
    for gen in range(1, max_generations + 1):
      gen_done = gen
      off = off_fit = None
      for s in steps:
        if s == "post_init":
          if gen == 1 and cfg.local_search is not None:
            pop = self._improve(pop)
            fit = self._cost(pop)
        elif s == "select":
          off = ga_ops.tournament_select(rng, pop, fit, cfg.population_size, cfg.tournament_k)
        elif s == "crossover":
          off = ga_ops.ox_batch(rng, off) if cfg.crossover == "ox" else ga_ops.pmx_batch(rng, off)
        elif s == "mutate":
          off = (ga_ops.swap_batch(rng, off, cfg.mutation_rate) if cfg.mutation == "swap"
                 else ga_ops.inversion_batch(rng, off, cfg.mutation_rate))
        elif s == "ls_offspring":
          off = self._improve(off)
        elif s == "eval_offspring":
          off_fit = self._cost(off)
        elif s == "survive":
          pop, fit, _ = ga_ops.survivors(pop, fit, off, off_fit, cfg.population_size)
        elif s == "ls_population":
          pop = self._improve(pop)
          fit = self._cost(pop)
        elif s == "periodic_offspring":
          if gen % cfg.periodic[0] == 0:
            off = self._improve(off)
        elif s == "periodic_population":
          if gen % cfg.periodic[0] == 0:
            pop = self._improve(pop)
            fit = self._cost(pop)
        elif s == "elite":
          k = min(cfg.elite_count, len(pop))
          idx = ga_ops.elite_indices(fit, k)
          improved = self._improve(pop[idx])
          pop[idx] = improved
          fit[idx] = self._cost(improved)
      ci = int(np.argmin(fit))
      cc = float(fit[ci])
      if cc < best_cost - 1e-6:
        best_tour = pop[ci].copy()
        best_cost = cc
        stall = 0
      else:
        stall += 1
      history.append(best_cost)
      if record:
        records.append((routes_digest(pop), fit.copy()))
      if stall >= patience:
        stop_reason = "no_improvements"
        break
    if cfg.local_search is not None and cfg.local_search_stage == "post_evolution":
      pop = self._improve(pop)
      fit = self._cost(pop)
      pi = int(np.argmin(fit))
      if float(fit[pi]) <= best_cost:
        best_tour = pop[pi].copy()
        best_cost = float(fit[pi])
        history[-1] = best_cost
    stats = {
      "best_fitness": best_cost,
      "generations_completed": gen_done,
      "stop_reason": stop_reason,
      "convergence_history": history,
    }
    return best_tour, pop, fit, stats, records
