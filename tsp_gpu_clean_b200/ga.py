"""The memetic GA loop and its generation pipeline, mirroring the reference's orchestration.

Follows `src/algorithms/metaheuristics/genetic_algorithm.py` of the reference:
`GenerationState` (:69-80), `GenerationStep` (:112-117), the core steps (:120-296),
`STAGE_SPECS` (:362-368), `_compose_pipeline` (:459-482), survival (:598-706), best
tracking (:709-783) and `evolve` (:789-965), with the same argument meanings, defaults
(`patience = int(2 * sqrt(n))`), early stops and stats keys.

The loop is agnostic to where the population lives: host NumPy arrays (every strategy
in drop-in mode) or CUDA tensors (B200 strategies with `return_gpu=True`). For CUDA
tensors the loop's own work runs on the device too: survival is `tspb_stable_rank` plus
`tspb_gather_rows`, and best tracking reads back one index and one cost per generation.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, Callable, Literal, Mapping, Protocol

import numpy as np

from . import native
from .device import device_tensor, is_device_array, ptr, stream_handle, torch
from .phase_timer import PhaseTimer
from .strategies.base import RouteAssessment


# ------------------------------------------------------------------------------ helpers
def assess_with_evaluator(evaluator: Any, routes: Any, context: Any, *, return_gpu: bool = False) -> RouteAssessment:
  """`assess_with_evaluator` (`src/protocols/vrp_strategies.py:199-216`)."""
  from .routes import ensure_routes_batch
  from .strategies.base import tour_assessment

  batch, _ = ensure_routes_batch(routes)
  hook = getattr(evaluator, "assess_batch", None)
  if callable(hook):
    try:
      res = hook(batch, context, return_gpu=return_gpu)
    except TypeError:
      res = hook(batch, context)
    if hasattr(res, "objectives"):
      return res
  try:
    obj = evaluator.evaluate_batch(batch, context, return_gpu=return_gpu)
  except TypeError:
    obj = evaluator.evaluate_batch(batch, context)
  return tour_assessment(obj)


def canonicalize_with_evaluator(evaluator: Any, route: Any, context: Any) -> np.ndarray:
  hook = getattr(evaluator, "canonicalize_route", None)
  if callable(hook):
    return np.asarray(hook(route, context), dtype=np.int32)
  if is_device_array(route):
    return route.cpu().numpy().astype(np.int32, copy=True)
  return np.asarray(route, dtype=np.int32).copy()


def _as_f64(x: Any, like_device: bool) -> Any:
  if like_device:
    return x.to(torch.float64) if is_device_array(x) else device_tensor(np.asarray(x, dtype=np.float64), torch.float64)
  return x.cpu().numpy().astype(np.float64) if is_device_array(x) else np.asarray(x, dtype=np.float64)


def _device_take_rows(src: "torch.Tensor", rows: "torch.Tensor") -> "torch.Tensor":
  src = src.contiguous()
  out = torch.empty((int(rows.shape[0]), int(src.shape[1])), dtype=torch.int32, device=src.device)
  native.call("tspb_gather_rows", ptr(src), int(src.shape[0]), int(src.shape[1]), ptr(rows), int(rows.shape[0]), ptr(out),
              stream_handle())
  return out


def stable_order(values: Any, keep: int) -> Any:
  """Indices of the `keep` smallest values by (value, index): NumPy lexsort or the device rank."""
  if is_device_array(values):
    v = values.to(torch.float64).contiguous()
    order = torch.empty(keep, dtype=torch.int32, device=v.device)
    native.call("tspb_stable_rank", ptr(v), int(v.shape[0]), keep, ptr(order), stream_handle())
    return order
  v = np.asarray(values, dtype=np.float64)
  zeros = np.zeros_like(v)
  return np.lexsort(np.vstack([v, zeros, zeros]))[:keep]


# ------------------------------------------------------------------------------ steps
@dataclass
class GenerationState:
  population: Any
  fitness: Any
  context: Any
  offspring: Any = None
  offspring_fitness: Any = None
  generation: int = 0
  population_assessment: RouteAssessment | None = None
  offspring_assessment: RouteAssessment | None = None


class GenerationStep(Protocol):
  def run(self, state: GenerationState, timer: PhaseTimer) -> None: ...


class SelectionStep:
  def __init__(self, strategy: Any, population_size: int) -> None:
    self.strategy = strategy
    self.population_size = population_size

  def run(self, state: GenerationState, timer: PhaseTimer) -> None:
    state.offspring = timer.measure("selection", self.strategy.select_batch, state.population, state.fitness,
                                    self.population_size, state.context)


class CrossoverStep:
  def __init__(self, strategy: Any) -> None:
    self.strategy = strategy

  def run(self, state: GenerationState, timer: PhaseTimer) -> None:
    if state.offspring is None:
      raise RuntimeError("CrossoverStep called before state.offspring was populated.")
    state.offspring = timer.measure("crossover", self.strategy.crossover_batch, state.offspring, state.context)


class MutationStep:
  def __init__(self, strategy: Any, mutation_rate: float) -> None:
    self.strategy = strategy
    self.mutation_rate = mutation_rate

  def run(self, state: GenerationState, timer: PhaseTimer) -> None:
    if state.offspring is None:
      raise RuntimeError("MutationStep called before state.offspring was populated.")
    state.offspring = timer.measure("mutation", self.strategy.mutate_batch, state.offspring, self.mutation_rate,
                                    state.context)


class EvaluationStep:
  def __init__(self, strategy: Any, target: Literal["offspring", "population"] = "offspring") -> None:
    self.strategy = strategy
    self.target = target

  def run(self, state: GenerationState, timer: PhaseTimer) -> None:
    routes = state.offspring if self.target == "offspring" else state.population
    if routes is None:
      raise RuntimeError("EvaluationStep target='offspring' called with state.offspring is None.")
    keep_gpu = bool(is_device_array(routes) and getattr(self.strategy, "return_gpu", False))
    a = timer.measure("evaluation", assess_with_evaluator, self.strategy, routes, state.context, return_gpu=keep_gpu)
    if self.target == "offspring":
      state.offspring_assessment = a
      state.offspring_fitness = a.objectives
    else:
      state.population_assessment = a
      state.fitness = a.objectives


class SurvivalStep:
  def __init__(self, survivor_selector: Callable) -> None:
    self.survivor_selector = survivor_selector

  def run(self, state: GenerationState, timer: PhaseTimer) -> None:
    if state.offspring is None or state.offspring_fitness is None:
      raise RuntimeError("SurvivalStep called before offspring and offspring_fitness were available.")
    state.population, state.fitness = timer.measure("survival", self.survivor_selector, state.population, state.fitness,
                                                    state.offspring, state.offspring_fitness)
    state.population_assessment = None


class LocalSearchStep:
  def __init__(self, strategy: Any, target: Literal["offspring", "population"] = "offspring", re_evaluate: Any = None):
    self.strategy = strategy
    self.target = target
    self.re_evaluate = re_evaluate

  def run(self, state: GenerationState, timer: PhaseTimer) -> None:
    if self.target == "offspring":
      if state.offspring is None:
        raise RuntimeError("LocalSearchStep target='offspring' called with state.offspring is None.")
      state.offspring = timer.measure("local_search", self.strategy.improve_batch, state.offspring, state.context)
      return
    state.population = timer.measure("local_search", self.strategy.improve_batch, state.population, state.context)
    if self.re_evaluate is not None:
      keep = bool(is_device_array(state.population) and getattr(self.re_evaluate, "return_gpu", False))
      a = timer.measure("evaluation", assess_with_evaluator, self.re_evaluate, state.population, state.context,
                        return_gpu=keep)
      state.population_assessment = a
      state.fitness = a.objectives


@dataclass(frozen=True)
class StageSpec:
  pipeline_steps: Callable[["GeneticAlgorithm"], list]
  post_loop_hook: bool = False
  requires_local_search: bool = True


def _steps_standard(ga: "GeneticAlgorithm") -> list:
  return [SelectionStep(ga.selection, ga.population_size), CrossoverStep(ga.crossover),
          MutationStep(ga.mutation, ga.mutation_rate), EvaluationStep(ga.evaluation, "offspring"),
          SurvivalStep(ga._select_survivors)]


def _steps_post_crossover(ga: "GeneticAlgorithm") -> list:
  if ga.local_search is None:
    return _steps_standard(ga)
  return [SelectionStep(ga.selection, ga.population_size), CrossoverStep(ga.crossover),
          LocalSearchStep(ga.local_search, "offspring"), MutationStep(ga.mutation, ga.mutation_rate),
          EvaluationStep(ga.evaluation, "offspring"), SurvivalStep(ga._select_survivors)]


def _steps_post_mutation(ga: "GeneticAlgorithm") -> list:
  if ga.local_search is None:
    return _steps_standard(ga)
  return [SelectionStep(ga.selection, ga.population_size), CrossoverStep(ga.crossover),
          MutationStep(ga.mutation, ga.mutation_rate), LocalSearchStep(ga.local_search, "offspring"),
          EvaluationStep(ga.evaluation, "offspring"), SurvivalStep(ga._select_survivors)]


def _steps_post_evaluation(ga: "GeneticAlgorithm") -> list:
  if ga.local_search is None:
    return _steps_standard(ga)
  return [SelectionStep(ga.selection, ga.population_size), CrossoverStep(ga.crossover),
          MutationStep(ga.mutation, ga.mutation_rate), EvaluationStep(ga.evaluation, "offspring"),
          SurvivalStep(ga._select_survivors), LocalSearchStep(ga.local_search, "population", re_evaluate=ga.evaluation)]


STAGE_SPECS: Mapping[str, StageSpec] = {
  "none": StageSpec(_steps_standard, post_loop_hook=False, requires_local_search=False),
  "post_crossover": StageSpec(_steps_post_crossover),
  "post_mutation": StageSpec(_steps_post_mutation),
  "post_evaluation": StageSpec(_steps_post_evaluation),
  "post_evolution": StageSpec(_steps_standard, post_loop_hook=True),
}

_PIPELINE_STRATEGY_ATTRS = ("strategy", "local_search", "evaluation", "re_evaluate")


# ------------------------------------------------------------------------------ GA
class GeneticAlgorithm:
  """Strategy-driven GA; same constructor and `evolve` contract as the reference."""

  def __init__(self, population_size: int = 256, mutation_rate: float = 0.02, seed: int | None = 42, *,
               initialization: Any, selection: Any, crossover: Any, mutation: Any, evaluation: Any,
               local_search: Any = None, local_search_stage: str = "post_mutation", enable_phase_timing: bool = True,
               pipeline: list | None = None) -> None:
    if local_search_stage not in STAGE_SPECS:
      raise ValueError(f"Invalid local_search_stage '{local_search_stage}'. Valid stages: {list(STAGE_SPECS.keys())}")
    self.population_size = population_size
    self.mutation_rate = mutation_rate
    self.seed = seed
    self.local_search_stage = local_search_stage
    self.initialization = initialization
    self.selection = selection
    self.crossover = crossover
    self.mutation = mutation
    self.evaluation = evaluation
    self.local_search = local_search
    self.timer = PhaseTimer(enabled=enable_phase_timing)
    self.generation = 0
    self.best_cost_history: list[float] = []
    self.h2d_bytes = 0
    self.d2h_bytes = 0
    self.kernel_launches = 0
    self.custom_pipeline_steps = list(pipeline) if pipeline is not None else []
    if pipeline is not None:
      core = any(isinstance(s, (SelectionStep, CrossoverStep, MutationStep, SurvivalStep)) for s in pipeline)
      self.pipeline = list(pipeline) if core else self._compose_pipeline(pipeline)
    else:
      self.pipeline = self._build_default_pipeline()

  def _compose_pipeline(self, extension_steps: list) -> list:
    steps = self._build_default_pipeline()
    pre: list = []
    for step in extension_steps:
      anchor = getattr(step, "stage_anchor", "post_survival")
      if anchor == "pre_selection":
        pre.append(step)
      elif anchor == "pre_evaluation":
        idx = next((i for i, s in enumerate(steps) if isinstance(s, EvaluationStep) and s.target == "offspring"), len(steps))
        steps.insert(idx, step)
      else:
        steps.append(step)
    return [*pre, *steps]

  def _build_default_pipeline(self) -> list:
    return STAGE_SPECS[self.local_search_stage].pipeline_steps(self)

  def _all_strategies(self) -> list:
    cands = [self.initialization, self.selection, self.crossover, self.mutation, self.evaluation, self.local_search]
    for step in self.pipeline:
      declared = getattr(step, "strategies", None)
      if callable(declared):
        cands.extend(declared())
      else:
        cands.extend(getattr(step, a, None) for a in _PIPELINE_STRATEGY_ATTRS)
    out, seen = [], set()
    for s in cands:
      if s is None or id(s) in seen:
        continue
      seen.add(id(s))
      out.append(s)
    return out

  def _reset_run_metrics(self) -> None:
    self.generation = 0
    self.best_cost_history = []
    self.h2d_bytes = self.d2h_bytes = self.kernel_launches = 0
    self.timer.reset()
    for s in self._all_strategies():
      if hasattr(s, "reset_metrics"):
        s.reset_metrics()

  def warmup(self, context: Any) -> None:
    seen: set[int] = set()
    for step in self.pipeline:
      hook = getattr(step, "warmup", None)
      if not callable(hook):
        continue
      hook(context)
      owned = getattr(step, "strategies", None)
      if callable(owned):
        seen.update(id(s) for s in owned())
    for s in self._all_strategies():
      if id(s) in seen:
        continue
      seen.add(id(s))
      hook = getattr(s, "warmup", None)
      if callable(hook):
        hook(context)

  def _collect_strategy_metrics(self) -> None:
    h = d = k = 0
    for s in self._all_strategies():
      h += int(getattr(s, "h2d_bytes", 0))
      d += int(getattr(s, "d2h_bytes", 0))
      k += int(getattr(s, "kernel_launches", 0))
    self.h2d_bytes, self.d2h_bytes, self.kernel_launches = h, d, k

  def _select_survivors(self, old_pop: Any, old_fitness: Any, new_pop: Any, new_fitness: Any):
    """Stable `(mu + lambda)` survival (`genetic_algorithm.py:618-706`, feasible tours)."""
    dev = is_device_array(old_pop) or is_device_array(new_pop)
    if dev:
      a = old_pop if is_device_array(old_pop) else device_tensor(np.asarray(old_pop, np.int32), torch.int32)
      b = new_pop if is_device_array(new_pop) else device_tensor(np.asarray(new_pop, np.int32), torch.int32)
      pop = torch.cat([a.to(torch.int32), b.to(torch.int32)], dim=0)
      fit = torch.cat([_as_f64(old_fitness, True), _as_f64(new_fitness, True)])
      order = stable_order(fit, self.population_size)
      return _device_take_rows(pop, order), fit[order.long()]
    pop = np.vstack([np.asarray(old_pop), np.asarray(new_pop)])
    fit = np.concatenate([_as_f64(old_fitness, False), _as_f64(new_fitness, False)])
    idx = stable_order(fit, self.population_size)
    return pop[idx], fit[idx]

  @staticmethod
  def _best_meta(fitness: Any) -> tuple[int, float]:
    if is_device_array(fitness):
      idx = int(torch.argmin(fitness).item())
      return idx, float(fitness[idx].item())
    idx = int(np.argmin(fitness))
    return idx, float(fitness[idx])

  @staticmethod
  def _extract_route_at(population: Any, idx: int) -> np.ndarray:
    raw = population[idx]
    if is_device_array(raw):
      return raw.cpu().numpy().astype(np.int32, copy=True)
    return np.asarray(raw, dtype=np.int32).copy()

  def evolve(self, context: Any, customers: Any, max_generations: int, optimal_cost: float | None = None,
             patience: int | None = None) -> tuple[np.ndarray, dict]:
    if len(customers) == 0:
      raise ValueError("customers sequence cannot be empty")
    n = len(customers)
    if patience is None:
      patience = int(2 * math.sqrt(n))
    self._reset_run_metrics()
    timer = self.timer
    population = timer.measure("initialization", self.initialization.initialize, customers, self.population_size, context)
    keep = bool(is_device_array(population) and getattr(self.evaluation, "return_gpu", False))
    pa = timer.measure("evaluation", assess_with_evaluator, self.evaluation, population, context, return_gpu=keep)
    fitness = pa.objectives
    best_idx, best_cost = timer.measure("host_sync", self._best_meta, fitness)
    initial_feasible = best_cost
    best_tour = timer.measure("host_sync", self._extract_route_at, population, best_idx)
    initial_best = best_cost
    self.best_cost_history = [best_cost]
    stall = 0
    stopped_early = False
    stop_reason = "max_generations"
    state = GenerationState(population=population, fitness=fitness, context=context, population_assessment=pa)
    for gen in range(max_generations):
      self.generation = gen + 1
      state.generation = self.generation
      for step in self.pipeline:
        step.run(state, timer)
      ci, cc = timer.measure("host_sync", self._best_meta, state.fitness)
      if cc < best_cost - 1e-6:
        best_tour = timer.measure("host_sync", self._extract_route_at, state.population, ci)
        best_cost = cc
        stall = 0
      else:
        stall += 1
      self.best_cost_history.append(best_cost)
      if optimal_cost is not None and optimal_cost > 0:
        if best_cost <= optimal_cost + 1e-6:
          stopped_early, stop_reason = True, "hit_optimal"
          break
        if (best_cost - optimal_cost) / optimal_cost * 100.0 < 1.0:
          stopped_early, stop_reason = True, "within_1pct_optimal"
          break
      if stall >= patience:
        stopped_early, stop_reason = True, "no_improvements"
        break
    if self.local_search is not None and STAGE_SPECS[self.local_search_stage].post_loop_hook:
      state.population = timer.measure("local_search", self.local_search.improve_batch, state.population, context)
      keep = bool(is_device_array(state.population) and getattr(self.evaluation, "return_gpu", False))
      a = timer.measure("evaluation", assess_with_evaluator, self.evaluation, state.population, context, return_gpu=keep)
      state.population_assessment = a
      state.fitness = a.objectives
      pi, pc = timer.measure("host_sync", self._best_meta, state.fitness)
      if pc <= best_cost:
        best_tour = timer.measure("host_sync", self._extract_route_at, state.population, pi)
        best_cost = pc
        self.best_cost_history[-1] = best_cost
    best_tour = canonicalize_with_evaluator(self.evaluation, best_tour, context)
    self._collect_strategy_metrics()
    self.final_population = state.population
    self.final_fitness = state.fitness
    stats = {
      "initial_fitness": initial_best,
      "initial_feasible_cost": initial_feasible,
      "best_fitness": best_cost,
      "best_is_feasible": True,
      "generations_completed": self.generation,
      "stopped_early": stopped_early,
      "stop_reason": stop_reason,
      "convergence_history": self.best_cost_history,
      "phase_timings": timer.summary(),
      "h2d_bytes": self.h2d_bytes,
      "d2h_bytes": self.d2h_bytes,
      "kernel_launches": self.kernel_launches,
    }
    return best_tour, stats
