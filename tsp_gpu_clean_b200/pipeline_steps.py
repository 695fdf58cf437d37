"""Extension generation steps, mirroring `src/algorithms/pipeline_steps.py` of the reference.

- `PostInitLocalSearchStep` (:85-125): refine the whole population once, at generation 1,
  and re-assess it.
- `EliteOnlyLocalSearchStep` (:128-195): refine the `elite_count` lowest-cost tours after
  survival and scatter them back. Elites are `argsort(fitness)[:k]` with NumPy's default
  sort, whose order among equal values is implementation-defined; only membership
  matters (each elite is refined independently). On the device the elites come from the
  stable `(fitness, index)` rank; when the k-th and (k+1)-th values tie, membership
  would depend on the sort, so those generations take the host `np.argsort` of the
  fitness vector (k + 1 values read back) to keep the reference's choice.
- `PeriodicLocalSearchStep` (:198-285): refine every `interval` generations.
- `PIPELINE_STEP_REGISTRY` / `register_pipeline_step` (:439-466).
"""

from __future__ import annotations

from typing import Any, ClassVar, Literal

import numpy as np

from . import native
from .device import device_tensor, is_device_array, ptr, stream_handle, torch
from .ga import assess_with_evaluator, stable_order


def _warmup_owned(strategies: list, context: Any) -> None:
  for s in strategies:
    hook = getattr(s, "warmup", None)
    if callable(hook):
      hook(context)


class _BaseLocalSearchPipelineStep:
  stage_anchor: ClassVar[str] = "post_survival"

  def __init__(self, local_search: Any, evaluation: Any) -> None:
    if local_search is None:
      raise ValueError(f"{self.__class__.__name__} requires a local_search strategy")
    if evaluation is None:
      raise ValueError(f"{self.__class__.__name__} requires an evaluation strategy")
    self.local_search = local_search
    self.evaluation = evaluation

  def strategies(self) -> list:
    return [self.local_search, self.evaluation]

  def public_params(self) -> dict:
    return {}

  def warmup(self, context: Any) -> None:
    _warmup_owned(self.strategies(), context)


class PostInitLocalSearchStep(_BaseLocalSearchPipelineStep):
  stage_anchor: ClassVar[str] = "pre_selection"

  def run(self, state, timer) -> None:
    if state.generation != 1:
      return
    state.population = timer.measure("local_search", self.local_search.improve_batch, state.population, state.context)
    keep = bool(is_device_array(state.population) and getattr(self.evaluation, "return_gpu", False))
    a = timer.measure("evaluation", assess_with_evaluator, self.evaluation, state.population, state.context, return_gpu=keep)
    state.population_assessment = a
    state.fitness = a.objectives


def elite_indices(fitness: Any, k: int) -> Any:
  """Elite rows: `np.argsort(fitness)[:k]` membership, on the device when fitness is."""
  if not is_device_array(fitness):
    return np.argsort(np.asarray(fitness))[:k]
  m = int(fitness.shape[0])
  if k >= m:
    return torch.arange(m, dtype=torch.int32, device=fitness.device)
  order = stable_order(fitness, k + 1)
  edge = fitness.to(torch.float64)[order[k - 1 : k + 1].long()].cpu().numpy()
  if edge[0] == edge[1]:  # boundary tie: the host sort decides membership
    host = np.argsort(fitness.cpu().numpy())[:k]
    return torch.from_numpy(host.astype(np.int32)).to(fitness.device)
  return order[:k].contiguous()


def _scatter_rows(dst: "torch.Tensor", rows: "torch.Tensor", src: "torch.Tensor") -> None:
  src_c = src.contiguous()  # keep the (possibly new) tensor alive until the launch is enqueued
  native.call("tspb_scatter_rows", ptr(src_c), int(src_c.shape[0]), int(src_c.shape[1]), ptr(rows), ptr(dst),
              int(dst.shape[0]), stream_handle())


class EliteOnlyLocalSearchStep(_BaseLocalSearchPipelineStep):
  stage_anchor: ClassVar[str] = "post_survival"

  def __init__(self, local_search: Any, evaluation: Any, elite_count: int = 10) -> None:
    super().__init__(local_search, evaluation)
    if elite_count <= 0:
      raise ValueError(f"elite_count must be > 0, got {elite_count}")
    self.elite_count = elite_count

  def public_params(self) -> dict:
    return {"elite_count": self.elite_count}

  def run(self, state, timer) -> None:
    pop_size = int(state.population.shape[0])
    k = min(self.elite_count, pop_size)
    if k <= 0:
      return
    dev = is_device_array(state.population)
    if dev:
      fit = state.fitness if is_device_array(state.fitness) else device_tensor(np.asarray(state.fitness), torch.float64)
      idx = elite_indices(fit, k).to(torch.int32).contiguous()
      from .ga import _device_take_rows

      elite = _device_take_rows(state.population, idx)
    else:
      idx = elite_indices(np.asarray(state.fitness), k)
      elite = state.population[idx]
    improved = timer.measure("local_search", self.local_search.improve_batch, elite, state.context)
    keep = bool(is_device_array(improved) and getattr(self.evaluation, "return_gpu", False))
    a = timer.measure("evaluation", assess_with_evaluator, self.evaluation, improved, state.context, return_gpu=keep)
    if dev:
      imp = improved if is_device_array(improved) else device_tensor(np.asarray(improved, np.int32), torch.int32)
      imp = imp.to(torch.int32)
      _scatter_rows(state.population, idx, imp)
      obj = a.objectives if is_device_array(a.objectives) else device_tensor(np.asarray(a.objectives), torch.float64)
      if not is_device_array(state.fitness):
        state.fitness = device_tensor(np.asarray(state.fitness), torch.float64)
      state.fitness[idx.long()] = obj.to(torch.float64)
    else:
      state.population[idx] = np.asarray(improved)
      state.fitness[idx] = np.asarray(a.objectives)
    state.population_assessment = None


class PeriodicLocalSearchStep:
  def __init__(self, local_search: Any, interval: int = 10, target: Literal["offspring", "population"] = "population",
               re_evaluate: Any = None) -> None:
    if local_search is None:
      raise ValueError("PeriodicLocalSearchStep requires a local_search strategy")
    if interval <= 0:
      raise ValueError(f"interval must be > 0, got {interval}")
    if target not in ("offspring", "population"):
      raise ValueError(f"target must be 'offspring' or 'population', got {target!r}")
    if target == "population" and re_evaluate is None:
      raise ValueError("re_evaluate EvaluationStrategy is required when target='population'")
    self.local_search = local_search
    self.interval = interval
    self.target = target
    self.re_evaluate = re_evaluate

  @property
  def stage_anchor(self) -> str:
    return "pre_evaluation" if self.target == "offspring" else "post_survival"

  def strategies(self) -> list:
    return [self.local_search] + ([self.re_evaluate] if self.re_evaluate is not None else [])

  def public_params(self) -> dict:
    return {"interval": self.interval, "target": self.target}

  def warmup(self, context: Any) -> None:
    _warmup_owned(self.strategies(), context)

  def run(self, state, timer) -> None:
    if state.generation % self.interval != 0:
      return
    if self.target == "offspring":
      if state.offspring is None:
        raise RuntimeError("PeriodicLocalSearchStep(target='offspring') called before offspring exists.")
      state.offspring = timer.measure("local_search", self.local_search.improve_batch, state.offspring, state.context)
      return
    state.population = timer.measure("local_search", self.local_search.improve_batch, state.population, state.context)
    if self.re_evaluate is not None:
      keep = bool(is_device_array(state.population) and getattr(self.re_evaluate, "return_gpu", False))
      a = timer.measure("evaluation", assess_with_evaluator, self.re_evaluate, state.population, state.context,
                        return_gpu=keep)
      state.population_assessment = a
      state.fitness = a.objectives


PIPELINE_STEP_REGISTRY: dict[str, type] = {
  "EliteOnlyLocalSearchStep": EliteOnlyLocalSearchStep,
  "PeriodicLocalSearchStep": PeriodicLocalSearchStep,
  "PostInitLocalSearchStep": PostInitLocalSearchStep,
}


def register_pipeline_step(name: str, step_cls: type, *, overwrite: bool = False) -> None:
  if not isinstance(name, str) or not name.strip():
    raise ValueError("Pipeline step name must be a non-empty string.")
  if not isinstance(step_cls, type):
    raise TypeError(f"Expected a pipeline step class (type), got {type(step_cls).__name__}.")
  if not callable(getattr(step_cls, "run", None)):
    raise TypeError(f"Pipeline step class '{step_cls.__name__}' must define a callable 'run(state, timer)' method.")
  if name in PIPELINE_STEP_REGISTRY and not overwrite:
    raise ValueError(f"Pipeline step '{name}' is already registered. Pass overwrite=True to replace it.")
  PIPELINE_STEP_REGISTRY[name] = step_cls
