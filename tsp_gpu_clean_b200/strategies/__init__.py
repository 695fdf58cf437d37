"""B200 strategies and their registry (mirrors `src/algorithms/strategies/__init__.py:87-207`)."""

from __future__ import annotations

from .initialization import InitializationB200PermRandom, InitializationB200TourNearestNeighbor
from .local_search import LocalSearchB200TourTwoOpt
from .or_opt import LocalSearchB200OrOpt
from .three_opt import LocalSearchB200ThreeOpt
from .operators import (
  CrossoverB200PermOrder,
  CrossoverB200PermPartiallyMapped,
  EvaluationB200Cost,
  MutationB200PermInversion,
  MutationB200PermSwap,
  SelectionB200Tournament,
)

STRATEGY_REGISTRY: dict[str, type] = {
  "CrossoverB200PermOrder": CrossoverB200PermOrder,
  "CrossoverB200PermPartiallyMapped": CrossoverB200PermPartiallyMapped,
  "EvaluationB200Cost": EvaluationB200Cost,
  "InitializationB200PermRandom": InitializationB200PermRandom,
  "InitializationB200TourNearestNeighbor": InitializationB200TourNearestNeighbor,
  "LocalSearchB200OrOpt": LocalSearchB200OrOpt,
  "LocalSearchB200ThreeOpt": LocalSearchB200ThreeOpt,
  "LocalSearchB200TourTwoOpt": LocalSearchB200TourTwoOpt,
  "MutationB200PermInversion": MutationB200PermInversion,
  "MutationB200PermSwap": MutationB200PermSwap,
  "SelectionB200Tournament": SelectionB200Tournament,
}

#: Required methods per protocol (`src/protocols/algorithm_strategies.py:62-210`).
PROTOCOL_METHODS: dict[str, tuple[str, ...]] = {
  "InitializationStrategy": ("initialize",),
  "SelectionStrategy": ("select", "select_batch"),
  "CrossoverStrategy": ("crossover", "crossover_batch"),
  "MutationStrategy": ("mutate", "mutate_batch"),
  "LocalSearchStrategy": ("improve", "improve_batch"),
  "EvaluationStrategy": ("assess_batch", "canonicalize_route", "evaluate", "evaluate_batch"),
}


def register_strategy(name: str, strategy_cls: type, *, overwrite: bool = False) -> None:
  """Register a class implementing at least one strategy protocol (`__init__.py:175-207`)."""
  if not isinstance(name, str) or not name.strip():
    raise ValueError("Strategy name must be a non-empty string.")
  if not isinstance(strategy_cls, type):
    raise TypeError(f"Expected a strategy class (type), got {type(strategy_cls).__name__}.")
  if not any(all(callable(getattr(strategy_cls, m, None)) for m in ms) for ms in PROTOCOL_METHODS.values()):
    raise TypeError(f"Strategy class '{strategy_cls.__name__}' does not implement any strategy protocol.")
  if name in STRATEGY_REGISTRY and not overwrite:
    raise ValueError(f"Strategy '{name}' is already registered. Pass overwrite=True to replace it.")
  STRATEGY_REGISTRY[name] = strategy_cls


__all__ = [
  "STRATEGY_REGISTRY",
  "CrossoverB200PermOrder",
  "CrossoverB200PermPartiallyMapped",
  "EvaluationB200Cost",
  "InitializationB200PermRandom",
  "InitializationB200TourNearestNeighbor",
  "LocalSearchB200OrOpt",
  "LocalSearchB200ThreeOpt",
  "LocalSearchB200TourTwoOpt",
  "MutationB200PermInversion",
  "MutationB200PermSwap",
  "SelectionB200Tournament",
  "register_strategy",
]
