"""Single-file entry point for `{"module": ".../tsp_gpu_clean_b200/plugin.py", "class": ...}` specs.

The reference's runner loads a `.py` module spec as a standalone file
(`src/benchmarking/runner/spec_resolver.py:29-71`), so package-relative imports inside the
strategy modules would not resolve. This file uses absolute imports only: it puts the
repository root on `sys.path`, imports the package and re-exports every B200 strategy,
pipeline step and the fused algorithm class, so one path serves every slot of a config.
"""

from __future__ import annotations

import sys
from pathlib import Path

_ROOT = str(Path(__file__).resolve().parents[1])
if _ROOT not in sys.path:
  sys.path.insert(0, _ROOT)

from tsp_gpu_clean_b200.pipeline_steps import (  # noqa: E402
  EliteOnlyLocalSearchStep,
  PeriodicLocalSearchStep,
  PostInitLocalSearchStep,
)
from tsp_gpu_clean_b200.runner import FusedGeneticAlgorithm  # noqa: E402
from tsp_gpu_clean_b200.strategies import (  # noqa: E402
  CrossoverB200PermOrder,
  CrossoverB200PermPartiallyMapped,
  EvaluationB200Cost,
  InitializationB200PermRandom,
  InitializationB200TourNearestNeighbor,
  LocalSearchB200OrOpt,
  LocalSearchB200ThreeOpt,
  LocalSearchB200TourTwoOpt,
  MutationB200PermInversion,
  MutationB200PermSwap,
  SelectionB200Tournament,
)

__all__ = [
  "CrossoverB200PermOrder",
  "CrossoverB200PermPartiallyMapped",
  "EliteOnlyLocalSearchStep",
  "EvaluationB200Cost",
  "FusedGeneticAlgorithm",
  "InitializationB200PermRandom",
  "InitializationB200TourNearestNeighbor",
  "LocalSearchB200OrOpt",
  "LocalSearchB200ThreeOpt",
  "LocalSearchB200TourTwoOpt",
  "MutationB200PermInversion",
  "MutationB200PermSwap",
  "PeriodicLocalSearchStep",
  "PostInitLocalSearchStep",
  "SelectionB200Tournament",
]
