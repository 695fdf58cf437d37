"""The B200 strategies inside the reference's own GA loop and ProblemContext.

The reference's `GeneticAlgorithm.evolve` (src/algorithms/metaheuristics/genetic_algorithm.py:
789-965) runs with its own `ProblemContext` (src/protocols/problem_context.py:75-616) and its
own pipeline steps (`PostInitLocalSearchStep`, `EliteOnlyLocalSearchStep`,
src/algorithms/pipeline_steps.py:103-195), with every strategy slot filled by this
package's B200 class: nearest-neighbour init, tournament, PMX, inversion, 2-opt and cost.
The run must equal the recorded run of the reference's CPU strategies on the same
100-city instance (`ga.npz`, tag c1): the population digest and fitness after every
generation, the best-fitness history, the best tour and the generator state at the end.

The reference is found through TSPB_REFERENCE (a checkout) or its offline install under
`baseline/_ref`; the run happens in a child process so the reference's top-level
packages (`algorithms`, `protocols`, `utils`, ...) stay out of the test process.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from reference_env import import_root

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = import_root()

CHILD = textwrap.dedent("""
  import hashlib, json, sys
  import numpy as np
  sys.path.insert(0, {golden!r})
  import make_golden
  make_golden.setup_import_root({src!r})
  from algorithms import GeneticAlgorithm
  from algorithms.pipeline_steps import EliteOnlyLocalSearchStep, PostInitLocalSearchStep
  from data_models.problem import Problem
  from protocols.problem_context import ProblemContext
  from tsp_gpu_clean_b200 import instances
  from tsp_gpu_clean_b200.strategies import (CrossoverB200PermPartiallyMapped, EvaluationB200Cost,
                                             InitializationB200TourNearestNeighbor, LocalSearchB200TourTwoOpt,
                                             MutationB200PermInversion, SelectionB200Tournament)

  class Recorder:
    stage_anchor = "post_survival"
    def __init__(self):
      self.digests, self.fitness = [], []
    def run(self, state, timer):
      pop = np.asarray(state.population, dtype=np.int32)
      self.digests.append(hashlib.sha256(np.ascontiguousarray(pop).tobytes()).hexdigest())
      self.fitness.append(np.asarray(state.fitness, dtype=np.float64).tolist())

  coords = instances.uniform_instance(100, 42)
  prob = Problem(name="synthetic", dimension=100, problem_type="TSP", edge_type="EUC_2D",
                 coordinates=np.asarray(coords, dtype=np.float64), distances=None)
  ctx = ProblemContext(prob, xp=np, seed=42)
  ls = LocalSearchB200TourTwoOpt(mode="best", max_iterations=10, candidate_k=20)
  ev = EvaluationB200Cost()
  rec = Recorder()
  steps = [PostInitLocalSearchStep(local_search=ls, evaluation=ev),
           EliteOnlyLocalSearchStep(local_search=ls, evaluation=ev, elite_count=16), rec]
  ga = GeneticAlgorithm(population_size=128, mutation_rate=0.05, seed=42,
                        initialization=InitializationB200TourNearestNeighbor(k=5, seed=42),
                        selection=SelectionB200Tournament(k=5, seed=42),
                        crossover=CrossoverB200PermPartiallyMapped(seed=42),
                        mutation=MutationB200PermInversion(seed=42), local_search=ls, evaluation=ev,
                        local_search_stage="none", pipeline=steps)
  best, stats = ga.evolve(context=ctx, customers=list(range(100)), max_generations=50, patience=10**9)
  kinds = sorted({{type(s).__module__.split(".")[0] for s in (ga.initialization, ga.selection, ga.crossover,
                                                              ga.mutation, ga.local_search, ga.evaluation)}})
  print(json.dumps({{"digests": rec.digests, "fitness": rec.fitness,
                    "history": [float(v) for v in stats["convergence_history"]],
                    "gens": int(stats["generations_completed"]), "best": np.asarray(best).tolist(),
                    "rng": int(ctx.rng.bit_generator.state["state"]["state"] % (1 << 63)),
                    "ga_module": type(ga).__module__, "ctx_module": type(ctx).__module__,
                    "strategy_packages": kinds, "two_opt_launches": int(ls.kernel_launches)}}))
""")


@pytest.mark.skipif(SRC is None, reason="reference not present (TSPB_REFERENCE or baseline/_ref)")
def test_reference_evolve_with_b200_strategies_equals_recorded_run(golden):
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  script = CHILD.format(golden=os.path.join(ROOT, "tests", "golden"), src=SRC)
  out = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=900, cwd=ROOT)
  assert out.returncode == 0, out.stderr[-3000:]
  got = json.loads(out.stdout.strip().splitlines()[-1])
  # the loop and the context are the reference's; every strategy is this package's
  assert got["ga_module"].startswith("algorithms.") and got["ctx_module"] == "protocols.problem_context"
  assert got["strategy_packages"] == ["tsp_gpu_clean_b200"]
  assert got["two_opt_launches"] > 0
  g = golden("ga.npz")
  assert got["gens"] == int(g["c1_gens"])
  assert got["digests"] == [str(d) for d in g["c1_digests"]]
  assert np.array_equal(np.asarray(got["fitness"], dtype=np.float64), g["c1_fitness"])
  assert got["history"] == [float(v) for v in g["c1_history"]]
  assert np.array_equal(np.asarray(got["best"], dtype=np.int32), g["c1_best"])
  assert got["rng"] == int(g["c1_rng"][0])
