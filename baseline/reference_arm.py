"""The reference's own CPU 2-opt, timed for `bench.py --impl reference`.

The reference (lucasgaldinos/tsp_gpu_clean) is installed offline into `baseline/_ref`
(`pip install --no-index --no-build-isolation --no-deps --target baseline/_ref <checkout>`),
or found as a checkout through TSPB_REFERENCE. Its CPU path for the 2-opt hot path is
`LocalSearchCPUTourTwoOpt.improve_batch`
(src/algorithms/strategies/local_search/two_opt.py:565-628) on a `ProblemContext`
(src/protocols/problem_context.py:75-616) built from a `Problem`
(src/data_models/problem.py). Nothing of this repository runs on that path.

Two things surround the call:
- the `converter` package of the `routing-data` dependency is absent from the offline
  wheelhouse; the 2-opt path never calls it, so a stand-in module lets the reference's
  `distances` package import (its TSPLIB metric functions raise if called);
- the metric counts the (i, j) pairs the scan evaluates, so `_pair_blocks`
  (two_opt.py:303-367), the generator every acceptance rule consumes, is wrapped by a
  pass-through that sums the sizes of the blocks it yields. The blocks, their order and
  every move are the reference's.
"""

from __future__ import annotations

import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
INSTALLED = os.path.join(HERE, "_ref")

_CONVERTER_STANDIN = '''
def nint(x):
    return int(x + 0.5)
def _unavailable(*args, **kwargs):
    raise NotImplementedError("routing-data is not installed")
att = ceil_2d = euclidean_2d = euclidean_3d = manhattan_2d = manhattan_3d = _unavailable
maximum_2d = maximum_3d = xray1 = _unavailable
'''

_READY = False
_COUNTS = {"pairs": 0, "passes": 0}


def import_root() -> str | None:
  """Directory holding the reference's packages (`algorithms`, `protocols`, ...), or None."""
  root = os.environ.get("TSPB_REFERENCE")
  if root and os.path.isdir(os.path.join(root, "src", "algorithms")):
    return os.path.join(root, "src")
  if os.path.isdir(os.path.join(INSTALLED, "algorithms")) and os.path.isdir(os.path.join(INSTALLED, "protocols")):
    return INSTALLED
  return None


def setup() -> None:
  """Put the reference on sys.path after the `converter` stand-in (once per process) and
  wrap its pair generator with the counter."""
  global _READY
  if _READY:
    return
  src = import_root()
  if src is None:
    raise RuntimeError("the reference is not installed (baseline/_ref) and TSPB_REFERENCE is unset")
  tmp = tempfile.mkdtemp(prefix="tspb_ref_standin_")
  pkg = os.path.join(tmp, "converter", "utils")
  os.makedirs(pkg)
  open(os.path.join(tmp, "converter", "__init__.py"), "w").close()
  open(os.path.join(pkg, "__init__.py"), "w").close()
  with open(os.path.join(pkg, "cost.py"), "w") as fh:
    fh.write(_CONVERTER_STANDIN)
  sys.path.insert(0, tmp)
  sys.path.insert(0, src)
  from algorithms.strategies import LocalSearchCPUTourTwoOpt

  blocks = LocalSearchCPUTourTwoOpt._pair_blocks

  def counted(self, *a, **kw):
    _COUNTS["passes"] += 1
    for i_idx, j_idx in blocks(self, *a, **kw):
      _COUNTS["pairs"] += int(i_idx.size)
      yield i_idx, j_idx

  LocalSearchCPUTourTwoOpt._pair_blocks = counted
  _READY = True


def two_opt_worker(args):
  """Refine one tour with the reference's CPU 2-opt, each mode to a local optimum.

  args = (coords, tour, modes, candidate_k). Returns ({mode: (tour, (passes, pairs))},
  seconds inside improve_batch)."""
  coords, tour, modes, k = args
  setup()
  from algorithms.strategies import LocalSearchCPUTourTwoOpt
  from data_models.problem import Problem
  from protocols.problem_context import ProblemContext

  problem = Problem(name="synthetic", dimension=len(coords), problem_type="TSP", edge_type="EUC_2D",
                    coordinates=np.asarray(coords, dtype=np.float64), distances=None)
  ctx = ProblemContext(problem, xp=np, seed=0)
  ctx.get_cpu_distances()  # the context's matrix and k-NN table, built before the timed calls
  ctx.get_cpu_candidate_list(k)
  out, secs = {}, 0.0
  for mode in modes:
    ls = LocalSearchCPUTourTwoOpt(max_iterations=10**9, mode=mode, candidate_k=k)
    _COUNTS["pairs"] = _COUNTS["passes"] = 0
    t0 = time.perf_counter()
    res = ls.improve_batch(np.ascontiguousarray(tour[None, :]).copy(), ctx)
    secs += time.perf_counter() - t0
    out[mode] = (np.asarray(res, dtype=np.int32)[0], (_COUNTS["passes"], _COUNTS["pairs"]))
  return out, secs


def ga_gens_per_s(coords, population: int, elite: int, post_init: bool, sample_gens: int, options: dict,
                  seed: int = 42) -> dict:
  """Generations/s of the reference's own `GeneticAlgorithm.evolve`
  (src/algorithms/metaheuristics/genetic_algorithm.py:789-965) with its CPU strategies, on
  one core: `options` picks the configuration (`crossover` "pmx"/"ox", `mutation`
  "inversion"/"swap", `init` "nn"/"random", `stage`, mutation `rate`), with 2-opt best
  k = 20 x 10 through `PostInitLocalSearchStep` / `EliteOnlyLocalSearchStep`
  (src/algorithms/pipeline_steps.py:103-195) as configured. The loop time is a run of
  `sample_gens` generations minus a run of none (initialisation and the post-init
  refinement), so it counts generations only. `seed` seeds the context and every strategy."""
  setup()
  from algorithms import GeneticAlgorithm
  from algorithms.pipeline_steps import EliteOnlyLocalSearchStep, PostInitLocalSearchStep
  from algorithms.strategies import (
    CrossoverCPUPermOrder,
    CrossoverCPUPermPartiallyMapped,
    EvaluationCPUCost,
    InitializationCPUPermRandom,
    InitializationCPUTourNearestNeighbor,
    LocalSearchCPUTourTwoOpt,
    MutationCPUPermInversion,
    MutationCPUPermSwap,
    SelectionCPUTournament,
  )
  from data_models.problem import Problem
  from protocols.problem_context import ProblemContext

  problem = Problem(name="synthetic", dimension=len(coords), problem_type="TSP", edge_type="EUC_2D",
                    coordinates=np.asarray(coords, dtype=np.float64), distances=None)

  def run(gens: int):
    ctx = ProblemContext(problem, xp=np, seed=seed)
    ctx.get_cpu_distances()
    ctx.get_cpu_candidate_list(20)
    ctx.get_cpu_candidate_list(5)
    ls = LocalSearchCPUTourTwoOpt(mode="best", max_iterations=10, candidate_k=20)
    ev = EvaluationCPUCost()
    steps = []
    if post_init:
      steps.append(PostInitLocalSearchStep(local_search=ls, evaluation=ev))
    if elite:
      steps.append(EliteOnlyLocalSearchStep(local_search=ls, evaluation=ev, elite_count=elite))
    init = (InitializationCPUPermRandom(seed=seed) if options["init"] == "random"
            else InitializationCPUTourNearestNeighbor(k=5, seed=seed))
    xo = CrossoverCPUPermOrder(seed=seed) if options["crossover"] == "ox" else CrossoverCPUPermPartiallyMapped(seed=seed)
    mut = MutationCPUPermSwap(seed=seed) if options["mutation"] == "swap" else MutationCPUPermInversion(seed=seed)
    ga = GeneticAlgorithm(population_size=population, mutation_rate=options["rate"], seed=seed, initialization=init,
                          selection=SelectionCPUTournament(k=5, seed=seed), crossover=xo, mutation=mut,
                          local_search=ls, evaluation=ev, local_search_stage=options["stage"],
                          pipeline=steps or None)
    t0 = time.perf_counter()
    _, stats = ga.evolve(context=ctx, customers=list(range(len(coords))), max_generations=gens, patience=10**9)
    return time.perf_counter() - t0, stats

  t_init, _ = run(0)
  t_all, stats = run(sample_gens)
  loop = max(t_all - t_init, 1e-9)
  return {"value": sample_gens / loop, "gens": sample_gens, "loop_s": loop,
          "history": [float(v) for v in stats["convergence_history"]]}
