"""Generate the golden fixtures by running the reference's own CPU strategies.

Run in a container that holds the reference checkout:

    python tests/golden/make_golden.py /path/to/tsp_gpu_clean

The reference imports `converter.utils.cost` from its git-only dependency
`routing-data` (v0.3.0), which is not installable offline; the hot path never
calls it, so this script writes a throwaway stand-in package into a temporary
directory first. Nothing from the reference is copied: the fixtures hold only
inputs and the outputs the reference produced for them.

Outputs (NumPy `.npz`, committed next to this script):
- `two_opt_small.npz`  2-opt best/first/multi_move, exhaustive and k-NN, n = 4..150,
                       plus integer-lattice tie cases and duplicate-candidate tables;
- `two_opt_c2.npz`     four tours of the 1000-city, 20-cluster instance refined to a
                       local optimum in best and first mode, with pass and pair counts;
- `ox_swap.npz`        Order Crossover and swap mutation batches, and two GA runs with them
                       (`python make_golden.py <reference root> ox` regenerates only this file)
- `distances.npz`      distance matrices and k-NN tables of every coordinate-based TSPLIB
                       edge type on seeded synthetic coordinates (`... dist`)
- `three_opt.npz`      exhaustive steepest 3-opt moves and refinements of the reference's
                       CPU 3-opt (`... three_opt`)
- `stage.npz`          random-permutation populations, and GA runs with 2-opt on every
                       offspring (`post_mutation`), two in the Chapter-4 configuration
                       (`... stage` regenerates only this file)
- `ops.npz`            tournament selection, PMX, inversion, tour cost, candidate
                       lists and the EUC_2D matrix on seeded inputs;
- `ga.npz`             full GA runs (the 100-city memetic run for 50 generations, a
                       3-generation 2000-city/512-tour run with 64 elites, and small
                       runs for every local-search stage), recorded per generation.
"""

from __future__ import annotations

import hashlib
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

_STUB = '''
def nint(x):
    return int(x + 0.5)
def _unavailable(*args, **kwargs):
    raise NotImplementedError("routing-data is not installed")
att = ceil_2d = euclidean_2d = euclidean_3d = manhattan_2d = manhattan_3d = _unavailable
maximum_2d = maximum_3d = xray1 = _unavailable
'''


def _setup(ref_root: str) -> None:
  """Import root of a reference checkout (its `src/`), with the stand-in dependency."""
  setup_import_root(os.path.join(ref_root, "src"))


def setup_import_root(src: str) -> None:
  """Put the reference's packages (a checkout's `src/`, or an installed copy holding
  `algorithms/`, `protocols/`, ...) and this repository on `sys.path`, after a stand-in
  for the uninstallable `converter` package."""
  tmp = tempfile.mkdtemp(prefix="golden_stub_")
  pkg = os.path.join(tmp, "converter", "utils")
  os.makedirs(pkg)
  open(os.path.join(tmp, "converter", "__init__.py"), "w").close()
  open(os.path.join(pkg, "__init__.py"), "w").close()
  with open(os.path.join(pkg, "cost.py"), "w") as fh:
    fh.write(_STUB)
  sys.path.insert(0, tmp)
  sys.path.insert(0, src)
  sys.path.insert(0, REPO)


def digest(a: np.ndarray) -> str:
  return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def lattice_matrix(n: int) -> np.ndarray:
  side = int(np.ceil(np.sqrt(n)))
  coords = np.array([[x, y] for x in range(side) for y in range(side)][:n], dtype=float)
  diff = coords[:, None, :] - coords[None, :, :]
  d = np.floor(np.sqrt((diff**2).sum(axis=2)) + 0.5).astype(np.int32)
  np.fill_diagonal(d, 0)
  return d


def main(ref_root: str) -> None:
  _setup(ref_root)
  from algorithms import GeneticAlgorithm
  from algorithms.pipeline_steps import EliteOnlyLocalSearchStep, PeriodicLocalSearchStep, PostInitLocalSearchStep
  from algorithms.strategies import (
    CrossoverCPUPermPartiallyMapped,
    EvaluationCPUCost,
    InitializationCPUTourNearestNeighbor,
    LocalSearchCPUTourTwoOpt,
    MutationCPUPermInversion,
    SelectionCPUTournament,
  )
  from data_models.problem import Problem
  from protocols.problem_context import ProblemContext

  from tsp_gpu_clean_b200 import instances

  def coord_problem(coords, name="synthetic"):
    return Problem(name=name, dimension=len(coords), problem_type="TSP", edge_type="EUC_2D",
                   coordinates=np.asarray(coords, dtype=np.float64), distances=None)

  def matrix_problem(d, name="explicit"):
    return Problem(name=name, dimension=d.shape[0], problem_type="TSP", edge_type="EXPLICIT",
                   coordinates=None, distances=d)

  # ------------------------------------------------------------------ 2-opt small
  out: dict[str, np.ndarray] = {}
  case = 0
  t0 = time.time()
  for n in (4, 5, 6, 8, 10, 17, 40, 100, 150):
    coords = instances.uniform_instance(n, 1000 + n)
    prob = coord_problem(coords)
    for k in (None, 3, 20):
      for mode in ("best", "first", "multi_move"):
        for iters in (1, 3, 10, 100000):
          ctx = ProblemContext(prob, xp=np, seed=0)
          tours = instances.random_tours(n, 4, 7 * n + (k or 0) + 31 * iters % 97)
          ls = LocalSearchCPUTourTwoOpt(max_iterations=iters, mode=mode, candidate_k=k)
          res = ls.improve_batch(tours.copy(), ctx)
          key = f"c{case}"
          out[key + "_coords"] = coords
          out[key + "_meta"] = np.array([n, -1 if k is None else k, ("best", "first", "multi_move").index(mode), iters])
          out[key + "_in"] = tours
          out[key + "_out"] = np.asarray(res, dtype=np.int32)
          if k is not None:
            out[key + "_cand"] = ctx.get_cpu_candidate_list(k)
          case += 1
  # integer lattice: many tied gains (explicit matrices, candidate tables recorded)
  for n in (9, 16, 25, 36):
    d = lattice_matrix(n)
    prob = matrix_problem(d)
    for k in (None, 3):
      for mode in ("best", "first", "multi_move"):
        ctx = ProblemContext(prob, xp=np, seed=0)
        tours = instances.random_tours(n, 4, 31 * n + (k or 0))
        res = LocalSearchCPUTourTwoOpt(max_iterations=10, mode=mode, candidate_k=k).improve_batch(tours.copy(), ctx)
        key = f"c{case}"
        out[key + "_dist"] = d
        out[key + "_meta"] = np.array([n, -1 if k is None else k, ("best", "first", "multi_move").index(mode), 10])
        out[key + "_in"] = tours
        out[key + "_out"] = np.asarray(res, dtype=np.int32)
        if k is not None:
          out[key + "_cand"] = ctx.get_cpu_candidate_list(k)
        case += 1
  # user-supplied candidate tables with repeated neighbours (duplicates are kept)
  for n in (12, 40):
    coords = instances.uniform_instance(n, 555 + n)
    prob = coord_problem(coords)
    base = ProblemContext(prob, xp=np, seed=0).get_cpu_candidate_list(6)
    dup = np.concatenate([base[:, :3], base[:, :3]], axis=1).astype(np.int32)
    for mode in ("best", "first", "multi_move"):
      ctx = ProblemContext(prob, xp=np, seed=0, candidate_cache={6: dup})
      tours = instances.random_tours(n, 4, 99 + n)
      res = LocalSearchCPUTourTwoOpt(max_iterations=100000, mode=mode, candidate_k=6).improve_batch(tours.copy(), ctx)
      key = f"c{case}"
      out[key + "_coords"] = coords
      out[key + "_meta"] = np.array([n, 6, ("best", "first", "multi_move").index(mode), 100000])
      out[key + "_in"] = tours
      out[key + "_out"] = np.asarray(res, dtype=np.int32)
      out[key + "_cand"] = dup
      case += 1
  out["num_cases"] = np.array(case)
  np.savez_compressed(os.path.join(HERE, "two_opt_small.npz"), **out)
  print(f"two_opt_small: {case} cases in {time.time() - t0:.1f}s")

  # ------------------------------------------------ 2-opt subset of the 1024-tour, 1000-city workload
  t0 = time.time()
  counts = {"pairs": 0, "passes": 0}
  orig_blocks = LocalSearchCPUTourTwoOpt._pair_blocks

  def counting_blocks(self, *a, **kw):
    counts["passes"] += 1
    for i_idx, j_idx in orig_blocks(self, *a, **kw):
      counts["pairs"] += int(i_idx.size)
      yield i_idx, j_idx

  LocalSearchCPUTourTwoOpt._pair_blocks = counting_blocks
  coords, tours = instances.two_opt_workload(tours=4)
  prob = coord_problem(coords, "c2")
  c2: dict[str, np.ndarray] = {"coords": coords, "tours_in": tours}
  for mode in ("best", "first"):
    outs, stats = [], []
    for t in range(len(tours)):
      ctx = ProblemContext(prob, xp=np, seed=0)
      counts["pairs"] = counts["passes"] = 0
      r = LocalSearchCPUTourTwoOpt(max_iterations=10**9, mode=mode, candidate_k=20).improve_batch(tours[t : t + 1].copy(), ctx)
      outs.append(np.asarray(r)[0])
      stats.append((counts["passes"], counts["pairs"]))
    c2[f"{mode}_out"] = np.stack(outs)
    c2[f"{mode}_stats"] = np.array(stats, dtype=np.int64)
  c2["cand20"] = ProblemContext(prob, xp=np, seed=0).get_cpu_candidate_list(20)
  LocalSearchCPUTourTwoOpt._pair_blocks = orig_blocks
  np.savez_compressed(os.path.join(HERE, "two_opt_c2.npz"), **c2)
  print(f"two_opt_c2 in {time.time() - t0:.1f}s: {c2['best_stats'].tolist()} {c2['first_stats'].tolist()}")

  # ------------------------------------------------------------------ operators
  t0 = time.time()
  ops: dict[str, np.ndarray] = {}
  for tag, n, pop_size, rate in (("a", 52, 129, 0.05), ("b", 100, 128, 0.5), ("c", 1000, 64, 1.0), ("d", 7, 10, 0.0)):
    coords = instances.uniform_instance(n, 4242 + n)
    prob = coord_problem(coords)
    ctx = ProblemContext(prob, xp=np, seed=123 + n)
    pop = instances.random_tours(n, pop_size, 17 + n)
    ev = EvaluationCPUCost()
    fit = np.asarray(ev.assess_batch(pop, ctx).objectives)
    sel = SelectionCPUTournament(k=5, seed=1).select_batch(pop, fit, pop_size, ctx)
    pmx = CrossoverCPUPermPartiallyMapped(seed=1).crossover_batch(sel, ctx)
    inv = MutationCPUPermInversion(seed=1).mutate_batch(pmx, rate, ctx)
    ops[f"{tag}_coords"] = coords
    ops[f"{tag}_meta"] = np.array([n, pop_size, 123 + n])
    ops[f"{tag}_rate"] = np.array(rate)
    ops[f"{tag}_pop"] = pop
    ops[f"{tag}_fit"] = fit
    ops[f"{tag}_sel"] = np.asarray(sel)
    ops[f"{tag}_pmx"] = np.asarray(pmx)
    ops[f"{tag}_inv"] = np.asarray(inv)
    ops[f"{tag}_rng_state"] = np.array([ctx.rng.bit_generator.state["state"]["state"] % (1 << 63)], dtype=np.int64)
  # EUC_2D matrix and k-NN tables, including exact .5 distances
  coords = instances.uniform_instance(300, 77)
  coords[:4] = [[0.0, 0.0], [0.5, 0.0], [1.5, 2.0], [3.0, 4.0]]
  prob = coord_problem(coords)
  ctx = ProblemContext(prob, xp=np, seed=0)
  ops["dist_coords"] = coords
  ops["dist_matrix"] = ctx.get_cpu_distances()
  ops["dist_cand5"] = ctx.get_cpu_candidate_list(5)
  ops["dist_cand20"] = ctx.get_cpu_candidate_list(20)
  big = instances.uniform_instance(5000, 78)
  ops["big_coords"] = big
  ops["big_digest"] = np.frombuffer(bytes.fromhex(digest(ProblemContext(coord_problem(big), xp=np, seed=0).get_cpu_distances())), dtype=np.uint8)
  np.savez_compressed(os.path.join(HERE, "ops.npz"), **ops)
  print(f"ops in {time.time() - t0:.1f}s")

  # ------------------------------------------------------------------ GA runs
  class Recorder:
    stage_anchor = "post_survival"

    def __init__(self):
      self.digests: list[str] = []
      self.fitness: list[np.ndarray] = []

    def run(self, state, timer):
      self.digests.append(digest(np.asarray(state.population, dtype=np.int32)))
      self.fitness.append(np.asarray(state.fitness, dtype=np.float64).copy())

  ga_out: dict[str, np.ndarray] = {}

  def run_ga(tag, coords, pop_size, gens, elite, stage="none", post_init=True, periodic=None, ls_iters=10,
             mutation_rate=0.05, patience=10**9, seed=42):
    t = time.time()
    prob = coord_problem(coords)
    ctx = ProblemContext(prob, xp=np, seed=seed)
    ls = LocalSearchCPUTourTwoOpt(mode="best", max_iterations=ls_iters, candidate_k=20)
    ev = EvaluationCPUCost()
    rec = Recorder()
    steps = []
    if post_init:
      steps.append(PostInitLocalSearchStep(local_search=ls, evaluation=ev))
    if periodic is not None:
      steps.append(PeriodicLocalSearchStep(local_search=ls, interval=periodic[0], target=periodic[1],
                                           re_evaluate=ev if periodic[1] == "population" else None))
    if elite:
      steps.append(EliteOnlyLocalSearchStep(local_search=ls, evaluation=ev, elite_count=elite))
    steps.append(rec)
    init = InitializationCPUTourNearestNeighbor(k=5, seed=42)
    captured = {}
    orig_init = init.initialize

    def cap_init(*a, **kw):
      res = orig_init(*a, **kw)
      captured["pop"] = np.asarray(res).copy()
      return res

    init.initialize = cap_init
    ga = GeneticAlgorithm(population_size=pop_size, mutation_rate=mutation_rate, seed=42, initialization=init,
                          selection=SelectionCPUTournament(k=5, seed=42), crossover=CrossoverCPUPermPartiallyMapped(seed=42),
                          mutation=MutationCPUPermInversion(seed=42), local_search=ls, evaluation=ev,
                          local_search_stage=stage, pipeline=steps)
    best, stats = ga.evolve(context=ctx, customers=list(range(len(coords))), max_generations=gens, patience=patience)
    ga_out[f"{tag}_coords"] = coords
    ga_out[f"{tag}_meta"] = np.array([pop_size, gens, elite or 0, int(post_init), ls_iters, seed,
                                      -1 if periodic is None else periodic[0],
                                      -1 if periodic is None else (0 if periodic[1] == "offspring" else 1)])
    ga_out[f"{tag}_stage"] = np.array(stage)
    ga_out[f"{tag}_rate"] = np.array(mutation_rate)
    if captured["pop"].size <= 200_000:
      ga_out[f"{tag}_init"] = captured["pop"]
    ga_out[f"{tag}_init_digest"] = np.array(digest(captured["pop"].astype(np.int32)))
    ga_out[f"{tag}_best"] = np.asarray(best, dtype=np.int32)
    ga_out[f"{tag}_history"] = np.asarray(stats["convergence_history"], dtype=np.float64)
    ga_out[f"{tag}_gens"] = np.array(stats["generations_completed"])
    ga_out[f"{tag}_digests"] = np.array(rec.digests)
    ga_out[f"{tag}_fitness"] = np.stack(rec.fitness) if rec.fitness else np.zeros((0, pop_size))
    ga_out[f"{tag}_rng"] = np.array([ctx.rng.bit_generator.state["state"]["state"] % (1 << 63)], dtype=np.int64)
    print(f"ga {tag}: {time.time() - t:.1f}s best={stats['best_fitness']} gens={stats['generations_completed']}")

  run_ga("c1", instances.uniform_instance(100, 42), 128, 50, 16)
  run_ga("c1default", instances.uniform_instance(100, 42), 128, 50, 16, patience=None)
  run_ga("pm", instances.uniform_instance(52, 5), 32, 5, 0, stage="post_mutation", post_init=False, ls_iters=3)
  run_ga("pc", instances.uniform_instance(52, 6), 33, 5, 0, stage="post_crossover", post_init=False, ls_iters=3)
  run_ga("pe", instances.uniform_instance(52, 7), 32, 5, 4, stage="post_evaluation", post_init=True, ls_iters=3)
  run_ga("px", instances.uniform_instance(52, 8), 32, 6, 0, stage="post_evolution", post_init=False, ls_iters=5)
  run_ga("pp", instances.uniform_instance(60, 9), 32, 6, 0, periodic=(2, "population"), post_init=False)
  run_ga("po", instances.uniform_instance(60, 10), 32, 6, 0, periodic=(3, "offspring"), post_init=False)
  run_ga("c3", instances.uniform_instance(2000, 2000), 512, 3, 64, post_init=False)
  ga_out["tags"] = np.array(["c1", "c1default", "pm", "pc", "pe", "px", "pp", "po", "c3"])
  np.savez_compressed(os.path.join(HERE, "ga.npz"), **ga_out)


def main_ox_swap(ref_root: str) -> None:
  """`ox_swap.npz`: Order Crossover and swap mutation batches of the reference's CPU
  strategies, and two GA runs that use them (tournament + OX + swap + 2-opt elites)."""
  _setup(ref_root)
  from algorithms import GeneticAlgorithm
  from algorithms.pipeline_steps import EliteOnlyLocalSearchStep, PostInitLocalSearchStep
  from algorithms.strategies import (
    CrossoverCPUPermOrder,
    EvaluationCPUCost,
    InitializationCPUTourNearestNeighbor,
    LocalSearchCPUTourTwoOpt,
    MutationCPUPermSwap,
    SelectionCPUTournament,
  )
  from data_models.problem import Problem
  from protocols.problem_context import ProblemContext

  from tsp_gpu_clean_b200 import instances

  def coord_problem(coords):
    return Problem(name="synthetic", dimension=len(coords), problem_type="TSP", edge_type="EUC_2D",
                   coordinates=np.asarray(coords, dtype=np.float64), distances=None)

  out: dict[str, np.ndarray] = {}
  for tag, n, pop_size, rate in (("a", 52, 129, 0.05), ("b", 100, 128, 0.5), ("c", 1000, 64, 1.0),
                                 ("d", 7, 10, 0.0), ("e", 4, 6, 1.0), ("f", 2, 5, 1.0)):
    coords = instances.uniform_instance(n, 5252 + n)
    ctx = ProblemContext(coord_problem(coords), xp=np, seed=321 + n)
    pop = instances.random_tours(n, pop_size, 29 + n)
    ox = CrossoverCPUPermOrder(seed=1).crossover_batch(pop.copy(), ctx)
    sw = MutationCPUPermSwap(seed=1).mutate_batch(np.asarray(ox).copy(), rate, ctx)
    out[f"{tag}_meta"] = np.array([n, pop_size, 321 + n])
    out[f"{tag}_rate"] = np.array(rate)
    out[f"{tag}_pop"] = pop
    out[f"{tag}_ox"] = np.asarray(ox, dtype=np.int32)
    out[f"{tag}_swap"] = np.asarray(sw, dtype=np.int32)
    out[f"{tag}_rng_state"] = np.array([ctx.rng.bit_generator.state["state"]["state"] % (1 << 63)], dtype=np.int64)

  def run_ga(tag, coords, pop_size, gens, elite, mutation_rate, post_init, patience):
    t = time.time()
    ctx = ProblemContext(coord_problem(coords), xp=np, seed=7)
    ls = LocalSearchCPUTourTwoOpt(mode="best", max_iterations=10, candidate_k=20)
    ev = EvaluationCPUCost()
    steps = []
    if post_init:
      steps.append(PostInitLocalSearchStep(local_search=ls, evaluation=ev))
    steps.append(EliteOnlyLocalSearchStep(local_search=ls, evaluation=ev, elite_count=elite))
    ga = GeneticAlgorithm(population_size=pop_size, mutation_rate=mutation_rate, seed=7,
                          initialization=InitializationCPUTourNearestNeighbor(k=5, seed=7),
                          selection=SelectionCPUTournament(k=5, seed=7), crossover=CrossoverCPUPermOrder(seed=7),
                          mutation=MutationCPUPermSwap(seed=7), local_search=ls, evaluation=ev,
                          local_search_stage="none", pipeline=steps)
    best, stats = ga.evolve(context=ctx, customers=list(range(len(coords))), max_generations=gens, patience=patience)
    out[f"ga_{tag}_coords"] = coords
    out[f"ga_{tag}_meta"] = np.array([pop_size, gens, elite, int(post_init), -1 if patience is None else patience])
    out[f"ga_{tag}_rate"] = np.array(mutation_rate)
    out[f"ga_{tag}_best"] = np.asarray(best, dtype=np.int32)
    out[f"ga_{tag}_history"] = np.asarray(stats["convergence_history"], dtype=np.float64)
    out[f"ga_{tag}_gens"] = np.array(stats["generations_completed"])
    out[f"ga_{tag}_rng"] = np.array([ctx.rng.bit_generator.state["state"]["state"] % (1 << 63)], dtype=np.int64)
    print(f"ga {tag}: {time.time() - t:.1f}s best={stats['best_fitness']} gens={stats['generations_completed']}")

  run_ga("ox1", instances.uniform_instance(100, 77), 128, 40, 16, 0.05, True, 10**9)
  run_ga("ox2", instances.clustered_instance(300, 12, 30.0, 78), 64, 30, 8, 0.3, False, None)
  np.savez_compressed(os.path.join(HERE, "ox_swap.npz"), **out)


def main_stage(ref_root: str) -> None:
  """`stage.npz`: the reference's random-permutation initialisation, and GA runs with
  2-opt on every offspring (`local_search_stage="post_mutation"`), the configuration of
  the reference's published Chapter-4 benchmarks (random init, tournament 5, OX, swap,
  2-opt k=20 x10), plus one run mixing the stage with PMX, inversion, NN init and the
  post-init and elite steps."""
  _setup(ref_root)
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

  from tsp_gpu_clean_b200 import instances

  def coord_problem(coords):
    return Problem(name="synthetic", dimension=len(coords), problem_type="TSP", edge_type="EUC_2D",
                   coordinates=np.asarray(coords, dtype=np.float64), distances=None)

  out: dict[str, np.ndarray] = {}
  for tag, n, pop_size in (("r1", 1, 3), ("r2", 2, 4), ("r3", 7, 9), ("r4", 100, 64), ("r5", 1002, 256)):
    coords = instances.uniform_instance(n, 900 + n)
    ctx = ProblemContext(coord_problem(coords), xp=np, seed=41 + n)
    customers = list(range(n)) if tag != "r3" else [3 * c + 5 for c in range(n)]
    pop = InitializationCPUPermRandom(seed=1).initialize(customers, pop_size, ctx)
    out[f"{tag}_meta"] = np.array([n, pop_size, 41 + n])
    out[f"{tag}_customers"] = np.asarray(customers, dtype=np.int32)
    pop = np.ascontiguousarray(pop, dtype=np.int32)
    if pop.size > 50_000:  # large populations are pinned by their digest
      out[f"{tag}_digest"] = np.frombuffer(hashlib.sha256(pop.tobytes()).digest(), dtype=np.uint8)
    else:
      out[f"{tag}_pop"] = pop
    out[f"{tag}_rng_state"] = np.array([ctx.rng.bit_generator.state["state"]["state"] % (1 << 63)], dtype=np.int64)

  def run_ga(tag, coords, pop_size, gens, mutation_rate, patience, chapter4=True, elite=0, post_init=False):
    t = time.time()
    ctx = ProblemContext(coord_problem(coords), xp=np, seed=42)
    ls = LocalSearchCPUTourTwoOpt(mode="best", max_iterations=10, candidate_k=20)
    ev = EvaluationCPUCost()
    steps = []
    if post_init:
      steps.append(PostInitLocalSearchStep(local_search=ls, evaluation=ev))
    if elite:
      steps.append(EliteOnlyLocalSearchStep(local_search=ls, evaluation=ev, elite_count=elite))
    if chapter4:
      init, xo, mut = InitializationCPUPermRandom(seed=42), CrossoverCPUPermOrder(seed=42), MutationCPUPermSwap(seed=42)
    else:
      init = InitializationCPUTourNearestNeighbor(k=5, seed=42)
      xo, mut = CrossoverCPUPermPartiallyMapped(seed=42), MutationCPUPermInversion(seed=42)
    ga = GeneticAlgorithm(population_size=pop_size, mutation_rate=mutation_rate, seed=42, initialization=init,
                          selection=SelectionCPUTournament(k=5, seed=42), crossover=xo, mutation=mut,
                          local_search=ls, evaluation=ev, local_search_stage="post_mutation",
                          pipeline=steps or None)
    best, stats = ga.evolve(context=ctx, customers=list(range(len(coords))), max_generations=gens, patience=patience)
    out[f"ga_{tag}_coords"] = coords
    out[f"ga_{tag}_meta"] = np.array([pop_size, gens, elite, int(post_init), -1 if patience is None else patience,
                                      int(chapter4)])
    out[f"ga_{tag}_rate"] = np.array(mutation_rate)
    out[f"ga_{tag}_best"] = np.asarray(best, dtype=np.int32)
    out[f"ga_{tag}_history"] = np.asarray(stats["convergence_history"], dtype=np.float64)
    out[f"ga_{tag}_gens"] = np.array(stats["generations_completed"])
    out[f"ga_{tag}_rng"] = np.array([ctx.rng.bit_generator.state["state"]["state"] % (1 << 63)], dtype=np.int64)
    print(f"ga {tag}: {time.time() - t:.1f}s best={stats['best_fitness']} gens={stats['generations_completed']}")

  run_ga("s1", instances.uniform_instance(100, 91), 64, 30, 0.02, 10**9)
  run_ga("s2", instances.clustered_instance(200, 8, 30.0, 92), 32, 25, 0.3, None)
  run_ga("s3", instances.uniform_instance(150, 93), 48, 20, 0.1, 10**9, chapter4=False, elite=6, post_init=True)
  np.savez_compressed(os.path.join(HERE, "stage.npz"), **out)


def dist_coords(edge_type: str, n: int, seed: int) -> np.ndarray:
  """Seeded synthetic coordinates for one TSPLIB edge type: planar or 3-D points in
  [0, 1000], ATT-like coordinates in [0, 8000], GEO DDD.MM latitudes and longitudes, and
  XRAY1 motor positions (phi in [0, 360), chi and two-theta in [0, 100])."""
  rng = np.random.default_rng(seed)
  if edge_type == "GEO":
    lat = rng.integers(-89, 90, n) + np.sign(rng.uniform(-1, 1, n)) * np.round(rng.uniform(0, 0.5999, n), 2)
    lon = rng.integers(-179, 180, n) + np.sign(rng.uniform(-1, 1, n)) * np.round(rng.uniform(0, 0.5999, n), 2)
    return np.stack([lat, lon], axis=1)
  if edge_type == "XRAY1":
    return np.stack([rng.uniform(0, 360, n), rng.uniform(0, 100, n), rng.uniform(0, 100, n)], axis=1)
  if edge_type == "ATT":
    return np.round(rng.uniform(0, 8000, (n, 2)))
  dim = 3 if edge_type.endswith("_3D") else 2
  return rng.uniform(0, 1000, (n, dim))


DIST_TYPES = ("EUC_2D", "EUC_3D", "MAN_2D", "MAN_3D", "MAX_2D", "MAX_3D", "CEIL_2D", "ATT", "GEO", "XRAY1")


def main_dist(ref_root: str) -> None:
  """`distances.npz`: the reference's `compute_distance_matrix` and `compute_candidate_list`
  (`src/distances/matrix.py:140-273`) for every coordinate-based TSPLIB edge type, on seeded
  synthetic coordinates: full matrices and 8-NN tables at n = 120, digests of the matrix
  and the 10-NN table at n = 2500 (the chunked path; its coordinates are regenerated by
  `dist_coords`)."""
  _setup(ref_root)
  from distances.matrix import compute_candidate_list, compute_distance_matrix

  out: dict[str, np.ndarray] = {}
  for j, et in enumerate(DIST_TYPES):
    for n, full in ((120, True), (2500, False)):
      c = dist_coords(et, n, 700 + 10 * j + (n > 1000))
      d = compute_distance_matrix(c, et)
      key = f"{et}_{n}"
      if full:
        out[f"{key}_coords"] = c
        out[f"{key}_matrix"] = np.asarray(d, dtype=np.int32)
        out[f"{key}_knn"] = np.asarray(compute_candidate_list(c, et, 8), dtype=np.int32)
      else:
        knn = np.ascontiguousarray(compute_candidate_list(c, et, 10), dtype=np.int32)
        out[f"{key}_digest"] = np.frombuffer(hashlib.sha256(np.ascontiguousarray(d, dtype=np.int32).tobytes())
                                             .digest(), dtype=np.uint8)
        out[f"{key}_knn_digest"] = np.frombuffer(hashlib.sha256(knn.tobytes()).digest(), dtype=np.uint8)
  np.savez_compressed(os.path.join(HERE, "distances.npz"), **out)


def main_three_opt(ref_root: str) -> None:
  """`three_opt.npz`: the reference's exhaustive CPU 3-opt (`cpu_three_opt_best_move`,
  `cpu_three_opt_refine` of its 3-opt experiment,
  `benchmark_scripts/experiments-and-examples/experiment-comparing-3opt-and-2opt/gpu_three_opt.py:133-277`)
  on open tours of uniform and integer-lattice instances (the lattices tie many deltas):
  the steepest move of every input tour and the tours after 1, 3 and unlimited passes."""
  _setup(ref_root)
  import importlib.util

  path = os.path.join(ref_root, "benchmark_scripts", "experiments-and-examples",
                      "experiment-comparing-3opt-and-2opt", "gpu_three_opt.py")
  spec = importlib.util.spec_from_file_location("reference_gpu_three_opt", path)
  mod = importlib.util.module_from_spec(spec)
  spec.loader.exec_module(mod)
  from tsp_gpu_clean_b200 import instances

  out: dict[str, np.ndarray] = {}
  cases = [("u5", instances.uniform_instance(5, 51), 6), ("u6", instances.uniform_instance(6, 52), 6),
           ("u9", instances.uniform_instance(9, 53), 6), ("u16", instances.uniform_instance(16, 54), 5),
           ("u40", instances.uniform_instance(40, 55), 3), ("lat16", None, 5), ("lat36", None, 3)]
  for tag, coords, tours_n in cases:
    t = time.time()
    if coords is None:
      side = int(tag[3:]) ** 0.5
      side = int(round(side))
      coords = np.array([[10.0 * x, 10.0 * y] for x in range(side) for y in range(side)])
    n = len(coords)
    diff = coords[:, None, :] - coords[None, :, :]
    D = (np.sqrt((diff * diff).sum(axis=2)) + 0.5).astype(np.int32)
    np.fill_diagonal(D, 0)
    tours = instances.random_tours(n, tours_n, 900 + n)
    out[f"{tag}_coords"] = coords
    out[f"{tag}_tours"] = tours
    out[f"{tag}_best"] = np.array([mod.cpu_three_opt_best_move(tt, D, is_closed=False) for tt in tours],
                                  dtype=np.int64)
    for iters in (1, 3, 1000):
      out[f"{tag}_refined{iters}"] = np.stack([mod.cpu_three_opt_refine(tt, D, max_iterations=iters, is_closed=False)
                                               for tt in tours]).astype(np.int32)
    print(f"3-opt {tag}: {time.time() - t:.1f}s")
  np.savez_compressed(os.path.join(HERE, "three_opt.npz"), **out)


if __name__ == "__main__":
  if len(sys.argv) < 2:
    sys.exit("usage: make_golden.py <reference checkout root> [all|core|ox|stage|dist|three_opt]")
  root = sys.argv[1]
  part = sys.argv[2] if len(sys.argv) > 2 else "all"
  if part in ("all", "core"):
    main(root)
  if part in ("all", "ox"):
    main_ox_swap(root)
  if part in ("all", "stage"):
    main_stage(root)
  if part in ("all", "dist"):
    main_dist(root)
  if part in ("all", "three_opt"):
    main_three_opt(root)
