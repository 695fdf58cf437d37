"""Benchmark-runner integration: algorithm configs that switch the reference's runner to B200.

The reference's runner builds every algorithm variant from an `algorithms.json` file
(`src/benchmarking/runner/config_loader.py:48-86`, `config_models.py:42-262`): either a
modular `GeneticAlgorithm` whose strategy slots name classes by `{"class"}` (the strategy
registry) or `{"module", "class"}` (a dotted module or a `.py` file relative to the config,
`spec_resolver.py:29-71, 306-339`), or a monolithic class given by `class_module` /
`class_name` and constructed with the GA parameters (`_instantiate_monolithic`). It then
runs seeded repetitions and records per-run statistics (`algorithm_runner.py:445-731`).

This module provides the same pieces for the B200 path:

- `FusedGeneticAlgorithm`: a monolithic algorithm class over the fused graph-replayed
  engine, constructible by the reference's `_instantiate_monolithic` and returning the
  reference's statistics keys (`genetic_algorithm.py:951-964`);
- `load_algorithms_config` / `instantiate`: the same schema and resolution rules, with the
  B200 strategy and pipeline-step registries;
- `run_repetitions`: the repetition loop (seeds `seed_base + r`, one context per
  repetition sharing one candidate cache, warm-up outside the measured runs) with the
  reference's result keys; `batch_repetitions=True` advances all repetitions of a fused
  algorithm together as one batch, each run identical to its sequential counterpart.

`tsp_gpu_clean_b200/configs/algorithms.b200.json` holds the reference's Chapter-4
configuration on the B200 classes, modular and fused.
"""

from __future__ import annotations

import copy
import hashlib
import importlib
import importlib.util
import inspect
import json
import math
import re
import sys
import time
import types
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any, Callable, Mapping

import numpy as np

STRATEGY_SLOTS = ("initialization", "selection", "crossover", "mutation", "evaluation", "local_search")
STATS_KEYS = ("initial_fitness", "initial_feasible_cost", "best_fitness", "best_is_feasible", "generations_completed",
              "stopped_early", "stop_reason", "convergence_history", "phase_timings", "h2d_bytes", "d2h_bytes",
              "kernel_launches")
RESULT_KEYS = ("times", "initial_costs", "final_costs", "gaps", "improvements", "generations", "stop_reasons",
               "phase_timings", "h2d_bytes", "d2h_bytes", "kernel_launches", "best_tours", "seeds")
_FILE_MODULES: dict[tuple[Path, int, int], types.ModuleType] = {}


def adaptive_generations(n: int) -> int:
  """`algorithm_runner.py:44-54`: 2 n sqrt(n) generations."""
  return int(2 * n * math.sqrt(n))


def adaptive_patience(n: int) -> int:
  """`algorithm_runner.py:57-67`: 2 sqrt(n) generations without improvement."""
  return int(2 * math.sqrt(n))


# ------------------------------------------------------------------------ the fused algorithm
class FusedGeneticAlgorithm:
  """The memetic GA on the fused engine, as a monolithic algorithm class of the runner.

  Constructor keywords are those `_instantiate_monolithic` passes (`population_size`,
  `mutation_rate`, `seed`, `local_search_stage`, and `two_opt_iterations` /
  `tournament_size` from strategy overrides) plus the configuration of the run: the
  operators (`crossover` "ox"|"pmx", `mutation` "swap"|"inversion", `initialization`
  "random"|"nn"), the 2-opt (`two_opt_mode` "best"|"batch"|"first", `candidate_k`) and the
  extension steps (`elite_count`, `post_init`). Defaults are the reference's Chapter-4
  configuration. The run's random draws come from `context.rng`, so `seed` is kept only as
  the reference keeps it.
  """

  def __init__(self, population_size: int = 256, mutation_rate: float = 0.02, seed: int | None = 42,
               local_search_stage: str = "post_mutation", tournament_size: int = 5, two_opt_iterations: int = 10,
               two_opt_mode: str = "best", candidate_k: int = 20, crossover: str = "ox", mutation: str = "swap",
               initialization: str = "random", nn_k: int = 5, elite_count: int = 0, post_init: bool = False,
               use_graph: bool = True, chunk: int = 16) -> None:
    if local_search_stage not in ("none", "post_mutation"):
      raise ValueError("FusedGeneticAlgorithm runs local_search_stage 'post_mutation' or 'none'")
    if two_opt_mode not in ("best", "batch", "first"):
      raise ValueError(f"Invalid two_opt_mode '{two_opt_mode}'")
    if crossover not in ("ox", "pmx") or mutation not in ("swap", "inversion") or initialization not in ("random", "nn"):
      raise ValueError("crossover 'ox'|'pmx', mutation 'swap'|'inversion', initialization 'random'|'nn'")
    self.population_size = int(population_size)
    self.mutation_rate = float(mutation_rate)
    self.seed = seed
    self.local_search_stage = local_search_stage
    self.tournament_size = int(tournament_size)
    self.two_opt_iterations = int(two_opt_iterations)
    self.two_opt_mode = two_opt_mode
    self.candidate_k = int(candidate_k)
    self.crossover = crossover
    self.mutation = mutation
    self.initialization = initialization
    self.nn_k = int(nn_k)
    self.elite_count = int(elite_count)
    self.post_init = bool(post_init)
    self.use_graph = bool(use_graph)
    self.chunk = int(chunk)
    self.kernel_launches = 0

  def _solver(self):
    from .batch import FusedBatchSolver
    from .fused import LocalSearchConfig

    return FusedBatchSolver(population_size=self.population_size, mutation_rate=self.mutation_rate,
                            tournament_k=self.tournament_size, nn_k=self.nn_k,
                            local_search=LocalSearchConfig(self.two_opt_mode, self.two_opt_iterations, self.candidate_k),
                            elite_count=self.elite_count, post_init=self.post_init, max_matrix_dimension=None,
                            use_graph=self.use_graph, chunk=self.chunk, crossover=self.crossover,
                            mutation=self.mutation, init=self.initialization,
                            local_search_stage=self.local_search_stage)

  def warmup(self, context: Any) -> None:
    """Build the library and run every launch path once on `context` (the runner's
    throw-away warm-up context), so no compilation lands in a measured run."""
    from .build import build_library

    build_library()
    self.evolve(context, list(range(int(context.dimension))), 1)

  def evolve(self, context: Any, customers: Any, max_generations: int, optimal_cost: float | None = None,
             patience: int | None = None) -> tuple[np.ndarray, dict]:
    """One run, `GeneticAlgorithm.evolve`'s contract (`genetic_algorithm.py:789-965`)."""
    (best, stats), = self.evolve_repetitions([context], customers, max_generations, optimal_cost, patience)
    return best, stats

  def evolve_repetitions(self, contexts: list, customers: Any, max_generations: int,
                         optimal_cost: float | None = None, patience: int | None = None) -> list:
    """Runs on several contexts of one problem advanced together; each result equals the
    run `evolve` gives on that context alone."""
    n = int(contexts[0].dimension)
    if list(customers) != list(range(n)):
      raise ValueError("FusedGeneticAlgorithm evolves full tours: customers must be range(dimension)")
    solver = self._solver()
    results = solver.evolve(contexts, int(max_generations), patience=patience, optimal_cost=optimal_cost)
    t = solver.last_timing
    runs = len(contexts)
    self.kernel_launches = solver.kernel_launches
    self.last_timing = t

    def phase(key: str) -> dict:
      ms = 1e3 * float(t.get(key, 0.0)) / runs
      return {"total_ms": ms, "calls": 1, "mean_ms": ms}

    timings = {"setup": phase("setup_s"), "tuning": phase("tune_s"), "post_init_and_capture": phase("postinit_capture_s"),
               "generations": phase("loop_s"), "results": phase("results_s")}
    k_eff = min(self.candidate_k, n - 1)
    h2d = n * 16 + n * k_eff * 4 + self.population_size * 8  # coordinates, k-NN table, row seeds
    out = []
    for best, st in results:
      d2h = n * 4 + 8 * len(st["convergence_history"])  # best tour and history
      stats = {
        "initial_fitness": st["initial_fitness"],
        "initial_feasible_cost": st["initial_fitness"],
        "best_fitness": st["best_fitness"],
        "best_is_feasible": True,
        "generations_completed": st["generations_completed"],
        "stopped_early": st["stopped_early"],
        "stop_reason": st["stop_reason"],
        "convergence_history": st["convergence_history"],
        "phase_timings": timings,
        "h2d_bytes": h2d,
        "d2h_bytes": d2h,
        "kernel_launches": solver.kernel_launches // runs,
      }
      out.append((best, stats))
    return out


# ------------------------------------------------------------------------ config loading
@dataclass
class GAParams:
  population_size: int = 256
  mutation_rate: float = 0.02
  seed: int = 42


@dataclass
class AlgorithmConfig:
  name: str
  use_gpu: bool = True
  description: str = ""
  metaheuristic: str = "GeneticAlgorithm"
  class_module: str | None = None
  class_name: str | None = None
  params: dict = field(default_factory=dict)
  strategies: dict = field(default_factory=dict)
  source_dir: Path | None = None


def load_algorithms_config(path: str | Path) -> tuple[GAParams, dict[str, AlgorithmConfig]]:
  """`default_params` (or `ga_params`) and `algorithm_configs` of an algorithms file
  (`config_loader.py:48-86`); module paths resolve relative to the file's folder."""
  p = Path(path)
  if p.is_dir():
    p = p / "algorithms.json"
  data = json.loads(p.read_text())
  d = data.get("default_params") or data.get("ga_params", {})
  params = GAParams(int(d.get("population_size", 256)), float(d.get("mutation_rate", 0.02)), int(d.get("seed", 42)))
  if "algorithm_configs" not in data:
    raise ValueError(f"{p}: missing 'algorithm_configs' section")
  src = p.parent.resolve()
  algos = {
    name: AlgorithmConfig(name=name, use_gpu=bool(c.get("use_gpu", False)), description=c.get("description", ""),
                          metaheuristic=c.get("metaheuristic", "GeneticAlgorithm"), class_module=c.get("class_module"),
                          class_name=c.get("class_name"), params=dict(c.get("params") or {}),
                          strategies=dict(c.get("strategies") or {}), source_dir=src)
    for name, c in data["algorithm_configs"].items()
  }
  return params, algos


def load_module(ref: str, base_dir: Path | None = None) -> types.ModuleType:
  """A dotted module name, or a `.py` file (absolute or relative to `base_dir`) loaded once
  per (path, mtime, size) under a name derived from its path (`spec_resolver.py:29-71`)."""
  if not (ref.endswith(".py") or "/" in ref or "\\" in ref):
    return importlib.import_module(ref)
  cand = Path(ref)
  path = cand.resolve() if cand.is_absolute() or base_dir is None else (base_dir / cand).resolve()
  if not path.is_file():
    raise FileNotFoundError(f"module file not found: '{ref}' (resolved to '{path}')")
  st = path.stat()
  key = (path, st.st_mtime_ns, st.st_size)
  if key in _FILE_MODULES:
    return _FILE_MODULES[key]
  # a file inside this package is the package's own module (its relative imports need it)
  pkg_root = Path(__file__).resolve().parent
  if pkg_root in path.parents or path.parent == pkg_root:
    rel = path.relative_to(pkg_root.parent).with_suffix("")
    mod = importlib.import_module(".".join(rel.parts))
  else:
    slug = re.sub(r"\W+", "_", path.stem).strip("_") or "module"
    name = f"_tspb_external_{slug}_{hashlib.sha256(str(path).encode()).hexdigest()[:12]}"
    spec = importlib.util.spec_from_file_location(name, path)
    if spec is None or spec.loader is None:
      raise ImportError(f"cannot load '{path}'")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    try:
      spec.loader.exec_module(mod)
    except Exception:
      sys.modules.pop(name, None)
      raise
  _FILE_MODULES[key] = mod
  return mod


def resolve_class(spec: Mapping[str, Any], registry: Mapping[str, type], base_dir: Path | None) -> type:
  name = spec.get("class")
  if not isinstance(name, str) or not name:
    raise ValueError(f"missing or invalid 'class' in {dict(spec)!r}")
  if spec.get("module"):
    cls = getattr(load_module(spec["module"], base_dir), name, None)
    if not isinstance(cls, type):
      raise ValueError(f"'{name}' is not a class in module '{spec['module']}'")
    return cls
  if name not in registry:
    raise ValueError(f"unknown class '{name}'; registered: {sorted(registry)}")
  return registry[name]


def build_component(spec: Mapping[str, Any] | None, registry: Mapping[str, type], *, seed: Any,
                    base_dir: Path | None, defaults: Mapping[str, Any] | None = None,
                    overrides: Mapping[str, Any] | None = None) -> Any:
  """Instantiate one strategy or pipeline step (`spec_resolver.py:306-339`): its `params`,
  then overrides, then defaults for accepted keywords not given, and `seed` when the class
  takes one; unknown keywords are rejected unless the class takes **kwargs."""
  if not spec or ("class" not in spec and "module" not in spec):
    return None
  cls = resolve_class(spec, registry, base_dir)
  sig = inspect.signature(cls)
  var_kw = any(p.kind == inspect.Parameter.VAR_KEYWORD for p in sig.parameters.values())
  params = dict(spec.get("params") or {})
  for k, v in (overrides or {}).items():
    if not var_kw and k not in sig.parameters:
      raise ValueError(f"class '{cls.__name__}' does not accept parameter '{k}'")
    params[k] = v
  for k, v in (defaults or {}).items():
    if k in sig.parameters and k not in params and v is not None:
      params[k] = v
  if "seed" in sig.parameters and "seed" not in params:
    params["seed"] = seed
  if not var_kw:
    bad = [k for k in params if k not in sig.parameters]
    if bad:
      raise ValueError(f"class '{cls.__name__}' does not accept parameters {bad}")
  return cls(**params)


def instantiate(cfg: AlgorithmConfig, defaults: GAParams, seed: int | None = None,
                strategy_overrides: Mapping[str, Mapping[str, Any]] | None = None) -> Any:
  """The algorithm of one config entry (`config_models.py:98-262`): monolithic when
  `class_module`/`class_name` are given, else a modular `ga.GeneticAlgorithm` whose slots
  come from the B200 strategy registry or `{"module", "class"}` specs."""
  from .pipeline_steps import PIPELINE_STEP_REGISTRY
  from .strategies import STRATEGY_REGISTRY

  for slot in list(cfg.strategies) + list(strategy_overrides or {}):
    if slot not in STRATEGY_SLOTS:
      raise ValueError(f"unknown strategy slot '{slot}' in '{cfg.name}'; valid: {list(STRATEGY_SLOTS)}")
  if cfg.class_module and cfg.class_name:
    cls = getattr(load_module(cfg.class_module, cfg.source_dir), cfg.class_name)
    kw: dict[str, Any] = {"population_size": defaults.population_size, "mutation_rate": defaults.mutation_rate,
                          "seed": seed if seed is not None else defaults.seed}
    kw.update(cfg.params)
    if seed is not None:
      kw["seed"] = seed
    so = strategy_overrides or {}
    if "max_iterations" in so.get("local_search", {}):
      kw["two_opt_iterations"] = so["local_search"]["max_iterations"]
    if "k" in so.get("selection", {}):
      kw["tournament_size"] = so["selection"]["k"]
    sig = inspect.signature(cls)
    if not any(p.kind == inspect.Parameter.VAR_KEYWORD for p in sig.parameters.values()):
      kw = {k: v for k, v in kw.items() if k in sig.parameters}
    return cls(**kw)

  from .ga import GeneticAlgorithm

  resolved_seed = seed if seed is not None else cfg.params.get("seed", defaults.seed)
  slots = {s: build_component(cfg.strategies.get(s), STRATEGY_REGISTRY, seed=resolved_seed, base_dir=cfg.source_dir,
                              overrides=(strategy_overrides or {}).get(s)) for s in STRATEGY_SLOTS}
  pipeline = None
  if cfg.params.get("pipeline") is not None:
    step_defaults = {"local_search": slots["local_search"], "evaluation": slots["evaluation"],
                     "re_evaluate": slots["evaluation"]}
    pipeline = [build_component(s, PIPELINE_STEP_REGISTRY, seed=resolved_seed, base_dir=cfg.source_dir,
                                defaults=step_defaults) for s in cfg.params["pipeline"]]
    pipeline = [p for p in pipeline if p is not None]
  return GeneticAlgorithm(population_size=int(cfg.params.get("population_size", defaults.population_size)),
                          mutation_rate=float(cfg.params.get("mutation_rate", defaults.mutation_rate)),
                          seed=resolved_seed, initialization=slots["initialization"], selection=slots["selection"],
                          crossover=slots["crossover"], mutation=slots["mutation"], evaluation=slots["evaluation"],
                          local_search=slots["local_search"],
                          local_search_stage=cfg.params.get("local_search_stage", "post_mutation"), pipeline=pipeline)


# ------------------------------------------------------------------------ repetitions
def run_repetitions(algorithm: Any, problem: Any, max_generations: int, repetitions: int, *,
                    seed_base: int = 42, optimal_cost: float | None = None, patience: int | None = None,
                    algorithm_factory: Callable[[int], Any] | None = None, batch_repetitions: bool = False,
                    warmup: bool = True) -> dict:
  """The repetition loop of `run_single_algorithm` (`algorithm_runner.py:445-731`) for a TSP
  problem: repetition r runs on `ProblemContext(problem, seed=seed_base + r)` (one candidate
  cache for all), after a warm-up on a separate context; returns the reference's per-run
  lists plus summary statistics. With `batch_repetitions` (an algorithm that has
  `evolve_repetitions`), all repetitions run together and each is given an equal share of
  the wall time."""
  from .problem import ProblemContext

  n = int(problem.dimension)
  customers = list(range(n))
  if patience is None:
    patience = adaptive_patience(n)
  cache: dict[int, np.ndarray] = {}
  if warmup and hasattr(algorithm, "warmup"):
    w = algorithm_factory(seed_base) if algorithm_factory else copy.deepcopy(algorithm)
    w.warmup(ProblemContext(problem, seed=seed_base, candidate_cache=cache))
  seeds = [seed_base + r for r in range(repetitions)]
  res: dict[str, list] = {k: [] for k in RESULT_KEYS}
  runs: list[tuple[Any, dict, float]] = []
  if batch_repetitions:
    if not hasattr(algorithm, "evolve_repetitions"):
      raise ValueError("batch_repetitions needs an algorithm with evolve_repetitions")
    ctxs = [ProblemContext(problem, seed=s, candidate_cache=cache) for s in seeds]
    t0 = time.perf_counter()
    out = algorithm.evolve_repetitions(ctxs, customers, max_generations, optimal_cost, patience)
    share = (time.perf_counter() - t0) / max(1, repetitions)
    runs = [(b, st, share) for b, st in out]
  else:
    for s in seeds:
      algo = algorithm_factory(s) if algorithm_factory else algorithm
      ctx = ProblemContext(problem, seed=s, candidate_cache=cache)
      t0 = time.perf_counter()
      best, st = algo.evolve(ctx, customers, max_generations, optimal_cost=optimal_cost, patience=patience)
      runs.append((best, st, time.perf_counter() - t0))
  for s, (best, st, elapsed) in zip(seeds, runs):
    init, final = float(st["initial_fitness"]), float(st["best_fitness"])
    res["seeds"].append(s)
    res["times"].append(elapsed)
    res["initial_costs"].append(init)
    res["final_costs"].append(final)
    res["gaps"].append((final - optimal_cost) / optimal_cost * 100.0 if optimal_cost and optimal_cost > 0 else np.nan)
    res["improvements"].append((init - final) / init * 100.0 if math.isfinite(init) and init > 0 else np.nan)
    res["generations"].append(st.get("generations_completed", 0))
    res["stop_reasons"].append(st.get("stop_reason", "completed"))
    res["phase_timings"].append(st.get("phase_timings", {}))
    res["h2d_bytes"].append(st.get("h2d_bytes", 0))
    res["d2h_bytes"].append(st.get("d2h_bytes", 0))
    res["kernel_launches"].append(st.get("kernel_launches", 0))
    res["best_tours"].append(np.asarray(best).tolist())
  costs = np.asarray(res["final_costs"], dtype=np.float64)
  times = np.asarray(res["times"], dtype=np.float64)
  gaps = np.asarray(res["gaps"], dtype=np.float64)
  res["summary"] = {
    "successful_runs": len(costs),
    "mean_cost": float(costs.mean()) if costs.size else None,
    "std_cost": float(costs.std(ddof=1)) if costs.size > 1 else 0.0,
    "best_cost": float(costs.min()) if costs.size else None,
    "mean_gap": float(np.nanmean(gaps)) if np.isfinite(gaps).any() else None,
    "mean_time": float(times.mean()) if times.size else None,
    "std_time": float(times.std(ddof=1)) if times.size > 1 else 0.0,
    "mean_generations": float(np.mean(res["generations"])) if res["generations"] else None,
  }
  return res
