"""Runner integration on the host: the B200 algorithms config resolves through this package's
loader and through the reference's own `AlgorithmConfig.instantiate`."""

from __future__ import annotations

import inspect
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
CONFIG = REPO / "tsp_gpu_clean_b200" / "configs" / "algorithms.b200.json"
sys.path.insert(0, str(Path(__file__).resolve().parent))
from reference_env import import_root  # noqa: E402

REFERENCE_SRC = import_root()  # a checkout's src/ (TSPB_REFERENCE) or the install under baseline/_ref


def test_config_instantiates_every_variant():
  from tsp_gpu_clean_b200 import runner
  from tsp_gpu_clean_b200.ga import GeneticAlgorithm
  from tsp_gpu_clean_b200.strategies import CrossoverB200PermOrder, InitializationB200PermRandom

  defaults, algos = runner.load_algorithms_config(CONFIG)
  assert (defaults.population_size, defaults.mutation_rate, defaults.seed) == (256, 0.02, 42)
  modular = runner.instantiate(algos["B200Modular"], defaults, seed=7)
  assert isinstance(modular, GeneticAlgorithm) and modular.local_search_stage == "post_mutation"
  assert isinstance(modular.crossover, CrossoverB200PermOrder)
  assert isinstance(modular.initialization, InitializationB200PermRandom) and modular.initialization.return_gpu
  assert modular.local_search.mode == "batch" and modular.local_search.candidate_k == 20
  fused = runner.instantiate(algos["B200Fused"], defaults, seed=7, strategy_overrides={"local_search":
                                                                                      {"max_iterations": 3}})
  assert isinstance(fused, runner.FusedGeneticAlgorithm)
  assert (fused.population_size, fused.mutation_rate, fused.seed, fused.two_opt_iterations) == (256, 0.02, 7, 3)
  assert (fused.crossover, fused.mutation, fused.initialization) == ("ox", "swap", "random")
  or_opt = runner.instantiate(algos["B200ModularOrOpt"], defaults)
  from tsp_gpu_clean_b200.strategies import LocalSearchB200OrOpt

  assert isinstance(or_opt.local_search, LocalSearchB200OrOpt) and or_opt.local_search.max_segment == 3
  memetic = runner.instantiate(algos["B200MemeticFused"], defaults)
  assert (memetic.population_size, memetic.elite_count, memetic.post_init, memetic.crossover) == (128, 16, True, "pmx")


def test_invalid_specs_are_rejected(tmp_path):
  from tsp_gpu_clean_b200 import runner

  defaults = runner.GAParams()
  bad_slot = runner.AlgorithmConfig(name="x", strategies={"decoder": {"class": "EvaluationB200Cost"}})
  with pytest.raises(ValueError):
    runner.instantiate(bad_slot, defaults)
  unknown = runner.AlgorithmConfig(name="x", strategies={"crossover": {"class": "NoSuchCrossover"}})
  with pytest.raises(ValueError):
    runner.instantiate(unknown, defaults)
  bad_param = runner.AlgorithmConfig(name="x", strategies={"crossover": {"class": "CrossoverB200PermOrder",
                                                                         "params": {"k": 3}}})
  with pytest.raises(ValueError):
    runner.instantiate(bad_param, defaults)
  with pytest.raises(FileNotFoundError):
    runner.load_module("missing_file.py", tmp_path)
  with pytest.raises(ValueError):
    runner.FusedGeneticAlgorithm(local_search_stage="post_crossover")


def test_fused_algorithm_takes_the_monolithic_keywords():
  """`_instantiate_monolithic` passes population_size, mutation_rate, seed and
  local_search_stage, plus two_opt_iterations / tournament_size from strategy overrides."""
  from tsp_gpu_clean_b200.runner import FusedGeneticAlgorithm

  params = inspect.signature(FusedGeneticAlgorithm).parameters
  for k in ("population_size", "mutation_rate", "seed", "local_search_stage", "two_opt_iterations",
            "tournament_size"):
    assert k in params
  evolve = inspect.signature(FusedGeneticAlgorithm.evolve).parameters
  assert list(evolve)[:4] == ["self", "context", "customers", "max_generations"]
  assert "optimal_cost" in evolve and "patience" in evolve


@pytest.mark.skipif(REFERENCE_SRC is None, reason="reference not present (set TSPB_REFERENCE)")
def test_reference_config_models_instantiate_the_b200_config():
  """The reference's `AlgorithmConfig.instantiate` builds its own GeneticAlgorithm wired with
  the B200 strategies (file-path specs through `plugin.py`, protocol contracts checked) and
  the fused algorithm through its monolithic path. Runs in a child process: the reference's
  packages go on its path, with stand-ins for the runner's storage and loader dependencies
  that configuration never calls."""
  script = textwrap.dedent(f"""
    import json, sys, types
    from pathlib import Path
    sys.path.insert(0, {str(REPO / "tests" / "golden")!r})
    import make_golden
    make_golden.setup_import_root({REFERENCE_SRC!r})
    for pkg, sub in (("benchmarking", "benchmarking"), ("benchmarking.runner", "benchmarking/runner")):
      m = types.ModuleType(pkg)
      m.__path__ = [str(Path({REFERENCE_SRC!r}) / sub)]
      sys.modules[pkg] = m
    from benchmarking.runner.config_models import AlgorithmConfig, GAParams
    path = Path({str(CONFIG)!r})
    data = json.loads(path.read_text())
    d = data["default_params"]
    dp = GAParams(population_size=int(d["population_size"]), mutation_rate=float(d["mutation_rate"]),
                  seed=int(d["seed"]))
    for name, c in data["algorithm_configs"].items():
      cfg = AlgorithmConfig(name=name, metaheuristic=c.get("metaheuristic", "GeneticAlgorithm"),
                            class_module=c.get("class_module"), class_name=c.get("class_name"),
                            use_gpu=bool(c.get("use_gpu")), description=c.get("description", ""),
                            params=c.get("params", {{}}), strategies=c.get("strategies", {{}}),
                            source_dir=path.parent.resolve())
      a = cfg.instantiate(dp, seed=43)
      slots = [type(getattr(a, s, None)).__name__ for s in ("initialization", "selection", "crossover",
                                                             "mutation", "local_search", "evaluation")]
      print(name, type(a).__name__, a.population_size, *slots)
  """)
  out = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=300, cwd=str(REPO))
  assert out.returncode == 0, out.stderr[-2000:]
  lines = {ln.split()[0]: ln.split()[1:] for ln in out.stdout.strip().splitlines()}
  assert lines["B200Modular"] == ["GeneticAlgorithm", "256", "InitializationB200PermRandom", "SelectionB200Tournament",
                                  "CrossoverB200PermOrder", "MutationB200PermSwap", "LocalSearchB200TourTwoOpt",
                                  "EvaluationB200Cost"]
  assert lines["B200ModularOrOpt"][6] == "LocalSearchB200OrOpt"
  assert lines["B200Fused"][:2] == ["FusedGeneticAlgorithm", "256"]
  assert lines["B200MemeticFused"][:2] == ["FusedGeneticAlgorithm", "128"]
