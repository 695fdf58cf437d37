"""Runner integration on the B200: the config's modular and fused variants run seeded
repetitions like the reference's runner and agree with each other and with the reference's
recorded run; the optimal-cost and patience stops give the reference's stop reasons."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONFIG = Path(__file__).resolve().parents[1] / "tsp_gpu_clean_b200" / "configs" / "algorithms.b200.json"


@pytest.fixture(scope="module")
def algos():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  from tsp_gpu_clean_b200 import runner

  return runner.load_algorithms_config(CONFIG)


def _problem(g):
  from tsp_gpu_clean_b200.problem import Problem

  return Problem.from_coordinates(np.asarray(g["ga_s1_coords"], dtype=np.float64))


def _make(algos, name, **params):
  from tsp_gpu_clean_b200 import runner

  defaults, cfgs = algos
  cfg = cfgs[name]
  cfg = runner.AlgorithmConfig(**{**cfg.__dict__, "params": {**cfg.params, **params}})
  return runner.instantiate(cfg, defaults)


def _same_runs(a, b):
  assert a["final_costs"] == b["final_costs"]
  assert a["generations"] == b["generations"]
  assert a["stop_reasons"] == b["stop_reasons"]
  assert a["best_tours"] == b["best_tours"]
  assert a["initial_costs"] == b["initial_costs"]


def test_modular_and_fused_repetitions_match_reference(algos, golden):
  """Chapter-4 configuration at population 64 on the recorded 100-city instance: the first
  repetition (seed 42) is the reference's recorded run; both variants agree on every run."""
  from tsp_gpu_clean_b200 import runner

  g = golden("stage.npz")
  problem = _problem(g)
  res = {}
  for name in ("B200Modular", "B200Fused"):
    algo = _make(algos, name, population_size=64)
    res[name] = runner.run_repetitions(algo, problem, 30, 3, seed_base=42, patience=10**9)
    r = res[name]
    assert r["seeds"] == [42, 43, 44]
    assert r["best_tours"][0] == g["ga_s1_best"].tolist()
    assert r["final_costs"][0] == float(g["ga_s1_history"][-1])
  _same_runs(res["B200Modular"], res["B200Fused"])
  fused = _make(algos, "B200Fused", population_size=64)
  batched = runner.run_repetitions(fused, problem, 30, 3, seed_base=42, patience=10**9, batch_repetitions=True)
  _same_runs(batched, res["B200Fused"])


def test_fused_stats_carry_the_reference_keys(algos, golden):
  from tsp_gpu_clean_b200 import runner
  from tsp_gpu_clean_b200.problem import ProblemContext

  g = golden("stage.npz")
  algo = _make(algos, "B200Fused", population_size=32)
  best, stats = algo.evolve(ProblemContext(_problem(g), seed=5), list(range(100)), 5)
  assert set(stats) == set(runner.STATS_KEYS)
  assert sorted(best.tolist()) == list(range(100))
  assert stats["generations_completed"] == len(stats["convergence_history"]) - 1


@pytest.mark.parametrize("kind", ["hit", "near", "patience_at_last"])
def test_early_stops_match_the_strategy_pipeline(algos, golden, kind):
  """hit_optimal, within_1pct_optimal, and patience running out exactly at the last
  generation (stopped early by the reference's rule) give the same generation count, stop
  reason and history on the fused engine as on the strategy pipeline."""
  from tsp_gpu_clean_b200.problem import ProblemContext

  g = golden("stage.npz")
  hist = np.asarray(g["ga_s1_history"])
  G, optimal, patience = 30, None, 10**9
  if kind == "hit":  # a generation whose improvement jumps from above 1 % straight onto the target
    jump = next(t for t in range(2, len(hist)) if (hist[t - 1] - hist[t]) / hist[t] * 100.0 >= 1.0)
    optimal = float(hist[jump])
  elif kind == "near":
    optimal = float(hist[9]) / 1.009
  else:
    last = int(np.nonzero(np.diff(hist) != 0)[0].max()) + 1  # generation of the last improvement
    G, patience = 30, 30 - last
  out = []
  for name in ("B200Modular", "B200Fused"):
    algo = _make(algos, name, population_size=64)
    ctx = ProblemContext(_problem(g), seed=42)
    best, stats = algo.evolve(ctx, list(range(100)), G, optimal_cost=optimal, patience=patience)
    out.append((np.asarray(best).tolist(), stats["generations_completed"], stats["stopped_early"],
                stats["stop_reason"], list(stats["convergence_history"]),
                ctx.rng.bit_generator.state["state"]["state"]))
  assert out[0] == out[1]
  reason = {"hit": "hit_optimal", "near": "within_1pct_optimal", "patience_at_last": "no_improvements"}[kind]
  assert out[1][2] is True and out[1][3] == reason
  if kind == "patience_at_last":
    assert out[1][1] == G
  else:  # the first generation at which the recorded history meets the reference's rule
    stop = next(t for t in range(1, len(hist)) if hist[t] <= optimal + 1e-6
                or (hist[t] - optimal) / optimal * 100.0 < 1.0)
    assert out[1][1] == stop and out[1][4] == hist[: stop + 1].tolist()


def test_or_opt_variant_runs_through_the_runner(algos, golden):
  """B200ModularOrOpt: the modular pipeline with Or-opt as its local search runs seeded
  repetitions end to end; every best tour is a permutation and histories never rise."""
  from tsp_gpu_clean_b200 import runner

  g = golden("stage.npz")
  problem = _problem(g)
  algo = _make(algos, "B200ModularOrOpt", population_size=32)
  r = runner.run_repetitions(algo, problem, 8, 2, seed_base=42, patience=10**9)
  n = len(g["ga_s1_coords"])
  for tour, final, initial in zip(r["best_tours"], r["final_costs"], r["initial_costs"]):
    assert sorted(tour) == list(range(n))
    assert final <= initial
  assert r["generations"] == [8, 8]
