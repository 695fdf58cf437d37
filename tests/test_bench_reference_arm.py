"""bench.py's reference arm on the CPU: one JSON line with impl "reference", the CPU
baseline it timed and a zero-copy e2e; ranks other than 0 print nothing and exit 0."""

from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, env_extra=None):
  env = dict(os.environ)
  env.pop("RANK", None)
  env.pop("WORLD_SIZE", None)
  env.update(env_extra or {})
  p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                     capture_output=True, text=True, env=env, cwd=ROOT, timeout=240)
  assert p.returncode == 0, p.stderr[-2000:]
  return [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]


@pytest.mark.timeout(300)
@pytest.mark.parametrize("args", [["--workload", "ga100", "--cpu-gens", "3"], ["--workload", "or_opt"]])
def test_reference_arm_prints_one_contract_line(args):
  lines = _run([*args, "--steps", "1", "--warmup", "3"])
  assert len(lines) == 1
  d = lines[0]
  assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
  sys.path.insert(0, ROOT)
  from baseline import reference_arm

  # the reference's own CPU code when it is installed; Or-opt has no reference counterpart
  want = "port" if args[1] == "or_opt" or reference_arm.import_root() is None else "reference"
  assert d["cpu_baseline"]["kind"] == want and d["cpu_baseline"]["cores"] >= 1
  assert d["cpu_baseline"]["value"] == d["value"] and d["e2e"]["value"] == d["value"]
  assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
  assert d["unit"] == d["e2e"]["unit"] and d["config"]["workload"]


@pytest.mark.timeout(120)
def test_reference_arm_other_ranks_exit_quietly():
  assert _run(["--workload", "ga100", "--cpu-gens", "3", "--steps", "1", "--warmup", "3"],
              {"RANK": "1", "WORLD_SIZE": "2"}) == []


def test_parity_check_flags_a_planted_difference():
  """bench.check_parity against the oracle's refinements: equal results pass; one move
  planted into the oracle's copy of a tour, or a changed pair count, fails the run."""
  import numpy as np

  sys.path.insert(0, ROOT)
  import bench

  rng = np.random.default_rng(3)
  tours = np.stack([rng.permutation(12) for _ in range(5)]).astype(np.int32)
  stats = np.arange(5 * 4, dtype=np.int64).reshape(5, 4)
  gpu = {m: (tours.copy(), stats.copy()) for m in bench.MODES}
  idx = bench.parity_indices(5, 3)
  assert idx == [0, 2, 4]

  def cpu(plant=None):
    results = []
    for i in idx:
      out = {}
      for m in bench.MODES:
        t = tours[i].copy()
        st = tuple(int(v) for v in stats[i][:3])
        if plant == ("tour", i, m):
          t[[1, 2]] = t[[2, 1]]
        if plant == ("pairs", i, m):
          st = (st[0], st[1] + 1, st[2])
        out[m] = (t, st)
      results.append(out)
    return {"indices": idx, "results": results}

  ok = bench.check_parity(gpu, cpu())
  assert ok["ok"] and ok["text"].startswith("bit-exact against the oracle port on 3/5 tours")
  bad = bench.check_parity(gpu, cpu(("tour", 2, "first")))
  assert not bad["ok"] and "first tour 2" in bad["mismatches"][0]
  bad = bench.check_parity(gpu, cpu(("pairs", 4, "best")))
  assert not bad["ok"] and "best tour 4" in bad["mismatches"][0]


def test_parity_check_against_the_reference_compares_passes_and_pairs():
  """The reference's worker reports (passes, pairs) per mode; the check compares those
  two counters and the tours, and names the reference."""
  import numpy as np

  sys.path.insert(0, ROOT)
  import bench

  rng = np.random.default_rng(4)
  tours = np.stack([rng.permutation(10) for _ in range(4)]).astype(np.int32)
  stats = np.arange(4 * 4, dtype=np.int64).reshape(4, 4)
  gpu = {m: (tours.copy(), stats.copy()) for m in bench.MODES}
  idx = [0, 3]
  results = [{m: (tours[i].copy(), (int(stats[i][0]), int(stats[i][1]))) for m in bench.MODES} for i in idx]
  ok = bench.check_parity(gpu, {"indices": idx, "results": results}, "reference")
  assert ok["ok"] and "the reference's CPU 2-opt" in ok["text"]
  results[1]["best"] = (tours[3].copy(), (int(stats[3][0]), int(stats[3][1]) + 1))
  assert not bench.check_parity(gpu, {"indices": idx, "results": results}, "reference")["ok"]
  # both arms hash the same refinements to the same digest
  dev = [{m: (tours[i],) for m in bench.MODES} for i in idx]
  assert bench.refined_digest(dev) == bench.refined_digest([{m: (tours[i], (0, 0)) for m in bench.MODES} for i in idx])


@pytest.mark.timeout(300)
def test_reference_worker_equals_the_oracle_port():
  """The installed reference's CPU 2-opt and the oracle port refine the same tour to the
  same local optimum with the same pass and pair counts (both modes, k = 20)."""
  import numpy as np

  sys.path.insert(0, ROOT)
  from baseline import reference_arm

  if reference_arm.import_root() is None:
    pytest.skip("the reference is not installed")
  from oracle import distances, two_opt
  from tsp_gpu_clean_b200 import instances

  coords = instances.clustered_instance(300, 8, 30.0, 77)
  tour = instances.random_tours(300, 1, 78)[0]
  out, secs = reference_arm.two_opt_worker((coords, tour, ("best", "first"), 20))
  D = distances.euc2d_matrix(coords)
  cand = distances.candidate_list(20, coords=coords)
  for mode in ("best", "first"):
    t, st = two_opt.improve_batch(tour[None, :], D, cand, mode, 10**9)
    assert np.array_equal(out[mode][0], t[0]), mode
    assert out[mode][1] == (int(st[0][0]), int(st[0][1])), mode
  assert secs > 0


@pytest.mark.timeout(300)
def test_reference_ga_timing_runs_the_same_ga_as_the_oracle():
  """The GA the CPU baseline times (the installed reference's GeneticAlgorithm.evolve with
  its CPU strategies) and the oracle GA give the same best-fitness history on the 100-city
  workload and on the Chapter-4 configuration."""
  sys.path.insert(0, ROOT)
  from baseline import reference_arm

  if reference_arm.import_root() is None:
    pytest.skip("the reference is not installed")
  import bench
  from tsp_gpu_clean_b200 import instances

  for name in ("ga100", "chapter4"):
    n, P, G, elite, post_init, seed, _ = bench.GA_WORKLOADS[name]
    o = bench.ga_options(name)
    ref = reference_arm.ga_gens_per_s(instances.uniform_instance(n, seed), P, elite, post_init, 2, o)
    assert ref["value"] > 0
    from oracle import distances as odist
    from oracle import ga as oga

    coords = instances.uniform_instance(n, seed)
    cache = {}

    def provider(k, coords=coords, cache=cache):
      if k not in cache:
        cache[k] = odist.candidate_list(k, coords=coords)
      return cache[k]

    cfg = oga.GAConfig(population_size=P, mutation_rate=o["rate"], nn_k=5, tournament_k=5,
                       local_search=oga.LocalSearchSpec("best", 10, 20), post_init=post_init,
                       elite_count=elite or None, local_search_stage=o["stage"], crossover=o["crossover"],
                       mutation=o["mutation"], init=o["init"])
    import numpy as np

    res = oga.OracleGA(odist.euc2d_matrix(coords), provider, cfg, np.random.default_rng(42)).evolve(2, patience=10**9)
    assert ref["history"] == [float(v) for v in res[3]["convergence_history"]], name
