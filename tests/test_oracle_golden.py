"""Pin the CPU oracle against golden vectors produced by the reference itself.

The fixtures under `tests/golden/` were generated by `tests/golden/make_golden.py`,
which runs the reference's CPU strategies. Every oracle function used as the
checker of the CUDA path must reproduce them bit for bit.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import iter_two_opt_cases
from oracle import distances, ga, ga_ops, two_opt
from tsp_gpu_clean_b200 import instances


def test_two_opt_small_cases_match_reference(golden):
  data = golden("two_opt_small.npz")
  count = 0
  for c, n, k, mode, iters, D, cand, tin, tout in iter_two_opt_cases(data):
    cand_used = two_opt.resolve_candidates(cand, tin, n) if k is not None else None
    got, _ = two_opt.improve_batch(tin, D, cand_used, mode, iters)
    assert np.array_equal(got, tout), f"case {c}: n={n} k={k} mode={mode} iters={iters}"
    count += 1
  assert count == int(data["num_cases"])


def test_candidate_tables_match_reference(golden):
  data = golden("two_opt_small.npz")
  for c, n, k, mode, iters, D, cand, tin, tout in iter_two_opt_cases(data):
    if cand is None or f"c{c}_coords" not in data or cand.shape[1] != min(k, n - 1):
      continue
    if n >= 12 and k == 6:
      continue  # hand-built duplicate tables
    assert np.array_equal(distances.candidate_list(k, coords=data[f"c{c}_coords"]), cand), c


@pytest.mark.parametrize("mode", ["best", "first"])
def test_two_opt_c2_subset_matches_reference_with_counts(golden, mode):
  data = golden("two_opt_c2.npz")
  D = distances.euc2d_matrix(data["coords"])
  cand = data["cand20"]
  assert np.array_equal(distances.candidate_list(20, coords=data["coords"]), cand)
  got, stats = two_opt.improve_batch(data["tours_in"][:1], D, cand, mode, 10**9)
  assert np.array_equal(got, data[f"{mode}_out"][:1])
  assert stats[0, 0] == data[f"{mode}_stats"][0, 0]  # passes
  assert stats[0, 1] == data[f"{mode}_stats"][0, 1]  # pairs evaluated


def test_c2_workload_generator_is_stable(golden):
  data = golden("two_opt_c2.npz")
  coords, tours = instances.two_opt_workload(tours=4)
  assert np.array_equal(coords, data["coords"])
  assert np.array_equal(tours, data["tours_in"])


def test_distance_matrix_and_knn_match_reference(golden):
  ops = golden("ops.npz")
  D = distances.euc2d_matrix(ops["dist_coords"])
  assert np.array_equal(D, ops["dist_matrix"])
  assert D[0, 1] == 1 and D[1, 0] == 1  # sqrt(0.25)+0.5 == 1.0 exactly
  assert np.array_equal(distances.candidate_list(5, coords=ops["dist_coords"]), ops["dist_cand5"])
  assert np.array_equal(distances.candidate_list(20, distances=D), ops["dist_cand20"])
  big = distances.euc2d_matrix(ops["big_coords"])
  assert hashlib.sha256(big.tobytes()).digest() == ops["big_digest"].tobytes()


@pytest.mark.parametrize("tag", ["a", "b", "c", "d"])
def test_operators_match_reference(golden, tag):
  ops = golden("ops.npz")
  n, pop_size, seed = (int(v) for v in ops[f"{tag}_meta"])
  rate = float(ops[f"{tag}_rate"])
  D = distances.euc2d_matrix(ops[f"{tag}_coords"])
  rng = np.random.default_rng(seed)
  pop = ops[f"{tag}_pop"]
  fit = ga_ops.tour_cost(pop, D)
  assert np.array_equal(fit, ops[f"{tag}_fit"])
  sel = ga_ops.tournament_select(rng, pop, fit, pop_size, 5)
  assert np.array_equal(sel, ops[f"{tag}_sel"])
  pmx = ga_ops.pmx_batch(rng, sel)
  assert np.array_equal(pmx, ops[f"{tag}_pmx"])
  inv = ga_ops.inversion_batch(rng, pmx, rate)
  assert np.array_equal(inv, ops[f"{tag}_inv"])
  assert rng.bit_generator.state["state"]["state"] % (1 << 63) == int(ops[f"{tag}_rng_state"][0])


def _run_oracle_ga(g, tag, record=True):
  coords = g[f"{tag}_coords"]
  pop_size, gens, elite, post_init, ls_iters, seed, per_int, per_tgt = (int(v) for v in g[f"{tag}_meta"])
  stage = str(g[f"{tag}_stage"])
  D = distances.euc2d_matrix(coords)
  cache = {}

  def provider(k):
    if k not in cache:
      cache[k] = distances.candidate_list(k, coords=coords)
    return cache[k]

  cfg = ga.GAConfig(population_size=pop_size, mutation_rate=float(g[f"{tag}_rate"]), nn_k=5, tournament_k=5,
                    local_search=ga.LocalSearchSpec("best", ls_iters, 20), local_search_stage=stage,
                    post_init=bool(post_init), elite_count=elite or None,
                    periodic=None if per_int < 0 else (per_int, "offspring" if per_tgt == 0 else "population"))
  rng = np.random.default_rng(seed)
  patience = None if tag == "c1default" else 10**9
  return ga.OracleGA(D, provider, cfg, rng).evolve(gens, patience=patience, record=record), rng


@pytest.mark.parametrize("tag", ["c1", "c1default", "pm", "pc", "pe", "px", "pp", "po"])
def test_ga_runs_match_reference(golden, tag):
  g = golden("ga.npz")
  (best, pop, fit, stats, records), rng = _run_oracle_ga(g, tag)
  assert np.array_equal(best, g[f"{tag}_best"])
  assert np.array_equal(np.asarray(stats["convergence_history"]), g[f"{tag}_history"])
  assert stats["generations_completed"] == int(g[f"{tag}_gens"])
  digests = [r[0] for r in records]
  assert digests == [str(d) for d in g[f"{tag}_digests"]]
  assert np.array_equal(np.stack([r[1] for r in records]), g[f"{tag}_fitness"])
  assert rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"{tag}_rng"][0])


def test_nn_init_matches_reference(golden):
  g = golden("ga.npz")
  coords = g["c1_coords"]
  rng = np.random.default_rng(42)
  pop = ga_ops.nn_init(rng, np.arange(100), 128, distances.candidate_list(5, coords=coords))
  assert np.array_equal(pop, g["c1_init"])


@pytest.mark.parametrize("tag", ["a", "b", "c", "d", "e", "f"])
def test_ox_and_swap_match_reference(golden, tag):
  g = golden("ox_swap.npz")
  n, pop_size, seed = (int(v) for v in g[f"{tag}_meta"])
  rng = np.random.default_rng(seed)
  ox = ga_ops.ox_batch(rng, g[f"{tag}_pop"])
  assert np.array_equal(ox, g[f"{tag}_ox"])
  sw = ga_ops.swap_batch(rng, ox, float(g[f"{tag}_rate"]))
  assert np.array_equal(sw, g[f"{tag}_swap"])
  assert rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"{tag}_rng_state"][0])
  for row in sw:
    assert np.array_equal(np.sort(row), np.arange(n))


@pytest.mark.parametrize("tag", ["ox1", "ox2"])
def test_oracle_ga_with_ox_and_swap_matches_reference(golden, tag):
  g = golden("ox_swap.npz")
  coords = g[f"ga_{tag}_coords"]
  pop_size, gens, elite, post_init, patience = (int(v) for v in g[f"ga_{tag}_meta"])
  D = distances.euc2d_matrix(coords)
  cache = {}

  def provider(k):
    if k not in cache:
      cache[k] = distances.candidate_list(k, coords=coords)
    return cache[k]

  cfg = ga.GAConfig(population_size=pop_size, mutation_rate=float(g[f"ga_{tag}_rate"]), nn_k=5, tournament_k=5,
                    local_search=ga.LocalSearchSpec("best", 10, 20), post_init=bool(post_init), elite_count=elite,
                    crossover="ox", mutation="swap")
  rng = np.random.default_rng(7)
  best, _, _, stats, _ = ga.OracleGA(D, provider, cfg, rng).evolve(gens, patience=None if patience < 0 else patience)
  assert stats["generations_completed"] == int(g[f"ga_{tag}_gens"])
  assert np.array_equal(np.asarray(stats["convergence_history"]), g[f"ga_{tag}_history"])
  assert np.array_equal(best, g[f"ga_{tag}_best"])
  assert rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"ga_{tag}_rng"][0])


@pytest.mark.parametrize("tag", ["r1", "r2", "r3", "r4", "r5"])
def test_random_init_matches_reference(golden, tag):
  import hashlib

  g = golden("stage.npz")
  n, pop_size, seed = (int(v) for v in g[f"{tag}_meta"])
  rng = np.random.default_rng(seed)
  pop = ga_ops.random_init(rng, g[f"{tag}_customers"], pop_size)
  if f"{tag}_pop" in g:
    assert np.array_equal(pop, g[f"{tag}_pop"])
  else:
    assert hashlib.sha256(np.ascontiguousarray(pop, dtype=np.int32).tobytes()).digest() == g[f"{tag}_digest"].tobytes()
  assert rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"{tag}_rng_state"][0])


def stage_config(g, tag):
  """GAConfig of a `stage.npz` run: 2-opt on every offspring, in the Chapter-4 configuration
  (random init, OX, swap) or with NN init, PMX, inversion and the post-init/elite steps."""
  pop_size, gens, elite, post_init, patience, chapter4 = (int(v) for v in g[f"ga_{tag}_meta"])
  cfg = ga.GAConfig(population_size=pop_size, mutation_rate=float(g[f"ga_{tag}_rate"]), nn_k=5, tournament_k=5,
                    local_search=ga.LocalSearchSpec("best", 10, 20), local_search_stage="post_mutation",
                    post_init=bool(post_init), elite_count=elite or None,
                    crossover="ox" if chapter4 else "pmx", mutation="swap" if chapter4 else "inversion",
                    init="random" if chapter4 else "nn")
  return cfg, gens, (None if patience < 0 else patience)


@pytest.mark.parametrize("tag", ["s1", "s2", "s3"])
def test_oracle_ga_with_post_mutation_stage_matches_reference(golden, tag):
  g = golden("stage.npz")
  coords = g[f"ga_{tag}_coords"]
  cfg, gens, patience = stage_config(g, tag)
  cache = {}

  def provider(k):
    if k not in cache:
      cache[k] = distances.candidate_list(k, coords=coords)
    return cache[k]

  rng = np.random.default_rng(42)
  best, _, _, stats, _ = ga.OracleGA(distances.euc2d_matrix(coords), provider, cfg, rng).evolve(gens, patience=patience)
  assert stats["generations_completed"] == int(g[f"ga_{tag}_gens"])
  assert np.array_equal(np.asarray(stats["convergence_history"]), g[f"ga_{tag}_history"])
  assert np.array_equal(best, g[f"ga_{tag}_best"])
  assert rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"ga_{tag}_rng"][0])


DIST_TYPES = ("EUC_2D", "EUC_3D", "MAN_2D", "MAN_3D", "MAX_2D", "MAX_3D", "CEIL_2D", "ATT", "GEO", "XRAY1")


@pytest.mark.parametrize("edge_type", DIST_TYPES)
def test_distance_types_match_reference(golden, edge_type):
  import hashlib

  from tests.golden.make_golden import dist_coords

  g = golden("distances.npz")
  c = g[f"{edge_type}_120_coords"]
  assert np.array_equal(distances.distance_matrix(c, edge_type), g[f"{edge_type}_120_matrix"])
  assert np.array_equal(distances.candidate_list(8, coords=c, edge_type=edge_type), g[f"{edge_type}_120_knn"])
  j = DIST_TYPES.index(edge_type)
  c = dist_coords(edge_type, 2500, 700 + 10 * j + 1)
  d = distances.distance_matrix(c, edge_type)
  assert hashlib.sha256(d.tobytes()).digest() == g[f"{edge_type}_2500_digest"].tobytes()
  knn = np.ascontiguousarray(distances.candidate_list(10, coords=c, edge_type=edge_type))
  assert hashlib.sha256(knn.tobytes()).digest() == g[f"{edge_type}_2500_knn_digest"].tobytes()


THREE_OPT_TAGS = ["u5", "u6", "u9", "u16", "u40", "lat16", "lat36"]


def _three_opt_matrix(coords):
  diff = coords[:, None, :] - coords[None, :, :]
  d = (np.sqrt((diff * diff).sum(axis=2)) + 0.5).astype(np.int32)
  np.fill_diagonal(d, 0)
  return d


@pytest.mark.parametrize("tag", THREE_OPT_TAGS)
def test_three_opt_matches_reference(golden, tag):
  from oracle import three_opt

  g = golden("three_opt.npz")
  D = _three_opt_matrix(g[f"{tag}_coords"])
  assert np.array_equal(D, distances.euc2d_matrix(g[f"{tag}_coords"]))
  for t, want in zip(g[f"{tag}_tours"], g[f"{tag}_best"]):
    assert tuple(three_opt.best_move(t, D)) == tuple(int(v) for v in want)
  for iters in (1, 3, 1000):
    got, _ = three_opt.improve_batch(g[f"{tag}_tours"], D, iters)
    assert np.array_equal(got, g[f"{tag}_refined{iters}"]), iters


@pytest.mark.parametrize("tag", THREE_OPT_TAGS)
def test_three_opt_kernel_rules_with_one_thread_equal_the_cpu_three_opt(golden, tag):
  """With one thread per tour the reference's grid kernels scan every anchor in the CPU
  3-opt's order and keep the first strictly smallest move, and multi_move applies at most
  min(1, n // 2) = 1 move per pass: the kernel restatement must then give the reference's
  CPU 3-opt refinements (which `three_opt.npz` records)."""
  from oracle import three_opt_kernel as tk

  g = golden("three_opt.npz")
  D = _three_opt_matrix(g[f"{tag}_coords"])
  for iters in (1, 3, 1000):
    for t, want in zip(g[f"{tag}_tours"], g[f"{tag}_refined{iters}"]):
      for mode in ("batch", "multi_move"):
        got, _ = tk.refine(t, D, None, 0, 1, mode, iters)
        assert np.array_equal(got, want), (tag, iters, mode)


def test_three_opt_kernel_rules_match_reference_kernels(golden):
  """The restatement against outputs of the reference's own 3-opt CUDA kernels
  (`three_opt_kernel.npz`, recorded by make_three_opt_kernel_golden.py)."""
  import os

  from conftest import GOLDEN
  from oracle import three_opt_kernel as tk

  if not os.path.exists(os.path.join(GOLDEN, "three_opt_kernel.npz")):
    pytest.skip("three_opt_kernel.npz not recorded yet")
  g = golden("three_opt_kernel.npz")
  for tag in g["tags"]:
    n, k, inner, tpb, multi, iters, B = (int(v) for v in g[f"{tag}_meta"])
    assert tk.virtual_threads(tpb, n) == B
    D = distances.euc2d_matrix(g[f"{tag}_coords"])
    cand = g[f"{tag}_cand"] if k > 0 else None
    mode = "multi_move" if multi else "batch"
    for t, want in zip(g[f"{tag}_in"], g[f"{tag}_out"]):
      got, _ = tk.refine(t, D, cand, inner, tpb, mode, iters)
      assert np.array_equal(got, want), str(tag)
