"""The uneven multi-instance batch against the reference's recorded runs and the oracle GA."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import distances as odist
from oracle import ga as oga

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch_mod():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  from tsp_gpu_clean_b200 import batch

  return batch


def _digest(t):
  return hashlib.sha256(np.ascontiguousarray(t.cpu().numpy(), dtype=np.int32).tobytes()).hexdigest()


def _oracle_run(coords, seed, P, rate, elite, post_init, mode, iters, k, G, patience):
  D = odist.euc2d_matrix(coords)
  cfg = oga.GAConfig(population_size=P, mutation_rate=rate, nn_k=5, tournament_k=5,
                     local_search=oga.LocalSearchSpec(mode, iters, k), post_init=post_init, elite_count=elite)
  cache = {}

  def provider(kk):
    if kk not in cache:
      cache[kk] = odist.candidate_list(kk, coords=coords)
    return cache[kk]

  rng = np.random.default_rng(seed)
  best, pop, fit, stats, _ = oga.OracleGA(D, provider, cfg, rng).evolve(G, patience=patience)
  return best, pop, fit, stats, rng


def _check_run(solver, res, ctxs, idx, oracle):
  obest, opop, ofit, ostats, orng = oracle
  best, stats = res[idx]
  assert stats["generations_completed"] == ostats["generations_completed"]
  assert np.array_equal(best, obest)
  assert np.array_equal(solver.final_population[idx].cpu().numpy(), opop)
  assert np.array_equal(solver.final_fitness[idx].cpu().numpy(), ofit)
  assert stats["convergence_history"] == ostats["convergence_history"]
  assert ctxs[idx].rng.bit_generator.state == orng.bit_generator.state


def _keep_sources():
  """A tuner that times launch shapes but never moves a matrix bucket to distances rebuilt
  from coordinates (odd candidates), so a test's mix of bucket sources does not depend on
  which source measured faster."""
  from tsp_gpu_clean_b200.autotune import BatchAutotuner

  class KeepSources(BatchAutotuner):
    def choose(self, key, candidates, probe):
      cands = list(candidates)
      if "|two_opt|" in key:
        cands = [c for c in cands if not c & 1] or cands
      return super().choose(key, cands, probe)

  return KeepSources()


def _lattice(w, h, step=10.0):
  return np.array([[x * step, y * step] for x in range(w) for y in range(h)], dtype=np.float64)


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_matches_reference_runs_and_oracle(batch_mod, golden, use_graph):
  """The 100-city reference runs (fixed and default patience) inside one batch with
  smaller and larger instances; the largest rebuilds distances from coordinates."""
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.instances import clustered_instance, uniform_instance
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  g = golden("ga.npz")
  c1 = g["c1_coords"]
  extra = [(uniform_instance(23, 5), 11), (clustered_instance(150, 6, 30.0, 6), 12), (uniform_instance(61, 7), 13)]
  specs = [(c1, 42, 10**9), (c1, 42, None)] + [(c, s, 10**9) for c, s in extra]
  ctxs = [ProblemContext(Problem.from_coordinates(c), seed=s) for c, s, _ in specs]
  solver = batch_mod.FusedBatchSolver(population_size=128, mutation_rate=0.05, tournament_k=5, nn_k=5,
                                      local_search=LocalSearchConfig("best", 10, 20), elite_count=16, post_init=True,
                                      max_matrix_dimension=120, use_graph=use_graph, bucket_bounds=(32, 100, 128),
                                      tuner=_keep_sources())
  res = solver.evolve(ctxs, 50, patience=[p for _, _, p in specs])
  assert any(b.coords for b in solver.buckets) and any(not b.coords for b in solver.buckets)
  for tag, idx in (("c1", 0), ("c1default", 1)):
    best, stats = res[idx]
    assert stats["generations_completed"] == int(g[f"{tag}_gens"])
    assert np.array_equal(np.asarray(stats["convergence_history"]), g[f"{tag}_history"])
    assert np.array_equal(best, g[f"{tag}_best"])
    assert _digest(solver.final_population[idx]) == str(g[f"{tag}_digests"][-1])
    assert np.array_equal(solver.final_fitness[idx].cpu().numpy(), g[f"{tag}_fitness"][-1])
    assert ctxs[idx].rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"{tag}_rng"][0])
  for j, (coords, seed) in enumerate(extra):
    _check_run(solver, res, ctxs, 2 + j, _oracle_run(coords, seed, 128, 0.05, 16, True, "best", 10, 20, 50, 10**9))
  assert solver.two_opt_totals["pairs"] > 0


@pytest.mark.parametrize("iters", [2, 50])
def test_batch_elite_boundary_ties_match_oracle(batch_mod, iters):
  """Lattice instances of different sizes tie at the elite edge in most generations. With
  few 2-opt passes the tied rows are often unconverged (the run pauses for the host's
  argsort); with many passes they are converged duplicates (settled on the device)."""
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  lattices = [(_lattice(6, 6), 3), (_lattice(5, 7), 4), (_lattice(8, 8), 5), (_lattice(4, 5), 6)]
  ctxs = [ProblemContext(Problem.from_coordinates(c), seed=s) for c, s in lattices]
  solver = batch_mod.FusedBatchSolver(population_size=40, mutation_rate=0.3, elite_count=6, post_init=False,
                                      local_search=LocalSearchConfig("best", iters, 8), max_matrix_dimension=40,
                                      bucket_bounds=(36,), chunk=4)
  res = solver.evolve(ctxs, 40, patience=10**9)
  ties = sum(st["elite_edge_ties"] for _, st in res)
  host = sum(st["host_elite_generations"] for _, st in res)
  if iters == 2:
    assert host > 0
  else:
    assert ties > host
  for idx, (coords, seed) in enumerate(lattices):
    _check_run(solver, res, ctxs, idx, _oracle_run(coords, seed, 40, 0.3, 6, False, "best", iters, 8, 40, 10**9))


@pytest.mark.parametrize("incremental", ["on", "off"])
def test_batch_first_mode_and_early_stop_match_oracle(batch_mod, incremental):
  """First mode, with (on) or without (off) the incremental restart through the reverse
  k-NN index (k = 12 for the grouped layout that it needs), and patience stops."""
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.instances import uniform_instance
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  insts = [(uniform_instance(n, 100 + n), 200 + n) for n in (9, 40, 77, 130)]
  ctxs = [ProblemContext(Problem.from_coordinates(c), seed=s) for c, s in insts]
  solver = batch_mod.FusedBatchSolver(population_size=24, mutation_rate=0.2, elite_count=5, post_init=True,
                                      local_search=LocalSearchConfig("first", 4, 12), max_matrix_dimension=100,
                                      incremental=incremental)
  res = solver.evolve(ctxs, 30, patience=3)
  assert any(st["stopped_early"] for _, st in res)
  for idx, (coords, seed) in enumerate(insts):
    _check_run(solver, res, ctxs, idx, _oracle_run(coords, seed, 24, 0.2, 5, True, "first", 4, 12, 30, 3))
  assert any(b.incremental for b in solver.buckets) == (incremental == "on")


@pytest.mark.parametrize("threads", [128, 1024])
def test_cta_pairs_match_oracle(batch_mod, threads):
  """Best-mode 2-opt with every row refined by a two-CTA cluster (pair="on"): post-init on
  every row, elites each generation, lattices whose elite edges tie, a rebuilt-distance
  bucket. Runs must equal the oracle's exactly (tours, fitness, history, generator)."""
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.instances import clustered_instance, uniform_instance
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  from tsp_gpu_clean_b200.autotune import BatchAutotuner

  class Pick(BatchAutotuner):
    """Pairs of `threads`-thread CTAs for the 2-opt; the middle candidate elsewhere."""

    def choose(self, key, candidates, probe):
      if "|two_opt|" in key:
        return next(c for c in candidates if c // 8 == threads and c & 4)
      return super().choose(key, candidates, probe)

  insts = [(uniform_instance(57, 31), 41), (clustered_instance(260, 8, 30.0, 32), 42), (_lattice(7, 7), 43),
           (uniform_instance(300, 33), 44)]
  ctxs = [ProblemContext(Problem.from_coordinates(c), seed=s) for c, s in insts]
  solver = batch_mod.FusedBatchSolver(population_size=32, mutation_rate=0.2, elite_count=6, post_init=True,
                                      local_search=LocalSearchConfig("best", 10, 8), max_matrix_dimension=280,
                                      pair="on", tuner=Pick(enabled=False), bucket_bounds=(64, 256), chunk=4)
  res = solver.evolve(ctxs, 25, patience=10**9)
  assert all(b.pair and b.two_opt_threads == threads for b in solver.buckets)
  assert any(b.coords for b in solver.buckets)
  for idx, (coords, seed) in enumerate(insts):
    _check_run(solver, res, ctxs, idx, _oracle_run(coords, seed, 32, 0.2, 6, True, "best", 10, 8, 25, 10**9))


def test_converged_row_skipping_changes_nothing(batch_mod):
  """Skipping the refinement of converged rows gives the same runs, with less 2-opt work."""
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.instances import uneven_batch
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  coords = uneven_batch(5, 21, n_min=30, n_max=400)
  out = []
  for skip in (True, False):
    ctxs = [ProblemContext(Problem.from_coordinates(c), seed=50 + i) for i, c in enumerate(coords)]
    solver = batch_mod.FusedBatchSolver(population_size=32, elite_count=6, skip_converged=skip,
                                        local_search=LocalSearchConfig("best", 10, 20))
    res = solver.evolve(ctxs, 25, patience=10**9)
    out.append(([r[0] for r in res], [p.cpu().numpy() for p in solver.final_population],
                solver.two_opt_totals["pairs"], [r[1]["convergence_history"] for r in res]))
  for a, b in zip(out[0][0], out[1][0]):
    assert np.array_equal(a, b)
  for a, b in zip(out[0][1], out[1][1]):
    assert np.array_equal(a, b)
  assert out[0][3] == out[1][3]
  assert out[0][2] < out[1][2]


def test_autotuner_cache_is_reused(batch_mod, tmp_path):
  from tsp_gpu_clean_b200.autotune import BatchAutotuner
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.instances import uneven_batch
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  coords = uneven_batch(6, 9, n_min=50, n_max=600)
  path = str(tmp_path / "tune.json")
  outs = []
  for rep in range(2):
    tuner = BatchAutotuner(cache_path=path)
    ctxs = [ProblemContext(Problem.from_coordinates(c), seed=i) for i, c in enumerate(coords)]
    solver = batch_mod.FusedBatchSolver(population_size=16, elite_count=4,
                                        local_search=LocalSearchConfig("best", 10, 20), tuner=tuner)
    res = solver.evolve(ctxs, 5, patience=10**9)
    outs.append([r[0] for r in res])
    if rep == 0:
      assert tuner.measured > 0
    else:
      assert tuner.measured == 0
  for a, b in zip(*outs):
    assert np.array_equal(a, b)


@pytest.mark.parametrize("concurrent", [True, False])
def test_rebuilt_distances_and_serial_buckets_match_oracle(batch_mod, concurrent):
  """A tuner that always picks distances rebuilt from coordinates (buckets drop their
  matrices), with buckets launched concurrently or one after another: same runs."""
  from tsp_gpu_clean_b200.autotune import BatchAutotuner
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.instances import uniform_instance
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  class PickRebuild(BatchAutotuner):
    def choose(self, key, candidates, probe):
      odd = [c for c in candidates if c & 1]
      return odd[-1] if ("two_opt" in key and odd) else list(candidates)[0]

  insts = [(uniform_instance(n, 300 + n), 400 + n) for n in (33, 90, 180, 260)]
  ctxs = [ProblemContext(Problem.from_coordinates(c), seed=s) for c, s in insts]
  solver = batch_mod.FusedBatchSolver(population_size=24, mutation_rate=0.1, elite_count=4, post_init=True,
                                      local_search=LocalSearchConfig("best", 10, 20), tuner=PickRebuild(),
                                      bucket_bounds=(64, 128), concurrent_buckets=concurrent)
  res = solver.evolve(ctxs, 15, patience=10**9)
  assert all(b.coords for b in solver.buckets)
  for idx, (coords, seed) in enumerate(insts):
    _check_run(solver, res, ctxs, idx, _oracle_run(coords, seed, 24, 0.1, 4, True, "best", 10, 20, 15, 10**9))


def test_device_tape_equals_numpy(batch_mod):
  """`tspb_tape_draw` (one thread per run) gives every run NumPy's draws and end state."""
  import ctypes

  import torch

  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle
  from tsp_gpu_clean_b200.fused import draw_generation_tape_numpy

  ns, G, P, kt = [5, 17, 300, 4899, 4], 12, 10, 5
  rngs = [np.random.default_rng(70 + i) for i in range(len(ns))]
  for i, r in enumerate(rngs):
    r.integers(0, 9, size=i, dtype=np.int32)
  refs = [np.random.Generator(np.random.PCG64()) for _ in ns]
  for r, q in zip(refs, rngs):
    r.bit_generator.state = q.bit_generator.state
  I = len(ns)
  h = (native.Pcg64 * I)(*[native.Pcg64.from_state(r.bit_generator.state) for r in rngs])
  d_gens = torch.frombuffer(bytearray(h), dtype=torch.uint8).cuda()
  d_ns = torch.tensor(ns, dtype=torch.int32, device="cuda")
  tape = [torch.zeros((I, G, P, kt), dtype=torch.int32, device="cuda"),
          torch.zeros((I, G, P // 2), dtype=torch.int32, device="cuda"),
          torch.zeros((I, G, P // 2), dtype=torch.int32, device="cuda"),
          torch.zeros((I, G, P), dtype=torch.float64, device="cuda"),
          torch.zeros((I, G, P), dtype=torch.int32, device="cuda"),
          torch.zeros((I, G, P), dtype=torch.int32, device="cuda")]
  states = torch.zeros(I * G * ctypes.sizeof(native.Pcg64), dtype=torch.uint8, device="cuda")
  native.call("tspb_tape_draw", ptr(d_gens), ptr(d_ns), I, G, P, kt, *[ptr(t) for t in tape], ptr(states),
              stream_handle())
  final = (native.Pcg64 * I).from_buffer_copy(d_gens.cpu().numpy().tobytes())
  per_gen = (native.Pcg64 * (I * G)).from_buffer_copy(states.cpu().numpy().tobytes())
  for i, (r, n) in enumerate(zip(refs, ns)):
    want, wst = draw_generation_tape_numpy(r, G, P, kt, n)
    for t, w in zip(tape, want):
      assert np.array_equal(t[i].cpu().numpy(), w)
    assert [per_gen[i * G + g].to_state() for g in range(G)] == list(wst)
    assert final[i].to_state() == r.bit_generator.state


def test_many_small_runs_device_tape_match_oracle(batch_mod):
  """34 runs (the tape is drawn on the device from 32 runs up), every one bit-exact."""
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.instances import uniform_instance
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  assert batch_mod.DEVICE_TAPE_MIN_RUNS <= 34
  insts = [(uniform_instance(5 + (7 * i) % 26, 500 + i), 600 + i) for i in range(34)]
  ctxs = [ProblemContext(Problem.from_coordinates(c), seed=s) for c, s in insts]
  solver = batch_mod.FusedBatchSolver(population_size=10, mutation_rate=0.2, elite_count=3, post_init=True,
                                      local_search=LocalSearchConfig("best", 5, 6))
  res = solver.evolve(ctxs, 6, patience=10**9)
  assert solver._dev_states is not None
  for idx, (coords, seed) in enumerate(insts):
    _check_run(solver, res, ctxs, idx, _oracle_run(coords, seed, 10, 0.2, 3, True, "best", 5, 6, 6, 10**9))


def test_sharded_solver_on_one_rank_equals_the_batch_solver(batch_mod):
  """Without a process group the sharded solver runs every instance on one batch solver:
  the same best tours and costs as FusedBatchSolver.evolve."""
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.instances import uneven_batch
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext
  from tsp_gpu_clean_b200.sharding import ShardedBatchSolver

  coords = uneven_batch(5, 33, n_min=20, n_max=300)

  def make():
    return batch_mod.FusedBatchSolver(population_size=24, elite_count=4,
                                      local_search=LocalSearchConfig("best", 10, 20))

  ref = make().evolve([ProblemContext(Problem.from_coordinates(c), seed=60 + i) for i, c in enumerate(coords)], 8,
                      patience=10**9)
  sharded = ShardedBatchSolver(make, population_size=24)
  got = sharded.evolve([ProblemContext(Problem.from_coordinates(c), seed=60 + i) for i, c in enumerate(coords)], 8,
                       patience=10**9)
  assert sharded.plan == [list(range(5))]
  for (best, stats), (tour, cost) in zip(ref, got):
    assert np.array_equal(best, tour) and cost == stats["best_fitness"]
