"""The graph-replayed fused GA against the reference's recorded runs and the oracle GA."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import distances as odist
from oracle import ga as oga

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fused_mod():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  from tsp_gpu_clean_b200 import fused

  return fused


def _digest(t):
  return hashlib.sha256(np.ascontiguousarray(t.cpu().numpy(), dtype=np.int32).tobytes()).hexdigest()


@pytest.mark.parametrize("engine", ["batch", "single"])
@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("tag", ["c1", "c1default", "c3"])
def test_fused_matches_reference(fused_mod, golden, tag, use_graph, engine):
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  g = golden("ga.npz")
  coords = g[f"{tag}_coords"]
  pop_size, gens, elite, post_init, ls_iters, seed, _, _ = (int(v) for v in g[f"{tag}_meta"])
  ctx = ProblemContext(Problem.from_coordinates(coords), seed=seed)
  solver = fused_mod.FusedMemeticSolver(population_size=pop_size, mutation_rate=float(g[f"{tag}_rate"]), tournament_k=5,
                                        nn_k=5, local_search=fused_mod.LocalSearchConfig("best", ls_iters, 20),
                                        elite_count=elite, post_init=bool(post_init), use_graph=use_graph, chunk=7,
                                        engine=engine)
  patience = None if tag == "c1default" else 10**9
  best, stats = solver.evolve(ctx, list(range(len(coords))), gens, patience=patience)
  assert stats["generations_completed"] == int(g[f"{tag}_gens"])
  assert np.array_equal(np.asarray(stats["convergence_history"]), g[f"{tag}_history"])
  assert np.array_equal(best, g[f"{tag}_best"])
  assert _digest(solver.final_population) == str(g[f"{tag}_digests"][-1])
  assert np.array_equal(solver.final_fitness.cpu().numpy(), g[f"{tag}_fitness"][-1])
  assert ctx.rng.bit_generator.state["state"]["state"] % (1 << 63) == int(g[f"{tag}_rng"][0])


@pytest.mark.parametrize("engine", ["batch", "single"])
def test_fused_with_elite_boundary_ties_matches_oracle(fused_mod, engine):
  """Integer-lattice cities give many equal tour lengths: ties across the elite edge
  make membership depend on NumPy's unstable argsort, resolved on the host."""
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  side = 6
  coords = np.array([[x * 10.0, y * 10.0] for x in range(side) for y in range(side)])
  n = len(coords)
  for seed in (3, 4):
    ctx = ProblemContext(Problem.from_coordinates(coords), seed=seed)
    solver = fused_mod.FusedMemeticSolver(population_size=40, mutation_rate=0.3, elite_count=6, post_init=False,
                                          local_search=fused_mod.LocalSearchConfig("best", 2, 8), chunk=5,
                                          engine=engine)
    best, stats = solver.evolve(ctx, list(range(n)), 40, patience=10**9)
    D = odist.euc2d_matrix(coords)
    cfg = oga.GAConfig(population_size=40, mutation_rate=0.3, nn_k=5, tournament_k=5,
                       local_search=oga.LocalSearchSpec("best", 2, 8), post_init=False, elite_count=6)
    cache = {}

    def provider(k):
      if k not in cache:
        cache[k] = odist.candidate_list(k, coords=coords)
      return cache[k]

    rng = np.random.default_rng(seed)
    obest, opop, ofit, ostats, _ = oga.OracleGA(D, provider, cfg, rng).evolve(40, patience=10**9)
    assert np.array_equal(best, obest)
    assert np.array_equal(solver.final_population.cpu().numpy(), opop)
    assert np.array_equal(solver.final_fitness.cpu().numpy(), ofit)
    assert stats["convergence_history"] == ostats["convergence_history"]
    assert ctx.rng.bit_generator.state == rng.bit_generator.state
