"""Distance matrices of every TSPLIB coordinate type on the B200 against the reference's
matrices (`tests/golden/distances.npz`), and the 2-opt and GA on non-EUC_2D problems
against the oracle."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import distances as odist
from oracle import ga as oga
from oracle import two_opt as otwo
from tests.golden.make_golden import DIST_TYPES, dist_coords

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  return torch


def _device_matrix(torch, c, edge_type, pad=0):
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  n, dim = c.shape
  ld = n + pad
  out = torch.full((n, ld), -7, dtype=torch.int32, device="cuda")
  dc = torch.from_numpy(np.ascontiguousarray(c, dtype=np.float64)).cuda()
  native.call("tspb_distance_matrix", ptr(dc), n, dim, native.EDGE_TYPE_CODES[edge_type], ptr(out), ld, stream_handle())
  h = out.cpu().numpy()
  assert (h[:, n:] == -7).all()  # the padding columns are untouched
  return np.ascontiguousarray(h[:, :n])


@pytest.mark.parametrize("edge_type", DIST_TYPES)
def test_distance_matrix_matches_reference(torch_mod, golden, edge_type):
  g = golden("distances.npz")
  c = g[f"{edge_type}_120_coords"]
  assert np.array_equal(_device_matrix(torch_mod, c, edge_type, pad=5), g[f"{edge_type}_120_matrix"])
  j = DIST_TYPES.index(edge_type)
  c = dist_coords(edge_type, 2500, 700 + 10 * j + 1)
  d = _device_matrix(torch_mod, c, edge_type)
  assert hashlib.sha256(d.tobytes()).digest() == g[f"{edge_type}_2500_digest"].tobytes()


def test_distance_matrix_rejects_bad_arguments(torch_mod):
  from tsp_gpu_clean_b200 import native

  lib = native.load_library()
  assert lib.tspb_distance_matrix(None, 4, 2, 99, None, 4, None) == native.TSPB_ERR_ARG
  assert lib.tspb_distance_matrix(None, 4, 2, native.EDGE_TYPE_CODES["XRAY1"], None, 4, None) == native.TSPB_ERR_ARG
  assert lib.tspb_distance_matrix(None, 4, 4, 0, None, 4, None) == native.TSPB_ERR_ARG
  assert lib.tspb_distance_matrix(None, 4, 2, 0, None, 3, None) == native.TSPB_ERR_ARG
  assert lib.tspb_distance_matrix(None, 0, 2, 0, None, 0, None) == native.TSPB_OK


@pytest.mark.parametrize("edge_type", ["ATT", "GEO", "CEIL_2D", "MAN_3D"])
def test_two_opt_on_non_euclidean_types_matches_oracle(torch_mod, edge_type):
  from tsp_gpu_clean_b200 import instances
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext
  from tsp_gpu_clean_b200.strategies import LocalSearchB200TourTwoOpt

  c = dist_coords(edge_type, 300, 55)
  ctx = ProblemContext(Problem.from_coordinates(c, edge_type=edge_type), seed=1)
  tours = instances.random_tours(300, 6, 9)
  D = odist.distance_matrix(c, edge_type)
  cand = odist.candidate_list(10, coords=c, edge_type=edge_type)
  for mode in ("best", "first"):
    got = LocalSearchB200TourTwoOpt(mode=mode, max_iterations=50, candidate_k=10).improve_batch(tours, ctx)
    want, _ = otwo.improve_batch(tours, D, otwo.resolve_candidates(cand, tours, 300), mode, 50)
    assert np.array_equal(got, want), mode


@pytest.mark.parametrize("edge_type", ["ATT", "GEO"])
def test_fused_ga_on_non_euclidean_types_matches_oracle(torch_mod, edge_type):
  from tsp_gpu_clean_b200.fused import FusedMemeticSolver, LocalSearchConfig
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  c = dist_coords(edge_type, 150, 77)
  ctx = ProblemContext(Problem.from_coordinates(c, edge_type=edge_type), seed=11)
  solver = FusedMemeticSolver(population_size=48, mutation_rate=0.1, elite_count=6, post_init=True,
                              local_search=LocalSearchConfig("best", 10, 12), chunk=5)
  best, stats = solver.evolve(ctx, list(range(150)), 20, patience=10**9)
  D = odist.distance_matrix(c, edge_type)
  cache = {}

  def provider(k):
    if k not in cache:
      cache[k] = odist.candidate_list(k, coords=c, edge_type=edge_type)
    return cache[k]

  cfg = oga.GAConfig(population_size=48, mutation_rate=0.1, nn_k=5, tournament_k=5,
                     local_search=oga.LocalSearchSpec("best", 10, 12), post_init=True, elite_count=6)
  rng = np.random.default_rng(11)
  obest, _, _, ostats, _ = oga.OracleGA(D, provider, cfg, rng).evolve(20, patience=10**9)
  assert np.array_equal(np.asarray(stats["convergence_history"]), np.asarray(ostats["convergence_history"]))
  assert np.array_equal(best, obest)
