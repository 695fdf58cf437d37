"""The context's k-NN table built on the device (`device.candidate_list`) equals the
reference's host table (`compute_candidate_list`, restated and pinned in the oracle),
boundary ties included."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import distances as odist
from tests.golden.make_golden import dist_coords
from tsp_gpu_clean_b200 import instances

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  return torch


def _cases():
  side = 40
  lattice = np.array([[3.0 * x, 3.0 * y] for x in range(side) for y in range(side)])
  rng = np.random.default_rng(4)
  m = rng.integers(1, 12, (300, 300))
  explicit = np.triu(m, 1) + np.triu(m, 1).T
  return [
    ("uniform1002", instances.uniform_instance(1002, 1002), "EUC_2D", None),
    ("clustered2000", instances.clustered_instance(2000, 20, 30.0, 9), "EUC_2D", None),
    ("lattice1600", lattice, "EUC_2D", None),
    ("att500", dist_coords("ATT", 500, 3), "ATT", None),
    ("geo400", dist_coords("GEO", 400, 5), "GEO", None),
    ("explicit300", None, "EXPLICIT", explicit.astype(np.int32)),
    ("tiny6", instances.uniform_instance(6, 2), "EUC_2D", None),
  ]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_device_knn_equals_reference_procedure(torch_mod, case):
  from tsp_gpu_clean_b200.device import candidate_list
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  name, coords, edge_type, matrix = case
  if matrix is not None:
    prob = Problem.from_matrix(matrix)
  else:
    prob = Problem.from_coordinates(coords, edge_type=edge_type)
  for k in (5, 20):
    ctx = ProblemContext(prob, seed=0)
    got = candidate_list(ctx, k)
    if matrix is not None:
      want = odist.candidate_list(k, distances=matrix)
    else:
      want = odist.candidate_list(k, coords=coords, edge_type=edge_type)
    assert np.array_equal(got, want), (name, k)
    assert ctx.get_cpu_candidate_list(k) is got  # stored in the context's cache


def test_device_knn_with_coordinate_distances(torch_mod):
  """Above the context's matrix threshold the table is computed from rebuilt distances."""
  from tsp_gpu_clean_b200.device import candidate_list
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  c = instances.clustered_instance(3000, 12, 40.0, 17)
  ctx = ProblemContext(Problem.from_coordinates(c), seed=0, max_matrix_dimension=1000)
  assert np.array_equal(candidate_list(ctx, 16), odist.candidate_list(16, coords=c))
