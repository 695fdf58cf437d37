"""The allocation-free multi_move entry point against the workspace entry point.

`tspb_two_opt_multi_move_static` serves callers that cannot allocate device memory (a
host callback, an allocator-free real-time loop, a plugin host that hands over only its
input and output buffers): it runs the multi_move 2-opt on a fixed scratch array inside
libtspb.so. This file is collected last so that a failure here never hides the results
of the other GPU tests; it also passes when run alone in a fresh process.
"""

from __future__ import annotations

import numpy as np
import pytest

from tsp_gpu_clean_b200 import instances

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import operands_for, ptr, stream_handle
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  coords = instances.clustered_instance(400, 10, 30.0, 91)
  ctx = ProblemContext(Problem.from_coordinates(coords), seed=0)
  ops = operands_for(ctx)
  dist, stride, _ = ops.distance_args(400)
  tabs = ops.candidates(20, ctx.get_cpu_candidate_list(20), 400)
  torch.cuda.synchronize()
  return torch, native.load_library(), ptr, stream_handle, dist, stride, tabs


def _run_workspace(env, tours, iters):
  torch, lib, ptr, sh, dist, stride, tabs = env
  t = torch.from_numpy(tours).cuda()
  num, n = tours.shape
  stats = torch.zeros((num, 4), dtype=torch.int64, device="cuda")
  status = torch.zeros(num, dtype=torch.int32, device="cuda")
  ws_bytes = lib.tspb_two_opt_workspace_bytes(num, n, tabs.k, 2, 256)
  ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
  rc = lib.tspb_two_opt(ptr(t), num, n, ptr(dist), stride, None, ptr(tabs.cand), ptr(tabs.cand_dist), None, None, None,
                        tabs.k, 2, iters, 256, ptr(stats), ptr(status), ptr(ws), ws_bytes, sh())
  assert rc == 0
  torch.cuda.synchronize()
  return t.cpu().numpy(), stats.cpu().numpy(), status.cpu().numpy()


def _run_static(env, tours, iters):
  torch, lib, ptr, sh, dist, stride, tabs = env
  t = torch.from_numpy(tours).cuda()
  num, n = tours.shape
  stats = torch.zeros((num, 4), dtype=torch.int64, device="cuda")
  status = torch.zeros(num, dtype=torch.int32, device="cuda")
  rc = lib.tspb_two_opt_multi_move_static(ptr(t), num, n, ptr(dist), stride, None, ptr(tabs.cand), ptr(tabs.cand_dist),
                                          tabs.k, iters, 256, ptr(stats), ptr(status), sh())
  assert rc == 0
  torch.cuda.synchronize()
  return t.cpu().numpy(), stats.cpu().numpy(), status.cpu().numpy()


def test_static_scratch_matches_workspace_entry_point_twice_in_a_row(env):
  tours = instances.random_tours(400, 24, 92)
  want, want_stats, want_status = _run_workspace(env, tours, 10**6)
  assert not want_status.any()
  for call in range(2):  # the scratch keeps the previous call's contents
    got, got_stats, got_status = _run_static(env, tours, 10**6)
    assert not got_status.any(), f"call {call}"
    assert np.array_equal(got, want), f"call {call}: tours differ"
    assert np.array_equal(got_stats, want_stats), f"call {call}: stats differ"
  # a different batch after the first two still matches (no stale state leaks in)
  tours2 = instances.random_tours(400, 7, 93)
  assert np.array_equal(_run_static(env, tours2, 3)[0], _run_workspace(env, tours2, 3)[0])


def test_static_scratch_rejects_shapes_beyond_its_size(env):
  torch, lib, ptr, sh, dist, stride, tabs = env
  # n = 1000, k = 20 needs 256 KiB per tour; 200 tours exceed 32 MiB
  assert lib.tspb_two_opt_workspace_bytes(200, 1000, 20, 2, 256) > (32 << 20)
  rc = lib.tspb_two_opt_multi_move_static(None, 200, 1000, ptr(dist), stride, None, ptr(tabs.cand), None, 20, 5, 256,
                                          None, None, sh())
  assert rc == 6  # TSPB_ERR_WORKSPACE, before any launch


def _pair(lib, ptr, sh, torch, tours, dist, stride, cand, cand_dist, k, iters, coords=None):
  """(workspace entry point, static entry point) outputs of one multi_move batch."""
  num, n = tours.shape
  outs = []
  for static in (False, True):
    t = torch.from_numpy(tours).cuda()
    stats = torch.zeros((num, 4), dtype=torch.int64, device="cuda")
    status = torch.zeros(num, dtype=torch.int32, device="cuda")
    if static:
      rc = lib.tspb_two_opt_multi_move_static(ptr(t), num, n, ptr(dist), stride, ptr(coords), ptr(cand),
                                              ptr(cand_dist), k, iters, 256, ptr(stats), ptr(status), sh())
    else:
      ws_bytes = lib.tspb_two_opt_workspace_bytes(num, n, k if cand is not None else 0, 2, 256)
      ws = torch.empty(max(int(ws_bytes), 1), dtype=torch.uint8, device="cuda")
      rc = lib.tspb_two_opt(ptr(t), num, n, ptr(dist), stride, ptr(coords), ptr(cand), ptr(cand_dist), None, None,
                            None, k, 2, iters, 256, ptr(stats), ptr(status), ptr(ws), int(ws_bytes), sh())
    assert rc == 0
    torch.cuda.synchronize()
    assert not status.cpu().numpy().any()
    outs.append((t.cpu().numpy(), stats.cpu().numpy()))
  return outs


def test_static_scratch_exhaustive_path(env):
  """Without candidates every (i, j) pair is a key: n^2/2 keys per tour in the scratch."""
  torch, lib, ptr, sh, dist, stride, tabs = env
  tours = instances.random_tours(400, 20, 94)
  assert lib.tspb_two_opt_workspace_bytes(20, 400, 0, 2, 256) <= (32 << 20)
  for _ in range(2):
    (want, want_stats), (got, got_stats) = _pair(lib, ptr, sh, torch, tours, dist, stride, None, None, 0, 10**6)
    assert np.array_equal(got, want)
    assert np.array_equal(got_stats, want_stats)


def test_static_scratch_spill_path(env):
  """A tour too long for shared memory keeps its arrays at the start of its scratch slice
  and its keys after them (a non-zero key offset)."""
  import torch as _torch

  torch, lib, ptr, sh, _, _, _ = env
  from tsp_gpu_clean_b200.device import operands_for
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  n = 20000  # 12 n bytes of tour arrays exceed the opt-in shared memory of a B200 CTA
  optin = _torch.cuda.get_device_properties(0).shared_memory_per_block_optin
  assert 12 * n > optin
  coords = instances.clustered_instance(n, 40, 30.0, 95)
  ctx = ProblemContext(Problem.from_coordinates(coords), seed=0)
  ops = operands_for(ctx)
  dist, stride, coords = ops.distance_args(n)  # above 10,000 cities: rebuilt from FP64 coordinates
  tabs = ops.candidates(8, ctx.get_cpu_candidate_list(8), n)
  tours = instances.random_tours(n, 3, 96)
  assert lib.tspb_two_opt_workspace_bytes(3, n, tabs.k, 2, 256) <= (32 << 20)
  for _ in range(2):
    (want, want_stats), (got, got_stats) = _pair(lib, ptr, sh, torch, tours, dist, stride, tabs.cand, tabs.cand_dist,
                                                 tabs.k, 3, coords)
    assert np.array_equal(got, want)
    assert np.array_equal(got_stats, want_stats)
  del dist, coords, tabs, ops, ctx
