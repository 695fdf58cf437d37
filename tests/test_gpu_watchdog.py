"""The device watchdog of the local-search kernels, made to run out on purpose.

`tspb_set_watchdog_cycles` lowers the cycle budget every later launch is given; with a
budget of one SM cycle every tour stops at its first pass check. The kernels must then
report TSPB_ERR_BUDGET per tour, leave each tour a valid permutation no longer than the
input, and leave the CUDA context usable: a launch with the default budget afterwards
refines the same tours exactly as the oracle does. No kernel is made to hang or fault:
the budget is an ordinary argument that the pass loop compares against clock64().
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import distances as odist
from oracle import two_opt as oracle_two_opt
from tsp_gpu_clean_b200 import instances

pytestmark = pytest.mark.gpu

N, TOURS, K = 300, 12, 20


@pytest.fixture(scope="module")
def env():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import operands_for
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  coords = instances.clustered_instance(N, 8, 30.0, 515)
  ctx = ProblemContext(Problem.from_coordinates(coords), seed=0)
  ops = operands_for(ctx)
  dist, stride, _ = ops.distance_args(N)
  tabs = ops.candidates(K, ctx.get_cpu_candidate_list(K), N)
  torch.cuda.synchronize()
  return {"torch": torch, "lib": native.load_library(), "native": native, "coords": coords, "ctx": ctx,
          "dist": dist, "stride": stride, "tabs": tabs, "D": odist.euc2d_matrix(coords),
          "cand": ctx.get_cpu_candidate_list(K)}


class tiny_budget:
  """Watchdog budget of one cycle inside the block, the default restored on exit."""

  def __init__(self, lib):
    self.lib = lib

  def __enter__(self):
    self.lib.tspb_set_watchdog_cycles(1)
    return self

  def __exit__(self, *exc):
    self.lib.tspb_set_watchdog_cycles(0)


def _lengths(D, tours):
  return np.array([int(D[t, np.roll(t, -1)].sum()) for t in tours])


def _two_opt(env, tours, mode, variant):
  torch, lib = env["torch"], env["lib"]
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  tabs = env["tabs"]
  d = torch.from_numpy(tours).cuda()
  num, n = tours.shape
  stats = torch.zeros((num, 4), dtype=torch.int64, device="cuda")
  status = torch.zeros(num, dtype=torch.int32, device="cuda")
  code = env["native"].MODE_CODES[mode]
  cand = cand_dist = rev_off = rev_idx = packed = None
  k = 0
  if variant != "exhaustive":
    cand, cand_dist, k = tabs.cand, tabs.cand_dist, tabs.k
  if variant == "scan":
    packed = tabs.packed
  if variant == "cached" or (variant == "scan" and mode == "first"):
    rev_off, rev_idx = tabs.rev_off, tabs.rev_idx
  ws_bytes = lib.tspb_two_opt_workspace_bytes(num, n, k, code, 128)
  ws = torch.empty(max(int(ws_bytes), 1), dtype=torch.uint8, device="cuda")
  rc = lib.tspb_two_opt(ptr(d), num, n, ptr(env["dist"]), env["stride"], None, ptr(cand), ptr(cand_dist), ptr(rev_off),
                        ptr(rev_idx), ptr(packed), k, code, 10**9, 128, ptr(stats), ptr(status), ptr(ws), int(ws_bytes),
                        stream_handle())
  assert rc == 0
  torch.cuda.synchronize()
  return d.cpu().numpy(), status.cpu().numpy(), stats.cpu().numpy()


@pytest.mark.parametrize("variant,mode", [("scan", "best"), ("scan", "first"), ("cached", "best"),
                                          ("cached", "first"), ("exhaustive", "best"), ("scan", "multi_move")])
def test_two_opt_watchdog_expires_with_tours_intact(env, variant, mode):
  lib, native = env["lib"], env["native"]
  tours = instances.random_tours(N, TOURS, 516)
  with tiny_budget(lib):
    out, status, stats = _two_opt(env, tours, mode, variant)
  assert (status == native.TSPB_ERR_BUDGET).all(), status
  for t in out:
    assert np.array_equal(np.sort(t), np.arange(N)), "a stopped tour must stay a permutation"
  assert (_lengths(env["D"], out) <= _lengths(env["D"], tours)).all()
  assert (stats[:, 0] <= 1).all(), "one cycle allows no more than the pass in flight"
  # the context is still usable and the default budget is back: full refinement = oracle
  cand = None if variant == "exhaustive" else env["cand"]
  got, status2, _ = _two_opt(env, tours, mode, variant)
  assert not status2.any()
  want, _ = oracle_two_opt.improve_batch(tours, env["D"], cand, mode, 10**9)
  assert np.array_equal(got, want)


def test_or_opt_and_three_opt_watchdog_expire(env):
  torch, lib, native = env["torch"], env["lib"], env["native"]
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  tabs = env["tabs"]
  tours = instances.random_tours(N, 4, 517)
  d = torch.from_numpy(tours).cuda()
  status = torch.zeros(4, dtype=torch.int32, device="cuda")
  stats = torch.zeros((4, 3), dtype=torch.int64, device="cuda")
  with tiny_budget(lib):
    rc = lib.tspb_or_opt(ptr(d), 4, N, ptr(env["dist"]), env["stride"], None, ptr(tabs.cand), ptr(tabs.cand_dist),
                         ptr(tabs.packed), tabs.k, 3, 10**6, 128, ptr(status), ptr(stats), stream_handle())
    assert rc == 0
    torch.cuda.synchronize()
  assert (status.cpu().numpy() == native.TSPB_ERR_BUDGET).all()
  for t in d.cpu().numpy():
    assert np.array_equal(np.sort(t), np.arange(N))

  import ctypes

  n3 = 60
  c3 = instances.uniform_instance(n3, 518)
  D3 = odist.euc2d_matrix(c3)
  d3 = torch.from_numpy(D3.astype(np.int32)).cuda()
  t3 = torch.from_numpy(instances.random_tours(n3, 3, 519)).cuda()
  need = ctypes.c_size_t(0)
  assert lib.tspb_three_opt_workspace_bytes(n3, 3, ctypes.byref(need)) == 0
  ws = torch.empty(max(int(need.value), 1), dtype=torch.uint8, device="cuda")
  st3 = torch.zeros(3, dtype=torch.int32, device="cuda")
  s3 = torch.zeros((3, 3), dtype=torch.int64, device="cuda")
  with tiny_budget(lib):
    rc = lib.tspb_three_opt(ptr(t3), 3, n3, ptr(d3), n3, None, 10**6, 256, ptr(ws), int(need.value), ptr(st3), ptr(s3),
                            stream_handle())
    assert rc == 0
    torch.cuda.synchronize()
  assert (st3.cpu().numpy() == native.TSPB_ERR_BUDGET).all()
  for t in t3.cpu().numpy():
    assert np.array_equal(np.sort(t), np.arange(n3))
