"""Population operators on the B200 against the reference's golden outputs and the oracle."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import distances as odist
from oracle import ga_ops
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


def _ctx(coords, seed):
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  return ProblemContext(Problem.from_coordinates(coords), seed=seed)


@pytest.mark.parametrize("tag", ["a", "b", "c", "d"])
@pytest.mark.parametrize("resident", [False, True])
def test_operators_match_reference(torch_mod, golden, tag, resident):
  from tsp_gpu_clean_b200.strategies import (
    CrossoverB200PermPartiallyMapped,
    EvaluationB200Cost,
    MutationB200PermInversion,
    SelectionB200Tournament,
  )

  ops = golden("ops.npz")
  n, pop_size, seed = (int(v) for v in ops[f"{tag}_meta"])
  ctx = _ctx(ops[f"{tag}_coords"], seed)
  pop = ops[f"{tag}_pop"]
  ev = EvaluationB200Cost(return_gpu=resident)
  x = torch_mod.from_numpy(pop).cuda() if resident else pop
  fit = ev.assess_batch(x, ctx, return_gpu=resident).objectives
  assert np.array_equal(fit.cpu().numpy() if resident else fit, ops[f"{tag}_fit"])
  sel = SelectionB200Tournament(k=5, seed=1).select_batch(x, fit, pop_size, ctx)
  pmx = CrossoverB200PermPartiallyMapped(seed=1).crossover_batch(sel, ctx)
  inv = MutationB200PermInversion(seed=1).mutate_batch(pmx, float(ops[f"{tag}_rate"]), ctx)
  host = (lambda t: t.cpu().numpy()) if resident else (lambda t: t)
  assert np.array_equal(host(sel), ops[f"{tag}_sel"])
  assert np.array_equal(host(pmx), ops[f"{tag}_pmx"])
  assert np.array_equal(host(inv), ops[f"{tag}_inv"])
  assert ctx.rng.bit_generator.state["state"]["state"] % (1 << 63) == int(ops[f"{tag}_rng_state"][0])


def test_pmx_and_inversion_random_vs_oracle(torch_mod):
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  torch = torch_mod
  rng = np.random.default_rng(5)
  for n in (2, 3, 7, 64, 1000, 4099):
    pop = instances.random_tours(n, 33, n)
    pairs = ga_ops.sample_distinct_pairs(rng, 16, 0, n) if n >= 2 else None
    want = ga_ops.pmx_apply(pop, pairs)
    d = torch.from_numpy(pop).cuda()
    out = torch.empty_like(d)
    st = torch.zeros(33, dtype=torch.int32, device="cuda")
    f = torch.from_numpy(pairs[:, 0].copy()).cuda()
    s = torch.from_numpy(pairs[:, 1].copy()).cuda()
    native.call("tspb_pmx", ptr(d), 33, n, ptr(f), ptr(s), ptr(out), ptr(st), stream_handle())
    assert np.array_equal(out.cpu().numpy(), want), n
    u = rng.random(33)
    u[:5] = 0.0
    p1 = rng.integers(0, n, 33).astype(np.int32)
    p2 = rng.integers(0, n, 33).astype(np.int32)
    want = ga_ops.inversion_apply(pop, 0.5, u, p1, p2)
    d = torch.from_numpy(pop).cuda()
    du, d1, d2 = torch.from_numpy(u).cuda(), torch.from_numpy(p1).cuda(), torch.from_numpy(p2).cuda()
    native.call("tspb_inversion", ptr(d), 33, n, ptr(du), 0.5, ptr(d1), ptr(d2), stream_handle())
    assert np.array_equal(d.cpu().numpy(), want), n


def test_stable_rank_and_validation(torch_mod):
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  torch = torch_mod
  rng = np.random.default_rng(9)
  for count in (1, 5, 256, 1024, 3000):
    f = rng.integers(0, 20, count).astype(np.float64)  # heavy ties
    keep = max(1, count // 2)
    order = torch.empty(keep, dtype=torch.int32, device="cuda")
    df = torch.from_numpy(f).cuda()
    native.call("tspb_stable_rank", ptr(df), count, keep, ptr(order), stream_handle())
    z = np.zeros_like(f)
    assert np.array_equal(order.cpu().numpy(), np.lexsort(np.vstack([f, z, z]))[:keep])
  tours = instances.random_tours(50, 6, 3)
  tours[2, 5] = tours[2, 6]
  tours[4, 0] = 50
  bad = torch.empty(6, dtype=torch.int32, device="cuda")
  dt = torch.from_numpy(tours).cuda()
  native.call("tspb_validate_perm", ptr(dt), 6, 50, ptr(bad), stream_handle())
  assert bad.cpu().numpy().tolist() == [0, 0, 1, 0, 1, 0]


def test_euc2d_matrix_and_costs_match_reference(torch_mod, golden):
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  torch = torch_mod
  ops = golden("ops.npz")
  for coords, expect in ((ops["dist_coords"], ops["dist_matrix"]), (ops["big_coords"], None)):
    n = len(coords)
    d = torch.empty((n, n), dtype=torch.int32, device="cuda")
    dc = torch.from_numpy(np.ascontiguousarray(coords)).cuda()
    native.call("tspb_euc2d_matrix", ptr(dc), n, ptr(d), n, stream_handle())
    got = d.cpu().numpy()
    if expect is not None:
      assert np.array_equal(got, expect)
    else:
      assert hashlib.sha256(got.tobytes()).digest() == ops["big_digest"].tobytes()
  # tour costs from the matrix and from rebuilt FP64 distances agree with the oracle
  coords = ops["big_coords"]
  tours = instances.random_tours(len(coords), 8, 4)
  want = ga_ops.tour_cost(tours, odist.euc2d_matrix(coords))
  from tsp_gpu_clean_b200.strategies import EvaluationB200Cost

  ctx = _ctx(coords, 0)
  assert np.array_equal(EvaluationB200Cost().evaluate_batch(tours, ctx), want)
  assert np.array_equal(EvaluationB200Cost(max_matrix_dimension=100).evaluate_batch(tours, ctx), want)


def test_nn_init_matches_reference(torch_mod, golden):
  from tsp_gpu_clean_b200.strategies import InitializationB200TourNearestNeighbor

  g = golden("ga.npz")
  ctx = _ctx(g["c1_coords"], 42)
  pop = InitializationB200TourNearestNeighbor(k=5, seed=42).initialize(list(range(100)), 128, ctx)
  assert np.array_equal(pop, g["c1_init"])
  ctx3 = _ctx(g["c3_coords"], 42)
  pop3 = InitializationB200TourNearestNeighbor(k=5, seed=42, return_gpu=True).initialize(list(range(2000)), 512, ctx3)
  assert hashlib.sha256(pop3.cpu().numpy().astype(np.int32).tobytes()).hexdigest() == str(g["c3_init_digest"])


def test_nn_init_jobs_shared_memory_matches_workspace_kernel(torch_mod):
  """Nearest-neighbour rows built with the working arrays in shared memory equal the
  workspace kernel's, for jobs of different sizes and k (k = 0: uniform choices only)."""
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  torch = torch_mod
  specs = [(4, 3), (7, 0), (500, 5), (5000, 5), (1200, 12)]
  rows = 9
  rng = np.random.default_rng(3)
  tabs = [odist.candidate_list(k, coords=instances.uniform_instance(n, n)) if k else np.zeros((n, 0), np.int32)
          for n, k in specs]
  d_cand = [torch.from_numpy(np.ascontiguousarray(t).reshape(-1).copy() if t.size else np.zeros(1, np.int32)).cuda()
            for t in tabs]
  seeds = rng.integers(0, 2**62, (len(specs), rows), dtype=np.int64)
  d_seeds = torch.from_numpy(seeds).cuda()
  outs = [[torch.full((rows, n), -1, dtype=torch.int32, device="cuda") for n, _ in specs] for _ in range(2)]

  def jobs_for(which):
    h = (native.NNJob * len(specs))()
    for i, ((n, k), c) in enumerate(zip(specs, d_cand)):
      h[i].n, h[i].k, h[i].rows = n, k, rows
      h[i].cand = c.data_ptr()
      h[i].seeds = d_seeds.data_ptr() + i * rows * 8
      h[i].out = outs[which][i].data_ptr()
    return torch.frombuffer(bytearray(h), dtype=torch.uint8).cuda()

  j0, j1 = jobs_for(0), jobs_for(1)
  per = [rows * (2 * n + k) for n, k in specs]
  off = np.concatenate([[0], np.cumsum(per)[:-1]]).astype(np.int64)
  ws = torch.empty(int(sum(per)), dtype=torch.int32, device="cuda")
  d_off = torch.from_numpy(off).cuda()
  native.call("tspb_nn_init_jobs", ptr(j0), len(specs), rows, ptr(ws), ptr(d_off), stream_handle())
  native.call("tspb_nn_init_jobs_smem", ptr(j1), len(specs), rows, max(n for n, _ in specs),
              max(k for _, k in specs), stream_handle())
  for (n, _), a, b in zip(specs, outs[0], outs[1]):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    assert np.array_equal(a, b), n
    assert (np.sort(a, axis=1) == np.arange(n)).all()
  lib = native.load_library()
  assert lib.tspb_nn_init_jobs_smem(ptr(j1), 1, 1, 70000, 5, None) == native.TSPB_ERR_UNSUPPORTED
  assert lib.tspb_nn_init_jobs_smem(None, 1, 1, 100, 5, None) == native.TSPB_ERR_ARG


def test_check_free_counts_cached_memory_and_rejects_impossible_requests(torch_mod, monkeypatch):
  """check_free reads torch's allocator counters first (no driver call when its cached
  memory covers the request) and raises VRAMInsufficientError for more than the device has."""
  from tsp_gpu_clean_b200.device import check_free
  from tsp_gpu_clean_b200.errors import VRAMInsufficientError

  block = torch_mod.empty(64 << 20, dtype=torch_mod.uint8, device="cuda")
  del block  # the 64 MiB stay reserved by the caching allocator
  calls = []
  real = torch_mod.cuda.mem_get_info
  monkeypatch.setattr(torch_mod.cuda, "mem_get_info", lambda *a: calls.append(1) or real(*a))
  check_free(32 << 20, "a request the cache covers")
  assert calls == []
  with pytest.raises(VRAMInsufficientError):
    check_free(1 << 50, "a petabyte")
  assert calls == [1]


def test_euc2d_rounding_boundaries_match_the_reference_formula(torch_mod):
  """Distances on and around half-integers (where a float root alone could round the other
  way), at several scales, equal NumPy's `int64(sqrt(dx*dx + dy*dy) + 0.5)`."""
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  torch = torch_mod
  rng = np.random.default_rng(77)
  pts = [(0.0, 0.0)]
  for m in (0, 1, 2, 7, 100, 1414, 4095, 30000, 65534, 200000, 1 << 20):
    for eps in (0.0, 1e-12, -1e-12, 1e-9, -1e-9, 1e-6, -1e-6, 1e-4, -1e-4, 3e-3, -3e-3):
      pts.append((0.0, m + 0.5 + eps))
      a = rng.uniform(0, np.pi / 2)
      r = m + 0.5 + eps
      pts.append((r * np.cos(a), r * np.sin(a)))
  # Pythagorean-style exact half-integers: (1.5, 2) -> 2.5, scaled
  for k in (1, 3, 101, 1001, 20001):
    pts.append((1.5 * k, 2.0 * k))
  pts += [tuple(p) for p in rng.uniform(0, 1000, (200, 2))]
  coords = np.asarray(pts, dtype=np.float64)
  n = len(coords)
  d = torch.empty((n, n), dtype=torch.int32, device="cuda")
  dc = torch.from_numpy(np.ascontiguousarray(coords)).cuda()
  native.call("tspb_euc2d_matrix", ptr(dc), n, ptr(d), n, stream_handle())
  assert np.array_equal(d.cpu().numpy(), odist.euc2d_matrix(coords))
