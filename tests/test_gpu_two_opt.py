"""2-opt on the B200 through the C ABI, bit-exact against the oracle and the golden vectors.

Covers every reference 2-opt parity case (`test_unit_two_opt_vectorized_scan.py`,
`test_unit_two_opt_boundaries.py` of the reference): modes best/first/multi_move/batch,
exhaustive and k-NN neighbourhoods, tie-heavy integer lattices, duplicated candidates,
short tours, zero iterations, untouched inputs, and tours run to a local optimum on
the 1000-city clustered instance with the oracle's pass and pair counts.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import iter_two_opt_cases
from oracle import distances as odist
from oracle import two_opt as otwo
from tsp_gpu_clean_b200 import instances

pytestmark = pytest.mark.gpu


class CoordDist:
  """EUC_2D lookups `D[a, c]` computed on demand (no n x n matrix on the host)."""

  def __init__(self, coords):
    self.coords = np.asarray(coords, dtype=np.float64)
    self.shape = (len(coords), len(coords))

  def __getitem__(self, idx):
    a, c = idx
    diff = self.coords[np.asarray(a)] - self.coords[np.asarray(c)]
    return (np.sqrt(diff[..., 0] * diff[..., 0] + diff[..., 1] * diff[..., 1]) + 0.5).astype(np.int64).astype(np.int32)


@pytest.fixture(scope="module")
def b200():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext
  from tsp_gpu_clean_b200.strategies.local_search import LocalSearchB200TourTwoOpt

  return Problem, ProblemContext, LocalSearchB200TourTwoOpt


def _ctx(b200, D=None, coords=None, cand=None, k=None):
  Problem, ProblemContext, _ = b200
  prob = Problem.from_coordinates(coords) if coords is not None else Problem.from_matrix(D)
  cache = {k: cand} if cand is not None else None
  return ProblemContext(prob, seed=0, candidate_cache=cache)


def test_golden_small_cases(b200, golden):
  data = golden("two_opt_small.npz")
  LS = b200[2]
  for c, n, k, mode, iters, D, cand, tin, tout in iter_two_opt_cases(data):
    coords = data.get(f"c{c}_coords")
    ctx = _ctx(b200, D=D if coords is None else None, coords=coords, cand=cand, k=k)
    for m in ([mode, "batch"] if mode == "best" else [mode]):
      for kern in (("scan", "scan_unpacked", "cached") if k is not None and m != "multi_move" else ("scan",)):
        before = tin.copy()
        ls = LS(max_iterations=iters, mode=m, candidate_k=k)
        ls.kernel = kern
        got = ls.improve_batch(tin, ctx)
        assert np.array_equal(tin, before), "input mutated"
        assert np.array_equal(got, tout), f"case {c}: n={n} k={k} mode={m} iters={iters} kernel={kern}"


@pytest.mark.parametrize("kern", ["scan", "scan_unpacked", "cached"])
@pytest.mark.parametrize("mode", ["best", "first"])
def test_golden_c2_local_optimum_with_counts(b200, golden, mode, kern):
  data = golden("two_opt_c2.npz")
  ctx = _ctx(b200, coords=data["coords"], cand=data["cand20"], k=20)
  ls = b200[2](max_iterations=10**9, mode=mode, candidate_k=20)
  ls.kernel = kern
  got = ls.improve_batch(data["tours_in"], ctx)
  assert np.array_equal(got, data[f"{mode}_out"])
  assert np.array_equal(ls.last_stats[:, 0], data[f"{mode}_stats"][:, 0]), "passes"
  assert np.array_equal(ls.last_stats[:, 1], data[f"{mode}_stats"][:, 1]), "oracle-equivalent pairs"


@pytest.mark.parametrize("kern", ["scan", "cached"])
@pytest.mark.parametrize("threads", [64, 128, 256, 512])
def test_kernel_block_sizes(b200, threads, kern):
  coords = instances.clustered_instance(700, 12, 30.0, 13)
  tours = instances.random_tours(700, 6, 14)
  ctx = _ctx(b200, coords=coords)
  D = odist.euc2d_matrix(coords)
  cand = ctx.get_cpu_candidate_list(20)
  for mode in ("best", "first"):
    ls = b200[2](max_iterations=10**9, mode=mode, candidate_k=20, threads_per_block=threads)
    ls.kernel = kern
    got = ls.improve_batch(tours, ctx)
    want, st = otwo.improve_batch(tours, D, cand, mode, 10**9)
    assert np.array_equal(got, want)
    assert np.array_equal(ls.last_stats[:, :3], st)


@pytest.mark.parametrize("mode", ["best", "first", "multi_move"])
@pytest.mark.parametrize("iters", [1, 10, 10**9])
def test_random_tours_vs_oracle(b200, mode, iters):
  coords = instances.clustered_instance(300, 10, 30.0, 11)
  tours = instances.random_tours(300, 12, 12)
  ctx = _ctx(b200, coords=coords)
  D = odist.euc2d_matrix(coords)
  cand = ctx.get_cpu_candidate_list(20)
  ls = b200[2](max_iterations=iters, mode=mode, candidate_k=20)
  got = ls.improve_batch(tours, ctx)
  want, st = otwo.improve_batch(tours, D, cand, mode, iters)
  assert np.array_equal(got, want)
  assert np.array_equal(ls.last_stats[:, :3], st)


@pytest.mark.parametrize("mode", ["best", "first", "multi_move"])
def test_exhaustive_vs_oracle(b200, mode):
  coords = instances.uniform_instance(120, 3)
  tours = instances.random_tours(120, 6, 4)
  ctx = _ctx(b200, coords=coords)
  D = odist.euc2d_matrix(coords)
  ls = b200[2](max_iterations=10**9, mode=mode, candidate_k=None)
  got = ls.improve_batch(tours, ctx)
  want, st = otwo.improve_batch(tours, D, None, mode, 10**9)
  assert np.array_equal(got, want)
  assert np.array_equal(ls.last_stats[:, :3], st)


def test_exhaustive_first_pair_count_spans_cpu_blocks(b200):
  # n = 800 has 318,801 pairs per scan: more than one 2^18 CPU block.
  coords = instances.uniform_instance(800, 21)
  tours = instances.random_tours(800, 2, 22)
  ctx = _ctx(b200, coords=coords)
  D = odist.euc2d_matrix(coords)
  ls = b200[2](max_iterations=40, mode="first", candidate_k=None)
  got = ls.improve_batch(tours, ctx)
  want, st = otwo.improve_batch(tours, D, None, "first", 40)
  assert np.array_equal(got, want)
  assert np.array_equal(ls.last_stats[:, :3], st)


@pytest.mark.parametrize("mode", ["best", "first", "multi_move"])
def test_fp64_rebuilt_distances_match_matrix(b200, mode):
  coords = instances.uniform_instance(500, 31)
  tours = instances.random_tours(500, 8, 32)
  ctx = _ctx(b200, coords=coords)
  LS = b200[2]
  a = LS(max_iterations=10**9, mode=mode, candidate_k=20).improve_batch(tours, ctx)
  b = LS(max_iterations=10**9, mode=mode, candidate_k=20, max_matrix_dimension=100).improve_batch(tours, ctx)
  assert np.array_equal(a, b)


def test_large_tour_uses_workspace_arrays(b200):
  # 20,000 cities: tour/pos/edge do not fit in shared memory and live in the workspace.
  coords = instances.uniform_instance(20000, 41)
  tours = instances.random_tours(20000, 2, 42)
  ctx = _ctx(b200, coords=coords)
  ls = b200[2](max_iterations=30, mode="best", candidate_k=8, max_matrix_dimension=1000)
  got = ls.improve_batch(tours, ctx)
  want, st = otwo.improve_batch(tours, CoordDist(coords), ctx.get_cpu_candidate_list(8), "best", 30)
  assert np.array_equal(got, want)
  assert np.array_equal(ls.last_stats[:, :3], st)


def test_contracts(b200):
  LS = b200[2]
  coords = instances.uniform_instance(30, 1)
  ctx = _ctx(b200, coords=coords)
  t = instances.random_tours(30, 3, 2)
  assert np.array_equal(LS(max_iterations=0).improve_batch(t, ctx), t)
  short = np.array([[2, 0, 1], [0, 1, 2]], dtype=np.int32)
  assert np.array_equal(LS(max_iterations=5).improve_batch(short, ctx), short)
  one = LS(max_iterations=5, candidate_k=5).improve_batch(t[0], ctx)
  assert one.shape == (30,)
  with pytest.raises(ValueError):
    LS(mode="naive")
  with pytest.raises(ValueError):
    LS(max_iterations=-1)
  bad = t.copy()
  bad[1, 3] = bad[1, 4]
  from tsp_gpu_clean_b200.errors import NotPermutationError

  with pytest.raises(NotPermutationError):
    LS(max_iterations=5, candidate_k=5).improve_batch(bad, ctx)


def test_device_resident_roundtrip(b200):
  import torch

  coords = instances.uniform_instance(200, 5)
  tours = instances.random_tours(200, 8, 6)
  ctx = _ctx(b200, coords=coords)
  LS = b200[2]
  host = LS(max_iterations=50, mode="best", candidate_k=20).improve_batch(tours, ctx)
  dev_in = torch.from_numpy(tours).cuda()
  dev = LS(max_iterations=50, mode="best", candidate_k=20).improve_batch(dev_in, ctx)
  assert dev.is_cuda
  assert np.array_equal(dev.cpu().numpy(), host)
  assert np.array_equal(dev_in.cpu().numpy(), tours)


_LAYOUT_ORACLE: dict = {}


@pytest.mark.parametrize("mode", ["best", "first"])
@pytest.mark.parametrize("k", [20, 12, 10, 7])
@pytest.mark.parametrize("threads", [128, 512])
def test_table_layouts_agree(b200, mode, k, threads):
  """Plain candidates, packed words, and packed words read in row groups (k % 4 == 0) give
  the same tours and the same pass/pair/move counts, equal to the oracle's."""
  import torch

  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import operands_for, ptr, stream_handle

  n, T = 250, 16
  coords = instances.clustered_instance(n, 12, 30.0, 31)
  tours = instances.random_tours(n, T, 32)
  ctx = _ctx(b200, coords=coords)
  ops = operands_for(ctx)
  dist, stride, _ = ops.distance_args(n, None)
  tabs = ops.candidates(k, ctx.get_cpu_candidate_list(k), n, None)
  assert tabs.packed is not None
  lib = native.load_library()
  outs = []
  for packed in (None, tabs.packed):
    work = torch.from_numpy(tours).cuda()
    stats = torch.zeros((T, 4), dtype=torch.int64, device="cuda")
    status = torch.zeros(T, dtype=torch.int32, device="cuda")
    rc = lib.tspb_two_opt(ptr(work), T, n, ptr(dist), stride, None, ptr(tabs.cand), ptr(tabs.cand_dist), None, None,
                          ptr(packed), tabs.k, native.MODE_CODES[mode], 10**9, threads, ptr(stats), ptr(status), None,
                          0, stream_handle())
    native.check("tspb_two_opt", rc)
    assert int(status.max().item()) == 0
    outs.append((work.cpu().numpy(), stats.cpu().numpy()))
  assert np.array_equal(outs[0][0], outs[1][0])
  # passes, oracle-equivalent pairs and moves agree; the count of gains actually computed
  # (column 3) depends on the round width in first mode (a round finishes before stopping)
  assert np.array_equal(outs[0][1][:, :3], outs[1][1][:, :3])
  key = (mode, k)
  if key not in _LAYOUT_ORACLE:
    _LAYOUT_ORACLE[key] = otwo.improve_batch(tours, odist.euc2d_matrix(coords), ctx.get_cpu_candidate_list(k), mode,
                                             10**9)
  want, st = _LAYOUT_ORACLE[key]
  assert np.array_equal(outs[1][0], want)
  assert np.array_equal(outs[1][1][:, :3], st)


@pytest.mark.parametrize("k,threads", [(20, 128), (8, 256), (7, 64), (12, 512)])
@pytest.mark.parametrize("max_iter", [10**9, 37])
def test_first_mode_incremental_restart_matches_full_rescan(b200, k, threads, max_iter):
  """First mode restarting from the affected entries and the move's row gives the tours
  and pass/pair/move counts of the full rescan from entry 0 and of the oracle, on a
  clustered, a uniform and a tie-heavy lattice instance, with grouped (k % 4 == 0) and
  plain packed tables."""
  import torch

  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import operands_for, ptr, stream_handle

  side = 17
  lattice = np.array([[5.0 * x, 5.0 * y] for x in range(side) for y in range(side)])
  for coords in (instances.clustered_instance(300, 10, 30.0, 71), instances.uniform_instance(180, 72), lattice):
    n, T = len(coords), 12
    tours = instances.random_tours(n, T, 73 + n)
    ctx = _ctx(b200, coords=coords)
    ops = operands_for(ctx)
    dist, stride, _ = ops.distance_args(n, None)
    tabs = ops.candidates(k, ctx.get_cpu_candidate_list(k), n, None)
    lib = native.load_library()
    outs = []
    for rev in (False, True):
      work = torch.from_numpy(tours).cuda()
      stats = torch.zeros((T, 4), dtype=torch.int64, device="cuda")
      status = torch.zeros(T, dtype=torch.int32, device="cuda")
      rc = lib.tspb_two_opt(ptr(work), T, n, ptr(dist), stride, None, ptr(tabs.cand), ptr(tabs.cand_dist),
                            ptr(tabs.rev_off) if rev else None, ptr(tabs.rev_idx) if rev else None, ptr(tabs.packed),
                            tabs.k, native.MODE_CODES["first"], max_iter, threads, ptr(stats), ptr(status), None, 0,
                            stream_handle())
      native.check("tspb_two_opt", rc)
      assert int(status.max().item()) == 0
      outs.append((work.cpu().numpy(), stats.cpu().numpy()))
    assert np.array_equal(outs[0][0], outs[1][0]), n
    assert np.array_equal(outs[0][1][:, :3], outs[1][1][:, :3]), n
    want, st = otwo.improve_batch(tours, odist.euc2d_matrix(coords), ctx.get_cpu_candidate_list(k), "first", max_iter)
    assert np.array_equal(outs[1][0], want), n
    assert np.array_equal(outs[1][1][:, :3], st), n


@pytest.mark.parametrize("threads", [128, 256])
@pytest.mark.parametrize("rev", [False, True])
def test_uncounted_launch_equals_counted_launch_and_oracle(b200, threads, rev):
  """A launch without a stats buffer runs the scan without first mode's per-row pair-count
  bookkeeping (and with 16n instead of 20n bytes of shared memory per tour); its tours must
  equal those of the counted launch and of the oracle, in both modes and table layouts."""
  import torch

  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import operands_for, ptr, stream_handle

  coords = instances.clustered_instance(500, 12, 30.0, 81)
  n, T = 500, 16
  tours = instances.random_tours(n, T, 82)
  ctx = _ctx(b200, coords=coords)
  ops = operands_for(ctx)
  dist, stride, _ = ops.distance_args(n, None)
  D = odist.euc2d_matrix(coords)
  lib = native.load_library()
  for k in (20, 7):  # grouped (k % 4 == 0) and plain packed words
    tabs = ops.candidates(k, ctx.get_cpu_candidate_list(k), n, None)
    for mode in ("best", "first"):
      outs = []
      for counted in (True, False):
        work = torch.from_numpy(tours).cuda()
        stats = torch.zeros((T, 4), dtype=torch.int64, device="cuda") if counted else None
        status = torch.zeros(T, dtype=torch.int32, device="cuda")
        use_rev = rev and mode == "first"
        rc = lib.tspb_two_opt(ptr(work), T, n, ptr(dist), stride, None, ptr(tabs.cand), ptr(tabs.cand_dist),
                              ptr(tabs.rev_off) if use_rev else None, ptr(tabs.rev_idx) if use_rev else None,
                              ptr(tabs.packed), tabs.k, native.MODE_CODES[mode], 10**9, threads, ptr(stats),
                              ptr(status), None, 0, stream_handle())
        native.check("tspb_two_opt", rc)
        assert int(status.max().item()) == 0
        outs.append(work.cpu().numpy())
      want, _ = otwo.improve_batch(tours, D, ctx.get_cpu_candidate_list(k), mode, 10**9)
      assert np.array_equal(outs[0], want), (k, mode)
      assert np.array_equal(outs[1], want), (k, mode)


def test_public_call_without_stats_equals_golden_c2(b200, golden):
  data = golden("two_opt_c2.npz")
  ctx = _ctx(b200, coords=data["coords"], cand=data["cand20"], k=20)
  for mode in ("best", "first"):
    ls = b200[2](max_iterations=10**9, mode=mode, candidate_k=20, threads_per_block=128)
    ls.collect_stats = False
    got = ls.improve_batch(data["tours_in"], ctx)
    assert ls.last_stats is None
    assert np.array_equal(got, data[f"{mode}_out"])
