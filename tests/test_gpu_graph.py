"""CUDA graphs of the library's launches (`tspb_graph_*`), the GA engines' replay path."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle import distances as odist
from tsp_gpu_clean_b200 import instances

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  from tsp_gpu_clean_b200 import native

  return native.load_library()


def test_replay_reads_the_buffers_at_replay_time(lib):
  """A captured tour-cost launch recomputes the costs of whatever the tour buffer holds
  when the graph replays, and writes them to the captured output buffer."""
  import torch

  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.batch import capture_graph
  from tsp_gpu_clean_b200.device import ptr, stream_handle

  n, num = 60, 8
  coords = instances.uniform_instance(n, 5)
  D = odist.euc2d_matrix(coords).astype(np.int32)
  d_D = torch.from_numpy(D).cuda()
  tours = instances.random_tours(n, num, 6)
  d_t = torch.from_numpy(tours.astype(np.int32)).cuda()
  costs = torch.zeros(num, dtype=torch.float64, device="cuda")

  def enqueue():
    native.call("tspb_tour_cost", ptr(d_t), num, n, ptr(d_D), n, None, 1, ptr(costs), stream_handle())

  g = capture_graph(enqueue)
  torch.cuda.synchronize()
  assert float(costs.abs().sum()) == 0.0  # capture records; it does not run
  for seed in (7, 8, 9):
    fresh = instances.random_tours(n, num, seed)
    d_t.copy_(torch.from_numpy(fresh.astype(np.int32)))
    g.replay()
    torch.cuda.synchronize()
    want = D[fresh, np.roll(fresh, -1, axis=1)].sum(axis=1).astype(np.float64)
    assert np.array_equal(costs.cpu().numpy(), want)
  g.release()
  g.release()  # idempotent


def test_argument_checks(lib):
  from tsp_gpu_clean_b200 import native

  out = ctypes.c_void_p(1)
  assert lib.tspb_graph_capture_begin(None) == native.TSPB_ERR_ARG
  assert lib.tspb_graph_capture_end(None, ctypes.byref(out)) == native.TSPB_ERR_ARG
  assert lib.tspb_graph_launch(None, None) == native.TSPB_ERR_ARG
  assert lib.tspb_graph_destroy(None) == native.TSPB_OK


def test_stream_handle_follows_the_current_stream(lib):
  """The raw current-stream handle the launches use is torch's current stream, inside and
  outside a stream context (graph capture relies on it)."""
  import torch

  from tsp_gpu_clean_b200.device import stream_handle

  assert stream_handle().value == (torch.cuda.current_stream().cuda_stream or None)
  side = torch.cuda.Stream()
  with torch.cuda.stream(side):
    assert stream_handle().value == side.cuda_stream
  assert stream_handle(side).value == side.cuda_stream
  assert stream_handle().value == (torch.cuda.current_stream().cuda_stream or None)
