"""The C ABI library loads and exports every symbol `include/tspb.h` declares (no GPU needed)."""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared() -> list[str]:
  names = []
  for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
    if h.endswith(".h"):
      text = open(os.path.join(ROOT, "include", h)).read()
      names += re.findall(r"^\s*(?:int|int64_t|size_t|const char\*)\s+(tspb_\w+)\s*\(", text, flags=re.M)
  return names


@pytest.fixture(scope="module")
def lib():
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  from tsp_gpu_clean_b200 import native

  return native.load_library()


def test_every_declared_symbol_is_exported_and_bound(lib):
  from tsp_gpu_clean_b200 import native

  names = _declared()
  assert len(names) >= 12
  for name in names:
    assert hasattr(lib, name), name
    assert name in native.SIGNATURES, f"{name} has no ctypes signature"
  assert set(native.SIGNATURES) <= set(names), "a binding without a header declaration"


def test_status_strings_and_version(lib):
  assert lib.tspb_version() >= 100
  assert lib.tspb_status_string(0) == b"ok"
  assert b"permutation" in lib.tspb_status_string(3)


def test_host_argument_checks_run_without_a_gpu(lib):
  # Argument validation returns before any CUDA call.
  assert lib.tspb_two_opt(None, -1, 10, None, 0, None, None, None, None, None, None, 0, 0, 1, 256, None, None, None, 0, None) == 1
  assert lib.tspb_two_opt(None, 0, 10, None, 0, None, None, None, None, None, None, 0, 0, 1, 256, None, None, None, 0, None) == 0
  assert lib.tspb_two_opt(None, 1, 10, None, 0, None, None, None, None, None, None, 0, 7, 1, 256, None, None, None, 0, None) == 1
  assert lib.tspb_tournament(None, 0, None, 4, 0, None, None) == 1
  assert lib.tspb_stable_rank(None, 4, 5, None, None) == 1


def test_watchdog_budget_is_a_runtime_setting(lib):
  # host-only: the setter returns the previous budget; <= 0 restores the default 2^36 cycles
  default = 1 << 36
  assert lib.tspb_set_watchdog_cycles(1000) == default
  assert lib.tspb_set_watchdog_cycles(5) == 1000
  assert lib.tspb_set_watchdog_cycles(0) == 5
  assert lib.tspb_set_watchdog_cycles(-1) == default
  assert lib.tspb_set_watchdog_cycles(0) == default
  assert b"memory" in lib.tspb_status_string(8)


def test_workspace_sizes(lib):
  # best/first with arrays in shared memory need no workspace; multi_move needs its key buffer.
  assert lib.tspb_two_opt_workspace_bytes(8, 1000, 20, 0, 256) == 0
  ws = lib.tspb_two_opt_workspace_bytes(8, 1000, 20, 2, 256)
  assert ws >= 8 * 32768 * 8


def test_gpu_strategy_fails_loudly_without_a_device(monkeypatch):
  import torch

  from tsp_gpu_clean_b200.errors import GPUUnavailableError
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext
  from tsp_gpu_clean_b200.strategies.local_search import LocalSearchB200TourTwoOpt

  monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
  ctx = ProblemContext(Problem.from_coordinates(np.random.default_rng(0).uniform(0, 1000, (20, 2))), seed=0)
  with pytest.raises(GPUUnavailableError):
    LocalSearchB200TourTwoOpt(max_iterations=3).improve_batch(np.arange(20, dtype=np.int32), ctx)
