"""Host-side device plumbing that needs no GPU: operand caches release their contexts."""

from __future__ import annotations

import gc
import weakref

import numpy as np


def test_operand_cache_does_not_keep_contexts_alive():
  """Device operands are cached per context in a weak-key table; the cached value must not
  hold the context strongly, or every context and its device matrices would live forever."""
  from tsp_gpu_clean_b200 import device
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  problem = Problem.from_coordinates(np.random.default_rng(0).uniform(0, 100, (12, 2)))
  ctx = ProblemContext(problem, seed=0)
  ops = device.operands_for(ctx)
  assert ops.context is ctx and device.operands_for(ctx) is ops
  again = ProblemContext(problem, seed=1)
  assert device.operands_for(again)._shared is ops._shared  # one problem, shared device data
  ref = weakref.ref(ctx)
  before = len(device._operands)
  del ctx, ops
  gc.collect()
  assert ref() is None
  assert len(device._operands) == before - 1


def test_pack_overflow_flags_are_read_lazily_and_in_one_batch():
  """CandidateTables keeps the packing kernel's overflow flag until the packed table is
  first used; check_packed reads many flags at once. (CPU tensors stand in for device ones.)"""
  import torch

  from tsp_gpu_clean_b200.device import CandidateTables, check_packed

  def tables(flag):
    z = torch.zeros((3, 2), dtype=torch.int32)
    return CandidateTables(z, z, torch.zeros(4, dtype=torch.int32), torch.zeros(6, dtype=torch.int32),
                           packed=z.clone(), overflow=torch.tensor([flag], dtype=torch.int32))

  ok, bad = tables(0), tables(1)
  assert ok.packed_words is not None and bad.packed_words is not None  # unchecked views
  check_packed([ok, bad])
  assert ok.packed is not None and bad.packed is None
  assert ok._overflow is None and bad._overflow is None  # read once
  lazy = tables(1)
  assert lazy.packed is None  # first use reads the flag
  none = CandidateTables(torch.zeros((3, 2)), None, None, None)
  check_packed([none])
  assert none.packed is None


def test_check_free_logic_against_fake_allocator_counters(monkeypatch):
  """check_free on the CPU with fakes of the two torch calls it makes: cached memory covers
  a request without asking the driver; otherwise free + cached decides; an uninitialised
  allocator counts as nothing cached."""
  import pytest
  import torch

  from tsp_gpu_clean_b200 import device
  from tsp_gpu_clean_b200.errors import VRAMInsufficientError

  state = {"stats": {"reserved_bytes": {"all": {"current": 100}}, "allocated_bytes": {"all": {"current": 40}}},
           "free": 1000, "driver_calls": 0}

  def fake_mem_get_info(*a):
    state["driver_calls"] += 1
    return state["free"], 10**6

  monkeypatch.setattr(torch.cuda, "memory_stats_as_nested_dict", lambda *a: state["stats"])
  monkeypatch.setattr(torch.cuda, "mem_get_info", fake_mem_get_info)
  device.check_free(60, "fits the cache")
  assert state["driver_calls"] == 0
  device.check_free(1000 + 60, "fits free + cached")
  assert state["driver_calls"] == 1
  with pytest.raises(VRAMInsufficientError):
    device.check_free(1000 + 61, "one byte too many")
  state["stats"] = {}
  device.check_free(1000, "no allocator yet")
  with pytest.raises(VRAMInsufficientError):
    device.check_free(1001, "no allocator yet, too large")


def test_checked_budget_covers_the_allocations_inside_it(monkeypatch):
  """One check for a batch's total: the check_free calls inside the block draw on it without
  querying the allocator; beyond it, or after the block, they query again."""
  import pytest
  import torch

  from tsp_gpu_clean_b200 import device
  from tsp_gpu_clean_b200.errors import VRAMInsufficientError

  calls = {"stats": 0}

  def fake_stats(*a):
    calls["stats"] += 1
    return {"reserved_bytes": {"all": {"current": 0}}, "allocated_bytes": {"all": {"current": 0}}}

  monkeypatch.setattr(torch.cuda, "memory_stats_as_nested_dict", fake_stats)
  monkeypatch.setattr(torch.cuda, "mem_get_info", lambda *a: (1000, 10**6))
  with device.checked_budget(900, "batch"):
    assert calls["stats"] == 1
    device.check_free(600, "first matrix")
    device.check_free(300, "second matrix")
    assert calls["stats"] == 1  # drawn from the checked total
    device.check_free(50, "beyond the total")
    assert calls["stats"] == 2
  device.check_free(10, "after the block")
  assert calls["stats"] == 3
  with pytest.raises(VRAMInsufficientError):
    with device.checked_budget(2000, "too large"):
      pass
  assert device._checked() == 0
