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
