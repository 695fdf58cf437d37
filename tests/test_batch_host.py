"""Host logic of the uneven batch: elite rows, buckets, the autotuner cache and the C
struct layout shared with libtspb.so. No GPU needed."""

from __future__ import annotations

import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from tsp_gpu_clean_b200 import native
from tsp_gpu_clean_b200.autotune import BatchAutotuner
from tsp_gpu_clean_b200.batch import FusedBatchSolver, elite_rows

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("P,elite", [(64, 8), (128, 16), (40, 6), (17, 3)])
def test_elite_rows_equal_the_per_run_argsort(P, elite):
  rng = np.random.default_rng(P)
  # few distinct values: ties across the elite edge in almost every row
  fit = rng.integers(0, 6, size=(300, P)).astype(np.float64) * 1000.0 + 12345.0
  rows = elite_rows(fit, elite)
  for r in range(fit.shape[0]):
    assert np.array_equal(rows[r], np.argsort(fit[r])[:elite])


def test_buckets_are_size_classes_largest_first():
  s = FusedBatchSolver(bucket_bounds=(100, 1000))
  ns = [50, 5000, 120, 999, 1001, 80, 4500]
  flags = [n > 4096 for n in ns]
  buckets = s._make_buckets(ns, flags)
  got = {(b.lo, b.hi, b.coords): [ns[i] for i in b.items] for b in buckets}
  assert got[(4, 100, False)] == [80, 50]
  assert got[(101, 1000, False)] == [999, 120]
  assert got[(1001, 1 << 16, False)] == [1001]
  assert got[(1001, 1 << 16, True)] == [5000, 4500]
  assert buckets[0].hi == 1 << 16  # the largest class is launched first
  assert all(b.max_n == max(ns[i] for i in b.items) for b in buckets)


def test_autotuner_picks_fastest_and_caches(tmp_path):
  path = str(tmp_path / "t.json")
  t = BatchAutotuner(cache_path=path)
  key = t.key("B200", "two_opt", mode="best", units=300, lo=1, hi=2)
  assert "units=512" in key
  calls = []

  def probe(c):
    calls.append(c)
    return {64: 3.0, 128: 1.0, 256: 2.0}[c]

  assert t.choose(key, [64, 128, 256], probe) == 128
  assert sorted(calls) == [64, 128, 256] and t.measured == 3
  t2 = BatchAutotuner(cache_path=path)
  assert t2.choose(key, [64, 128, 256], lambda c: pytest.fail("cached key measured again")) == 128
  assert t2.measured == 0
  # a cached choice that is no longer a candidate is measured again
  assert t2.choose(key, [64, 256], probe) == 256
  off = BatchAutotuner(enabled=False)
  assert off.choose("k", [64, 128, 256], lambda c: pytest.fail("disabled tuner measured")) == 128


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_ctypes_structs_match_the_c_header(tmp_path):
  fields_i = [f[0] for f in native.BatchInstance._fields_]
  fields_b = [f[0] for f in native.BatchState._fields_]
  fields_j = [f[0] for f in native.NNJob._fields_]
  src = ["#include <stdio.h>", "#include <stddef.h>", '#include "tspb.h"', "int main(void) {"]
  src.append('printf("%zu\\n", sizeof(tspb_nn_job));')
  for f in fields_j:
    src.append(f'printf("%zu\\n", offsetof(tspb_nn_job, {f}));')
  src.append('printf("%zu\\n", sizeof(tspb_batch_instance));')
  for f in fields_i:
    src.append(f'printf("%zu\\n", offsetof(tspb_batch_instance, {f}));')
  src.append('printf("%zu\\n", sizeof(tspb_batch));')
  for f in fields_b:
    src.append(f'printf("%zu\\n", offsetof(tspb_batch, {f}));')
  src.append("return 0; }")
  c = tmp_path / "layout.c"
  c.write_text("\n".join(src))
  exe = tmp_path / "layout"
  subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
  out = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
  want = [ctypes.sizeof(native.NNJob)] + [getattr(native.NNJob, f).offset for f in fields_j]
  want += [ctypes.sizeof(native.BatchInstance)] + [getattr(native.BatchInstance, f).offset for f in fields_i]
  want += [ctypes.sizeof(native.BatchState)] + [getattr(native.BatchState, f).offset for f in fields_b]
  assert out == want
