"""The native restatement of NumPy's PCG64 stream draws the GA tape exactly as NumPy does:
same tournament, PMX, inversion draws, same generator state after each generation and at
the end. Host path (no GPU needed)."""

from __future__ import annotations

import numpy as np
import pytest

from tsp_gpu_clean_b200.fused import draw_generation_tape, draw_generation_tape_numpy


@pytest.mark.parametrize("seed,P,kt,n,G,pre", [(1, 64, 5, 1000, 7, 3), (5, 7, 3, 13, 9, 0), (9, 128, 5, 4, 5, 1),
                                                (11, 2, 1, 5, 11, 2), (13, 512, 5, 2000, 40, 5), (17, 33, 4, 3, 6, 7),
                                                (19, 64, 5, 4899, 25, 0)])
def test_native_tape_equals_numpy(seed, P, kt, n, G, pre):
  a, b = np.random.default_rng(seed), np.random.default_rng(seed)
  if pre:  # leave NumPy's buffered 32-bit half set or clear
    a.integers(0, 7, size=pre, dtype=np.int32)
    b.integers(0, 7, size=pre, dtype=np.int32)
  got, gst = draw_generation_tape(a, G, P, kt, n)
  want, wst = draw_generation_tape_numpy(b, G, P, kt, n)
  for x, y in zip(got, want):
    assert x.dtype == y.dtype and np.array_equal(x, y)
  assert [gst[g] for g in range(G)] == list(wst)
  assert a.bit_generator.state == b.bit_generator.state
  # both generators continue identically
  assert np.array_equal(a.integers(0, 1000, 17), b.integers(0, 1000, 17))


def test_other_bit_generators_use_numpy():
  a = np.random.Generator(np.random.MT19937(4))
  b = np.random.Generator(np.random.MT19937(4))
  got, _ = draw_generation_tape(a, 3, 16, 5, 50)
  want, _ = draw_generation_tape_numpy(b, 3, 16, 5, 50)
  assert all(np.array_equal(x, y) for x, y in zip(got, want))
  assert np.array_equal(a.integers(0, 1 << 30, 64), b.integers(0, 1 << 30, 64))
