import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)


def pytest_configure(config):
  config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libtspb.so")
  config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def golden():
  cache = {}

  def load(name):
    if name not in cache:
      cache[name] = dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))
    return cache[name]

  return load


def iter_two_opt_cases(data):
  """Yield `(case_id, n, k, mode, iters, D, cand, tours_in, tours_out)` from two_opt_small.npz."""
  from oracle import distances

  modes = ("best", "first", "multi_move")
  for c in range(int(data["num_cases"])):
    key = f"c{c}"
    n, k, m, iters = (int(v) for v in data[key + "_meta"])
    if key + "_dist" in data:
      D = data[key + "_dist"]
    else:
      D = distances.euc2d_matrix(data[key + "_coords"])
    cand = data.get(key + "_cand")
    yield c, n, (None if k < 0 else k), modes[m], iters, D, cand, data[key + "_in"], data[key + "_out"]
