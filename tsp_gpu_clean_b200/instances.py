"""Seeded synthetic TSP instances and tour batches for the benchmark workloads.

All coordinates are float64 in `[0, 1000]^2` and distances are TSPLIB EUC_2D
(`nint(sqrt(dx^2 + dy^2))` as int32), the same edge type the reference uses
for its coordinate problems (`src/distances/matrix.py:84-86`).

Workloads (named by what they are):

- `uniform_instance(n, seed)`: n uniform cities (the 100-city GA run and the
  2000-city fused run).
- `clustered_instance(n, centres, sigma, seed)`: Gaussian mixture around uniform
  centres, clipped to the square (the 1000-city, 20-cluster 2-opt batch).
- `random_tours(n, count, seed)`: independent random permutations.
- `uneven_batch(count, seed)`: instance sizes log-uniform in `[50, 5000]`, half
  uniform, half mixtures with 10-50 centres.
"""

from __future__ import annotations

import math

import numpy as np


def uniform_instance(n: int, seed: int) -> np.ndarray:
  rng = np.random.default_rng(seed)
  return rng.uniform(0.0, 1000.0, (n, 2))


def clustered_instance(n: int, centres: int, sigma: float, seed: int) -> np.ndarray:
  rng = np.random.default_rng(seed)
  c = rng.uniform(0.0, 1000.0, (centres, 2))
  labels = rng.integers(0, centres, n)
  return np.clip(c[labels] + rng.normal(0.0, sigma, (n, 2)), 0.0, 1000.0)


def random_tours(n: int, count: int, seed: int) -> np.ndarray:
  rng = np.random.default_rng(seed)
  return np.stack([rng.permutation(n) for _ in range(count)]).astype(np.int32)


def uneven_batch(count: int, seed: int, n_min: int = 50, n_max: int = 5000) -> list[np.ndarray]:
  rng = np.random.default_rng(seed)
  out = []
  for idx in range(count):
    n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
    sub = int(rng.integers(0, 2**31 - 1))
    if idx % 2 == 0:
      out.append(uniform_instance(n, sub))
    else:
      out.append(clustered_instance(n, int(rng.integers(10, 51)), 30.0, sub))
  return out


#: The 2-opt batch workload: 1024 random tours of a 1000-city, 20-cluster instance.
TWO_OPT_N = 1000
TWO_OPT_TOURS = 1024
TWO_OPT_INSTANCE_SEED = 20260
TWO_OPT_TOUR_SEED = 20261


def two_opt_workload(tours: int = TWO_OPT_TOURS) -> tuple[np.ndarray, np.ndarray]:
  coords = clustered_instance(TWO_OPT_N, 20, 30.0, TWO_OPT_INSTANCE_SEED)
  return coords, random_tours(TWO_OPT_N, tours, TWO_OPT_TOUR_SEED)
