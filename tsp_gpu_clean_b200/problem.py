"""Problem instance and run context, mirroring the reference's data contract for TSP.

- `Problem` keeps the fields of the reference's frozen dataclass that the hot path
  reads (`src/data_models/problem.py`): name, dimension, problem_type, edge_type,
  coordinates, distances and `constraints.return_to_depot`.
- `ProblemContext` mirrors `src/protocols/problem_context.py:75-616`: one seeded
  `np.random.Generator` shared by every strategy (`:185-188`), lazily built host
  distances (`:266-301`) and k-NN candidate lists cached per k (`:420-454`), with an
  optional shared `candidate_cache` (`:123, 207`).

The k-NN table is built on the host with the reference's own procedure
(`argpartition` then `lexsort`, `src/distances/matrix.py:140-211`), so a distance tie
at the k-th boundary is resolved as the reference resolves it on the same machine.
B200 strategies also accept the reference's own `ProblemContext`: they only read
the attributes defined here.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np

DEFAULT_MAX_MATRIX_DIMENSION = 10_000
VRP_PROBLEM_TYPES = frozenset({"CVRP", "OVRP", "DCVRP"})


@dataclass(frozen=True)
class Constraints:
  return_to_depot: bool = True


@dataclass(frozen=True, eq=False)
class Problem:
  name: str
  dimension: int
  problem_type: str
  edge_type: str
  coordinates: np.ndarray | None
  distances: np.ndarray | None
  constraints: Constraints = field(default_factory=Constraints)

  @property
  def is_vrp(self) -> bool:
    return self.problem_type in VRP_PROBLEM_TYPES

  @classmethod
  def from_coordinates(cls, coords: np.ndarray, name: str = "synthetic", edge_type: str = "EUC_2D") -> "Problem":
    coords = np.asarray(coords, dtype=np.float64)
    if edge_type not in COORDINATE_EDGE_TYPES:
      raise ValueError(f"unsupported coordinate edge type {edge_type!r}; supported: {sorted(COORDINATE_EDGE_TYPES)}")
    return cls(name=name, dimension=len(coords), problem_type="TSP", edge_type=edge_type, coordinates=coords,
               distances=None)

  @classmethod
  def from_matrix(cls, dist: np.ndarray, name: str = "explicit") -> "Problem":
    dist = np.asarray(dist, dtype=np.int32)
    return cls(name=name, dimension=dist.shape[0], problem_type="TSP", edge_type="EXPLICIT", coordinates=None, distances=dist)


def make_rng(seed: Any = None) -> np.random.Generator:
  """`make_rng` of `src/utils/rng.py:23-45`."""
  if isinstance(seed, np.random.Generator):
    return seed
  if callable(seed):
    rng = seed()
    if not isinstance(rng, np.random.Generator):
      raise TypeError(f"Callable seed factory must return np.random.Generator, got {type(rng)!r}")
    return rng
  if isinstance(seed, (list, tuple)):
    return np.random.default_rng(np.random.SeedSequence(list(seed)))
  if seed is None or isinstance(seed, (int, np.integer)):
    return np.random.default_rng(seed)
  raise TypeError(f"Unsupported seed type: {type(seed)!r}")


def resolve_rng(context: Any = None, fallback: Any = None) -> np.random.Generator:
  """`resolve_rng` of `src/utils/rng.py:48-64`: the context generator wins."""
  rng = getattr(context, "rng", None) if context is not None else None
  if isinstance(rng, np.random.Generator):
    return rng
  return make_rng(fallback)


COORDINATE_EDGE_TYPES = frozenset(("EUC_2D", "EUC_3D", "MAN_2D", "MAN_3D", "MAX_2D", "MAX_3D", "CEIL_2D", "ATT", "GEO",
                                   "XRAY1"))


def _geo_radians(x: np.ndarray) -> np.ndarray:
  deg = np.trunc(x)
  return 3.141592 * (deg + 5.0 * (x - deg) / 3.0) / 180.0


def distance_block(rows: np.ndarray, coords: np.ndarray, edge_type: str = "EUC_2D") -> np.ndarray:
  """`(len(rows), n)` int64 block of a TSPLIB coordinate type, as `_distance_block` computes
  it (`matrix.py:44-131`); the context's k-NN tables are built from these blocks."""
  if edge_type == "XRAY1":
    phi = np.abs(rows[:, None, 0] - coords[None, :, 0])
    cost = np.maximum(np.maximum(np.minimum(phi, np.abs(phi - 360.0)), np.abs(rows[:, None, 1] - coords[None, :, 1])),
                      np.abs(rows[:, None, 2] - coords[None, :, 2]))
    return np.trunc(100.0 * cost + 0.5).astype(np.int32).astype(np.int64)
  if edge_type == "GEO":
    la, lo = _geo_radians(rows[:, 0])[:, None], _geo_radians(rows[:, 1])[:, None]
    lb, lp = _geo_radians(coords[:, 0])[None, :], _geo_radians(coords[:, 1])[None, :]
    q1, q2, q3 = np.cos(lo - lp), np.cos(la - lb), np.cos(la + lb)
    return (6378.388 * np.arccos(np.clip(0.5 * ((1.0 + q1) * q2 - (1.0 - q1) * q3), -1.0, 1.0)) + 1.0).astype(np.int64)
  diff = rows[:, None, :] - coords[None, :, :]
  if edge_type in ("EUC_2D", "EUC_3D"):
    return (np.sqrt(np.sum(diff * diff, axis=2)) + 0.5).astype(np.int64)
  if edge_type == "CEIL_2D":
    return np.ceil(np.sqrt(np.sum(diff * diff, axis=2))).astype(np.int64)
  if edge_type == "ATT":
    r = np.sqrt(np.sum(diff * diff, axis=2) / 10.0)
    t = (r + 0.5).astype(np.int64)
    return np.where(t < r, t + 1, t)
  if edge_type in ("MAN_2D", "MAN_3D"):
    return (np.sum(np.abs(diff), axis=2) + 0.5).astype(np.int64)
  if edge_type in ("MAX_2D", "MAX_3D"):
    return (np.max(np.abs(diff), axis=2) + 0.5).astype(np.int64)
  raise ValueError(f"unsupported coordinate edge type {edge_type!r}")


def euc2d_block(rows: np.ndarray, coords: np.ndarray) -> np.ndarray:
  """EUC_2D block `nint(sqrt(dx^2 + dy^2))` as int64 (`matrix.py:82-86`)."""
  return distance_block(rows, coords, "EUC_2D")


def compute_distance_matrix(coords: np.ndarray, edge_type: str = "EUC_2D") -> np.ndarray:
  """Host matrix of a coordinate type, int32, zero diagonal (`matrix.py:214-273`); the
  device builds the same matrix with `tspb_distance_matrix`."""
  coords = np.asarray(coords, dtype=np.float64)
  n = coords.shape[0]
  if n <= 2048:
    d = distance_block(coords, coords, edge_type)
  else:
    d = np.concatenate([distance_block(coords[s : s + 512], coords, edge_type) for s in range(0, n, 512)], axis=0)
  out = d.astype(np.int32)
  np.fill_diagonal(out, 0)
  return out


def compute_candidate_list(k: int, distances: np.ndarray | None = None, coords: np.ndarray | None = None,
                           edge_type: str = "EUC_2D") -> np.ndarray:
  """Host k-NN table `(n, min(k, n-1))` int32 (`matrix.py:140-211`)."""
  n = int(distances.shape[0] if distances is not None else coords.shape[0])
  if n <= 1 or k <= 0:
    return np.zeros((n, 0), dtype=np.int32)
  k_eff = min(k, n - 1)
  out = np.empty((n, k_eff), dtype=np.int32)
  big = int(np.iinfo(np.int64).max)
  for s in range(0, n, 512):
    e = min(s + 512, n)
    if distances is not None:
      block = np.asarray(distances[s:e], dtype=np.int64)
    else:
      block = distance_block(np.asarray(coords[s:e], dtype=np.float64), np.asarray(coords, dtype=np.float64),
                             edge_type)
    r = np.arange(e - s)
    block[r, np.arange(s, e)] = big
    cols = np.argpartition(block, k_eff, axis=1)[:, :k_eff]
    cd = block[r[:, None], cols]
    order = np.lexsort((cols, cd), axis=1)
    out[s:e] = cols[r[:, None], order]
  return out


class ProblemContext:
  """Run context: one RNG, lazy host caches, and the candidate-list cache."""

  def __init__(
    self,
    problem: Problem,
    xp: Any = np,
    seed: Any = None,
    max_matrix_dimension: int = DEFAULT_MAX_MATRIX_DIMENSION,
    candidate_cache: dict[int, np.ndarray] | None = None,
  ) -> None:
    if problem.distances is None and problem.coordinates is None:
      raise ValueError(f"Problem '{problem.name}' has no distances or coordinates to compute distance matrix from.")
    self.xp = xp
    self.problem = problem
    self.dimension = problem.dimension
    self.max_matrix_dimension = max_matrix_dimension
    self.rng = make_rng(seed)
    self.seed = seed
    self.h2d_bytes = 0
    self._cpu_distances: np.ndarray | None = None
    self._cpu_candidate_lists: dict[int, np.ndarray] = candidate_cache if candidate_cache is not None else {}

  @property
  def return_to_depot(self) -> bool:
    return bool(self.problem.constraints.return_to_depot)

  @property
  def is_closed(self) -> bool:
    return self.problem.problem_type in VRP_PROBLEM_TYPES and self.return_to_depot

  def get_cpu_distances(self) -> np.ndarray:
    if self._cpu_distances is None:
      if self.problem.distances is not None:
        self._cpu_distances = self.problem.distances
      else:
        self._cpu_distances = compute_distance_matrix(self.problem.coordinates, self.problem.edge_type)
    return self._cpu_distances

  def get_cpu_coordinates(self) -> np.ndarray | None:
    return self.problem.coordinates

  def get_cpu_candidate_list(self, k: int = 20) -> np.ndarray:
    cached = self._cpu_candidate_lists.get(k)
    if cached is None:
      if self.problem.distances is not None:
        cached = compute_candidate_list(k, distances=self.problem.distances)
      else:
        cached = compute_candidate_list(k, coords=self.problem.coordinates, edge_type=self.problem.edge_type)
      self._cpu_candidate_lists[k] = cached
    return cached

  def __repr__(self) -> str:
    return f"<ProblemContext: {self.problem.name} ({self.problem.problem_type}, N={self.dimension})>"
