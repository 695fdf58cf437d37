"""NumPy restatement of the reference distance matrices and k-NN candidate lists.

- `euc2d_block` / `euc2d_matrix`: `src/distances/matrix.py:77-86` and `:214-273`
  (separate multiplies and one add, `sqrt`, `+ 0.5`, truncation, zero diagonal).
- `distance_block` / `distance_matrix`: every coordinate-based TSPLIB type of
  `_distance_block` (`matrix.py:44-131`): EUC_2D/3D, MAN_2D/3D, MAX_2D/3D, CEIL_2D, ATT,
  GEO (DDD.MM degrees, PI = 3.141592, radius 6378.388 km, `pairwise.py:62-65`) and XRAY1.
- `candidate_list`: `src/distances/matrix.py:140-211` (`argpartition` then
  `lexsort`; the same NumPy calls, so a distance tie at the k-th boundary is
  resolved exactly as the reference resolves it on the same machine).

Test infrastructure only (see the package docstring).
"""

from __future__ import annotations

import numpy as np

CHUNK_THRESHOLD = 2048  # matrix.py:35
CHUNK_SIZE = 512  # matrix.py:38


def euc2d_block(rows: np.ndarray, coords: np.ndarray) -> np.ndarray:
  """`(len(rows), n)` int64 block, `matrix.py:82-86`."""
  diff = rows[:, None, :] - coords[None, :, :]
  sq = np.sum(diff * diff, axis=2)
  return (np.sqrt(sq) + 0.5).astype(np.int64)


def euc2d_matrix(coords: np.ndarray) -> np.ndarray:
  """Full int32 matrix with zero diagonal, `matrix.py:249-273`."""
  coords = np.asarray(coords, dtype=np.float64)
  n = coords.shape[0]
  if n <= CHUNK_THRESHOLD:
    d = euc2d_block(coords, coords)
  else:
    d = np.concatenate([euc2d_block(coords[s : s + CHUNK_SIZE], coords) for s in range(0, n, CHUNK_SIZE)], axis=0)
  out = d.astype(np.int32)
  np.fill_diagonal(out, 0)
  return out


GEO_PI = 3.141592
GEO_RADIUS = 6378.388
EDGE_TYPES = ("EUC_2D", "EUC_3D", "MAN_2D", "MAN_3D", "MAX_2D", "MAX_3D", "CEIL_2D", "ATT", "GEO", "XRAY1")


def _geo_radians(x: np.ndarray) -> np.ndarray:
  deg = np.trunc(x)
  return GEO_PI * (deg + 5.0 * (x - deg) / 3.0) / 180.0


def distance_block(rows: np.ndarray, coords: np.ndarray, edge_type: str) -> np.ndarray:
  """`(len(rows), n)` int64 block of one TSPLIB coordinate type (`matrix.py:57-131`)."""
  rows = np.asarray(rows, dtype=np.float64)
  coords = np.asarray(coords, dtype=np.float64)
  if edge_type == "XRAY1":
    phi = np.abs(rows[:, None, 0] - coords[None, :, 0])
    dphi = np.minimum(phi, np.abs(phi - 360.0))
    dchi = np.abs(rows[:, None, 1] - coords[None, :, 1])
    dth = np.abs(rows[:, None, 2] - coords[None, :, 2])
    cost = np.maximum(np.maximum(dphi / 1.0, dchi / 1.0), dth / 1.0)
    return np.trunc(100.0 * cost + 0.5).astype(np.int32).astype(np.int64)
  if edge_type == "GEO":
    la, lo = _geo_radians(rows[:, 0])[:, None], _geo_radians(rows[:, 1])[:, None]
    lb, lp = _geo_radians(coords[:, 0])[None, :], _geo_radians(coords[:, 1])[None, :]
    q1, q2, q3 = np.cos(lo - lp), np.cos(la - lb), np.cos(la + lb)
    arg = np.clip(0.5 * ((1.0 + q1) * q2 - (1.0 - q1) * q3), -1.0, 1.0)
    return (GEO_RADIUS * np.arccos(arg) + 1.0).astype(np.int64)
  diff = rows[:, None, :] - coords[None, :, :]
  if edge_type in ("EUC_2D", "EUC_3D"):
    return (np.sqrt(np.sum(diff * diff, axis=2)) + 0.5).astype(np.int64)
  if edge_type in ("MAN_2D", "MAN_3D"):
    return (np.sum(np.abs(diff), axis=2) + 0.5).astype(np.int64)
  if edge_type in ("MAX_2D", "MAX_3D"):
    return (np.max(np.abs(diff), axis=2) + 0.5).astype(np.int64)
  if edge_type == "CEIL_2D":
    return np.ceil(np.sqrt(np.sum(diff * diff, axis=2))).astype(np.int64)
  if edge_type == "ATT":
    r = np.sqrt(np.sum(diff * diff, axis=2) / 10.0)
    t = (r + 0.5).astype(np.int64)
    return np.where(t < r, t + 1, t)
  raise ValueError(f"unsupported edge type {edge_type!r}")


def distance_matrix(coords: np.ndarray, edge_type: str = "EUC_2D") -> np.ndarray:
  """Full int32 matrix of one TSPLIB coordinate type with a zero diagonal (`matrix.py:214-273`)."""
  coords = np.asarray(coords, dtype=np.float64)
  n = coords.shape[0]
  if n <= CHUNK_THRESHOLD:
    d = distance_block(coords, coords, edge_type)
  else:
    d = np.concatenate([distance_block(coords[s : s + CHUNK_SIZE], coords, edge_type)
                        for s in range(0, n, CHUNK_SIZE)], axis=0)
  out = d.astype(np.int32)
  np.fill_diagonal(out, 0)
  return out


def candidate_list(k: int, *, distances: np.ndarray | None = None, coords: np.ndarray | None = None,
                   edge_type: str = "EUC_2D") -> np.ndarray:
  """`(n, min(k, n-1))` int32 k-NN table, self excluded (`matrix.py:177-211`)."""
  if distances is not None:
    n = int(distances.shape[0])
  elif coords is not None:
    n = int(coords.shape[0])
  else:
    raise ValueError("candidate_list needs distances or coords")
  if n <= 1 or k <= 0:
    return np.zeros((n, 0), dtype=np.int32)
  k_eff = min(k, n - 1)
  sentinel = int(np.iinfo(np.int64).max)
  out = np.empty((n, k_eff), dtype=np.int32)
  for s in range(0, n, CHUNK_SIZE):
    e = min(s + CHUNK_SIZE, n)
    if distances is not None:
      block = np.asarray(distances[s:e], dtype=np.int64)
    else:
      block = distance_block(np.asarray(coords[s:e], dtype=np.float64), np.asarray(coords, dtype=np.float64),
                             edge_type)
    rows = np.arange(e - s)
    block[rows, np.arange(s, e)] = sentinel
    cols = np.argpartition(block, k_eff, axis=1)[:, :k_eff]
    cd = block[rows[:, None], cols]
    order = np.lexsort((cols, cd), axis=1)
    out[s:e, :] = cols[rows[:, None], order]
  return out
