"""NumPy restatement of the reference EUC_2D distance matrix and k-NN candidate lists.

- `euc2d_block` / `euc2d_matrix`: `src/distances/matrix.py:77-86` and `:214-273`
  (separate multiplies and one add, `sqrt`, `+ 0.5`, truncation, zero diagonal).
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


def candidate_list(k: int, *, distances: np.ndarray | None = None, coords: np.ndarray | None = None) -> np.ndarray:
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
      block = euc2d_block(np.asarray(coords[s:e], dtype=np.float64), np.asarray(coords, dtype=np.float64))
    rows = np.arange(e - s)
    block[rows, np.arange(s, e)] = sentinel
    cols = np.argpartition(block, k_eff, axis=1)[:, :k_eff]
    cd = block[rows[:, None], cols]
    order = np.lexsort((cols, cd), axis=1)
    out[s:e, :] = cols[rows[:, None], order]
  return out
