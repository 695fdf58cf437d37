"""NumPy restatement of the reference CPU 2-opt (cyclic TSP topology).

Follows `src/algorithms/strategies/local_search/two_opt.py` of the reference:

- scan order, exhaustive: `_exhaustive_pairs` (:158-201, cyclic branch :194-196);
- scan order, candidate mode: `_pair_blocks` (:337-367);
- gains: `_pair_deltas` (:204-245, closed/cyclic branch);
- acceptance rules: `_step_best` (:386-440), `_step_first` (:442-489),
  `_step_multi_move` (:491-563);
- pass loop: `_refine` (:565-595), batch loop `improve_batch` (:611-628).

Every step also reports how many `(i, j)` pairs the reference evaluated in that
pass, which is the oracle-equivalent delta count used by the benchmark.

Test infrastructure only (see the package docstring).
"""

from __future__ import annotations

from functools import lru_cache

import numpy as np

#: Pairs per exhaustive block (`two_opt.py:155`); `first` stops at the first block
#: holding an improving pair, so the block size shapes the pair count.
PAIR_BLOCK = 1 << 18

MODES = ("best", "first", "multi_move")


@lru_cache(maxsize=16)
def exhaustive_pairs(n: int) -> tuple[np.ndarray, np.ndarray]:
  """All `(i, j)` with `0 <= i`, `i + 2 <= j <= n - 1`, minus `(0, n - 1)`, row-major.

  `two_opt.py:188-196`.
  """
  i_raw, j_raw = np.triu_indices(n, k=2)
  i_idx = i_raw.astype(np.int32)
  j_idx = j_raw.astype(np.int32)
  keep = ~((i_idx == 0) & (j_idx == n - 1))
  return i_idx[keep], j_idx[keep]


def inverse_positions(tour: np.ndarray) -> np.ndarray:
  """`pos[tour[p]] = p`, `-1` for absent ids (`src/utils/route_helpers.py:111-131`)."""
  if tour.size == 0:
    return np.full(0, -1, dtype=np.int32)
  size = max(int(tour.size), int(tour.max()) + 1)
  pos = np.full(size, -1, dtype=np.int32)
  pos[tour] = np.arange(tour.size, dtype=np.int32)
  return pos


def candidate_pairs(tour: np.ndarray, pos: np.ndarray, cand: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
  """Candidate-mode pairs in `(i, r)` row-major order, duplicates kept (`two_opt.py:347-367`)."""
  n = len(tour)
  rows = n - 2
  nb = cand[tour[:rows]]
  ok = (nb >= 0) & (nb < pos.size)
  if bool(ok.all()):
    j_mat = pos[nb]
  else:
    j_mat = np.where(ok, pos[np.clip(nb, 0, max(pos.size - 1, 0))], -1)
  i_mat = np.arange(rows, dtype=np.int32)[:, None]
  keep = (j_mat > i_mat + 1) & (j_mat < n)
  if rows:
    keep[0, :] &= j_mat[0, :] < n - 1
  i_keep, _ = np.nonzero(keep)
  return i_keep.astype(np.int32), j_mat[keep].astype(np.int32)


def pair_blocks(tour: np.ndarray, pos, cand):
  """Yield `(i, j)` blocks in scan order (`two_opt.py:337-367`)."""
  if cand is None:
    i_all, j_all = exhaustive_pairs(len(tour))
    for s in range(0, i_all.size, PAIR_BLOCK):
      yield i_all[s : s + PAIR_BLOCK], j_all[s : s + PAIR_BLOCK]
    return
  yield candidate_pairs(tour, pos, cand)


def pair_deltas(tour, succ, edge, D, i, j) -> np.ndarray:
  """`d(a,c) + d(b,d) - d(a,b) - d(c,d)` in int64 (`two_opt.py:237-245`)."""
  a = tour[i]
  b = succ[i]
  c = tour[j]
  d = succ[j]
  return np.asarray(D[a, c], dtype=np.int64) + np.asarray(D[b, d], dtype=np.int64) - edge[i] - edge[j]


def _scan_context(tour, D, cand):
  """`(succ, edge, pos)` of one pass (`two_opt.py:369-384`)."""
  succ = np.roll(tour, -1)
  edge = D[tour, succ].astype(np.int64)
  pos = inverse_positions(tour) if cand is not None else None
  return succ, edge, pos


def step(tour: np.ndarray, D: np.ndarray, cand, mode: str) -> tuple[bool, int]:
  """One acceptance step applied in place; returns `(applied, pairs_evaluated)`."""
  n = len(tour)
  if n < 4:
    return False, 0
  succ, edge, pos = _scan_context(tour, D, cand)
  pairs = 0
  if mode == "best":  # two_opt.py:386-440
    best, bi, bj = 0, -1, -1
    for i, j in pair_blocks(tour, pos, cand):
      pairs += int(i.size)
      if i.size == 0:
        continue
      g = pair_deltas(tour, succ, edge, D, i, j)
      p = int(np.argmin(g))
      if int(g[p]) < best:
        best, bi, bj = int(g[p]), int(i[p]), int(j[p])
    if best < 0:
      tour[bi + 1 : bj + 1] = tour[bi + 1 : bj + 1][::-1]
      return True, pairs
    return False, pairs
  if mode == "first":  # two_opt.py:442-489
    for i, j in pair_blocks(tour, pos, cand):
      pairs += int(i.size)
      if i.size == 0:
        continue
      imp = pair_deltas(tour, succ, edge, D, i, j) < 0
      if not bool(imp.any()):
        continue
      p = int(np.argmax(imp))
      a, b = int(i[p]), int(j[p])
      tour[a + 1 : b + 1] = tour[a + 1 : b + 1][::-1]
      return True, pairs
    return False, pairs
  if mode == "multi_move":  # two_opt.py:491-563
    gains, starts, ends = [], [], []
    for i, j in pair_blocks(tour, pos, cand):
      pairs += int(i.size)
      if i.size == 0:
        continue
      g = pair_deltas(tour, succ, edge, D, i, j)
      imp = g < 0
      if not bool(imp.any()):
        continue
      gains.append(g[imp])
      starts.append(i[imp])
      ends.append(j[imp])
    if not gains:
      return False, pairs
    order = np.argsort(np.concatenate(gains), kind="stable")
    fi = np.concatenate(starts)
    fj = np.concatenate(ends)
    occ = np.zeros(n, dtype=bool)
    applied = False
    for s in order:
      a, b = int(fi[s]), int(fj[s])
      lo = max(0, a)
      if occ[lo : b + 1].any():
        continue
      tour[a + 1 : b + 1] = tour[a + 1 : b + 1][::-1]
      occ[lo : b + 1] = True
      applied = True
    return applied, pairs
  raise ValueError(f"unknown mode {mode!r}")


def refine(tour: np.ndarray, D: np.ndarray, cand, mode: str, max_iterations: int):
  """Up to `max_iterations` steps on a copy (`two_opt.py:565-595`).

  Returns `(tour, stats)` with `stats = (passes, pairs, moves_applied_passes)`;
  `passes` counts every step call, including the final non-improving one.
  """
  out = np.array(tour, dtype=np.int32, copy=True)
  if len(out) < 4 or max_iterations <= 0:
    return out, (0, 0, 0)
  passes = pairs = applied = 0
  for _ in range(max_iterations):
    ok, p = step(out, D, cand, mode)
    passes += 1
    pairs += p
    if not ok:
      break
    applied += 1
  return out, (passes, pairs, applied)


def improve_batch(tours: np.ndarray, D: np.ndarray, cand, mode: str, max_iterations: int):
  """Refine every row independently (`two_opt.py:611-628`); returns `(tours, stats (N,3))`."""
  tours = np.asarray(tours, dtype=np.int32)
  was_1d = tours.ndim == 1
  batch = tours.reshape(1, -1) if was_1d else tours
  out = np.empty_like(batch)
  stats = np.zeros((len(batch), 3), dtype=np.int64)
  for r in range(len(batch)):
    out[r], stats[r] = refine(batch[r], D, cand, mode, max_iterations)
  return (out[0] if was_1d else out), stats


def resolve_candidates(cand_table, tours: np.ndarray, dimension: int):
  """`_resolve_candidates` for the cyclic TSP topology (`two_opt.py:117-149`)."""
  if cand_table is None:
    return None
  route_len = int(tours.shape[-1]) if tours.ndim >= 1 and tours.size > 0 else 0
  if route_len != dimension:
    return None
  largest = int(tours.max()) if tours.size else -1
  if largest >= cand_table.shape[0]:
    return None
  return cand_table
