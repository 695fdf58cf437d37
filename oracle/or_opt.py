"""NumPy definition of the candidate-list Or-opt local search (test infrastructure only).

Parity unpinned against the reference: lucasgaldinos/tsp_gpu_clean has no Or-opt strategy
(its local-search package holds 2-opt, and its 3-opt experiment covers segment moves only
as one reconnection case of exhaustive 3-opt). This module therefore defines the operator
that `tspb_or_opt` implements, restating the Or-opt neighbourhood (I. Or, 1976: move a
segment of one to three consecutive cities elsewhere in the tour, optionally reversed)
with the same k-NN candidate and fixed-start conventions as the reference's candidate
2-opt (`src/algorithms/strategies/local_search/two_opt.py:347-367`). Two independent
restatements are kept: `best_move` (NumPy arrays over a pass) and `best_move_loops`
(plain loops); the tests pin each against the other, the applied delta against the
tour-length change, and the neighbourhood against the 3-opt oracle (pinned to the
reference's CPU 3-opt): every Or-opt move is a 3-opt reconnection, so 3-opt local optima
admit no improving Or-opt move.

Definition, for an open cyclic tour `t` (a permutation of 0..n-1 whose position 0 never
moves), a k-NN table `N` of shape (n, k) and symmetric distances `D`:

- a move is `(i, L, r, o)`: the segment `S = t[i .. i+L-1]` with `1 <= L <= max_segment`,
  `1 <= i` and `i + L - 1 <= n - 1`; `o = 0` inserts it forward after `c = N[t[i]][r]`,
  `o = 1` (only for `L >= 2`) reversed after `c = N[t[i+L-1]][r]`;
- with `p = t[i-1]`, `q = t[(i+L) % n]`, `j = pos[c]` and `e = t[(j+1) % n]`, the move is
  valid when `j < i - 1` or `j > i + L - 1`; its delta is
  `D[p,q] - D[p,s0] - D[sl,q] + D[x,c] + D[y,e] - D[c,e]` with `(x, y) = (s0, sl)` forward
  and `(sl, s0)` reversed (`s0 = t[i]`, `sl = t[i+L-1]`), in exact integers;
- the scan key is `(((i-1) * max_segment + (L-1)) * k + r) * 2 + o`; a pass applies the
  move with the smallest negative delta, the smallest key among equal deltas;
- the move removes `S` and re-inserts it (forward or reversed) between `c` and `e`;
  positions outside `[min(i, j+1), max(j, i+L-1)]` keep their cities;
- refinement repeats passes until none improves or `max_iterations` passes ran.
"""

from __future__ import annotations

import numpy as np

NO_MOVE = (0, -1, -1, -1, -1)


def _keys(i, L, r, o, max_segment, k):
  return (((i - 1) * max_segment + (L - 1)) * k + r) * 2 + o


def best_move(tour: np.ndarray, D: np.ndarray, cand: np.ndarray, max_segment: int = 3):
  """`(delta, i, L, r, o)` of the best improving move, `NO_MOVE` when none improves, and
  the number of valid entries of the pass."""
  t = np.asarray(tour, dtype=np.int64)
  n = t.shape[0]
  cand = np.asarray(cand, dtype=np.int64)
  k = cand.shape[1] if cand.ndim == 2 else 0
  if n < 3 or k == 0:
    return NO_MOVE, 0
  pos = np.empty(n, dtype=np.int64)
  pos[t] = np.arange(n)
  Dl = np.asarray(D, dtype=np.int64)
  best = None
  valid_total = 0
  for L in range(1, min(max_segment, n - 1) + 1):
    i = np.arange(1, n - L + 1)  # segment starts
    s0, sl = t[i], t[i + L - 1]
    p, q = t[i - 1], t[(i + L) % n]
    base = Dl[p, q] - Dl[p, s0] - Dl[sl, q]
    for o in ((0, 1) if L >= 2 else (0,)):
      x, y = (s0, sl) if o == 0 else (sl, s0)
      c = cand[x]  # (rows, k)
      j = pos[c]
      e = t[(j + 1) % n]
      ok = (j < (i - 1)[:, None]) | (j > (i + L - 1)[:, None])
      delta = base[:, None] + Dl[x[:, None], c] + Dl[y[:, None], e] - Dl[c, e]
      valid_total += int(ok.sum())
      imp = ok & (delta < 0)
      if not imp.any():
        continue
      ii, rr = np.nonzero(imp)
      d = delta[ii, rr]
      key = _keys(i[ii], L, rr, o, max_segment, k)
      m = np.lexsort((key, d))[0]
      cand_best = (int(d[m]), int(key[m]), int(i[ii[m]]), L, int(rr[m]), o)
      if best is None or (cand_best[0], cand_best[1]) < (best[0], best[1]):
        best = cand_best
  if best is None:
    return NO_MOVE, valid_total
  return (best[0], best[2], best[3], best[4], best[5]), valid_total


def best_move_loops(tour, D, cand, max_segment: int = 3):
  """The same search as plain loops over the scan key order (small tours)."""
  t = [int(v) for v in tour]
  n = len(t)
  k = len(cand[0]) if n and len(cand) else 0
  if n < 3 or k == 0:
    return NO_MOVE
  pos = [0] * n
  for idx, v in enumerate(t):
    pos[v] = idx
  best = None
  for i in range(1, n):
    for L in range(1, max_segment + 1):
      if i + L - 1 > n - 1:
        continue
      s0, sl, p, q = t[i], t[i + L - 1], t[i - 1], t[(i + L) % n]
      for r in range(k):
        for o in (0, 1):
          if o == 1 and L < 2:
            continue
          x, y = (s0, sl) if o == 0 else (sl, s0)
          c = int(cand[x][r])
          j = pos[c]
          if i - 1 <= j <= i + L - 1:
            continue
          e = t[(j + 1) % n]
          delta = int(D[p][q]) - int(D[p][s0]) - int(D[sl][q]) + int(D[x][c]) + int(D[y][e]) - int(D[c][e])
          if delta < 0:
            key = _keys(i, L, r, o, max_segment, k)
            if best is None or (delta, key) < best[:2]:
              best = (delta, key, i, L, r, o)
  if best is None:
    return NO_MOVE
  return (best[0], best[2], best[3], best[4], best[5])


def apply_move(tour: np.ndarray, cand: np.ndarray, i: int, L: int, r: int, o: int) -> np.ndarray:
  """The tour after move `(i, L, r, o)`."""
  t = np.asarray(tour)
  n = t.shape[0]
  x = t[i] if o == 0 else t[i + L - 1]
  c = int(cand[x][r])
  j = int(np.nonzero(t == c)[0][0])
  seg = t[i:i + L] if o == 0 else t[i:i + L][::-1]
  rest = np.concatenate([t[:i], t[i + L:]])
  # c's index in `rest`: unchanged when it sat before the segment, else shifted by L
  jr = j if j < i else j - L
  out = np.concatenate([rest[:jr + 1], seg, rest[jr + 1:]])
  assert out.shape[0] == n and out[0] == t[0]
  return out.astype(t.dtype)


def tour_length(tour, D) -> int:
  t = np.asarray(tour, dtype=np.int64)
  return int(np.asarray(D, dtype=np.int64)[t, np.roll(t, -1)].sum())


def refine(tour, D, cand, max_iterations: int, max_segment: int = 3):
  """`(tour, passes, moves, evaluated)`: passes of `best_move` until none improves or
  `max_iterations` passes ran (a pass that finds nothing counts)."""
  t = np.asarray(tour, dtype=np.int32).copy()
  passes = moves = evaluated = 0
  while passes < max_iterations:
    (delta, i, L, r, o), valid = best_move(t, D, cand, max_segment)
    passes += 1
    evaluated += valid
    if i < 0:
      break
    t = apply_move(t, cand, i, L, r, o)
    moves += 1
  return t, passes, moves, evaluated
