"""NumPy restatement of the reference's exhaustive CPU 3-opt (open tours, symmetric distances).

Follows `three_opt_delta_cpu`, `apply_three_opt_case_cpu`, `cpu_three_opt_best_move` and
`cpu_three_opt_refine` of the reference's 3-opt experiment
(`benchmark_scripts/experiments-and-examples/experiment-comparing-3opt-and-2opt/gpu_three_opt.py:143-277`):

- cuts `0 <= i < j < k <= n - 1` remove the edges (a, b) = (t[i], t[i+1]),
  (c, d) = (t[j], t[j+1]) and (e, f) = (t[k], t[(k+1) % n]);
- scan order: i ascending, j ascending; for each (i, j) first the pure 2-opt case 1 at
  k = j (when j > i + 1), then k ascending with cases 2..7 in order; case 2 needs
  k > j + 1 and case 3 is skipped for i = 0, k = n - 1;
- the steepest move is the first one in scan order with the smallest negative delta;
- a move is applied as up to three segment reversals: [i+1, j] for cases 1, 4, 5, 7,
  [j+1, k] for cases 2, 4, 5, 6, then [i+1, k] for cases 3, 5, 6, 7;
- refinement repeats the steepest move for up to `max_iterations` passes.

Each (i, j) row of the scan is evaluated as NumPy arrays over k; the first minimum of a
row in (k, case) order is its earliest best move. Test infrastructure only (see the
package docstring).
"""

from __future__ import annotations

import numpy as np


def best_move(tour: np.ndarray, D: np.ndarray) -> tuple[int, int, int, int, int]:
  """`(delta, i, j, k, case)` of the steepest improving move, `(0, -1, -1, -1, 0)` if none
  (`cpu_three_opt_best_move`, `gpu_three_opt.py:219-253`)."""
  t = np.asarray(tour, dtype=np.int64)
  n = len(t)
  if n < 4:
    return (0, -1, -1, -1, 0)
  D = np.asarray(D, dtype=np.int64)
  nxt = np.roll(t, -1)
  edge = D[t, nxt]
  best = (0, -1, -1, -1, 0)
  kmax = n - 1
  for i in range(kmax - 1):
    a, b = t[i], t[i + 1]
    dab = edge[i]
    for j in range(i + 1, kmax):
      c, d = t[j], t[j + 1]
      dcd = edge[j]
      if j > i + 1:
        d1 = int(D[a, c] + D[b, d] - dab - dcd)
        if d1 < best[0]:
          best = (d1, i, j, j, 1)
      ks = np.arange(j + 1, kmax + 1)
      if ks.size == 0:
        continue
      e, f = t[ks], nxt[ks]
      def_ = edge[ks]
      old3 = dab + dcd + def_
      deltas = np.stack([
        D[c, e] + D[d, f] - dcd - def_,  # case 2
        D[a, e] + D[b, f] - dab - def_,  # case 3
        D[a, c] + D[b, e] + D[d, f] - old3,  # case 4
        D[a, d] + D[b, e] + D[c, f] - old3,  # case 5
        D[a, d] + D[c, e] + D[b, f] - old3,  # case 6
        D[a, e] + D[b, d] + D[c, f] - old3,  # case 7
      ], axis=1)
      big = np.iinfo(np.int64).max
      deltas[ks <= j + 1, 0] = big
      if i == 0:
        deltas[ks == n - 1, 1] = big
      flat = int(np.argmin(deltas))
      dmin = int(deltas.reshape(-1)[flat])
      if dmin < best[0]:
        r, cidx = divmod(flat, 6)
        best = (dmin, i, j, int(ks[r]), cidx + 2)
  return best


def apply_move(tour: np.ndarray, i: int, j: int, k: int, case: int) -> np.ndarray:
  """`apply_three_opt_case_cpu` (`gpu_three_opt.py:197-216`)."""
  out = np.asarray(tour, dtype=np.int32).copy()
  if case in (1, 4, 5, 7):
    out[i + 1 : j + 1] = out[i + 1 : j + 1][::-1]
  if case in (2, 4, 5, 6):
    out[j + 1 : k + 1] = out[j + 1 : k + 1][::-1]
  if case in (3, 5, 6, 7):
    out[i + 1 : k + 1] = out[i + 1 : k + 1][::-1]
  return out


def refine(tour: np.ndarray, D: np.ndarray, max_iterations: int = 10) -> tuple[np.ndarray, int]:
  """`cpu_three_opt_refine` (`gpu_three_opt.py:256-277`); also returns the moves applied."""
  cur = np.asarray(tour, dtype=np.int32).copy()
  moves = 0
  if len(cur) < 4 or max_iterations <= 0:
    return cur, 0
  for _ in range(max_iterations):
    delta, i, j, k, case = best_move(cur, D)
    if delta >= 0 or case == 0:
      break
    cur = apply_move(cur, i, j, k, case)
    moves += 1
  return cur, moves


def improve_batch(tours: np.ndarray, D: np.ndarray, max_iterations: int = 10) -> tuple[np.ndarray, list[int]]:
  out, moves = [], []
  for t in np.asarray(tours):
    r, m = refine(t, D, max_iterations)
    out.append(r)
    moves.append(m)
  return np.stack(out).astype(np.int32) if out else np.zeros((0, 0), np.int32), moves
