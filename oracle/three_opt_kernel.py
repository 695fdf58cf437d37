"""Restatement of the reference's 3-opt CUDA kernels: candidate-pruned scan and multi_move.

Test infrastructure only (see the package docstring). The reference defines these two
parts of its experimental 3-opt only through its kernels
(`benchmark_scripts/experiments-and-examples/experiment-comparing-3opt-and-2opt/kernels/`:
`three_opt_common.cuh`, `three_opt_batch.cu`, `three_opt_multi_move.cu`, driven by
`LocalSearchGPUThreeOpt._improve_grid`, `gpu_three_opt.py:452-537`), so their results are
those of its thread layout, restated here on the CPU:

- B = prev_power_of_2(min(threads_per_block, n)) clamped to [1, 256] "threads" per tour
  (`gpu_three_opt.py:478-479`, `utils/gpu_helpers.py:103-106`); thread t scans the anchors
  i = t, t + B, ... in increasing order and keeps its own best move, replacing it only by a
  strictly smaller delta (`three_opt_consider`, `three_opt_common.cuh:59-77`), starting
  from delta 0 (only improving moves are kept).
- Candidate scan of anchor i (`three_opt_scan_neighborhood`, `three_opt_common.cuh:289-384`),
  a = t[i], b = t[(i + 1) % n], d_ab = d(a, b), pos = tour positions, cand rows sorted:
    1. 2-opt seeds: r1 = 0..k-1, v1 = N[a][r1], p1 = pos[v1], valid when p1 > i + 1 and not
       (i == 0 and p1 == n - 1): case 1 at (i, p1, p1), delta
       d(a, v1) - d_ab - d(v1, t[p1+1]) + d(b, t[p1+1]);
    2. pass A: r1 = 0.. while d(a, v1) < d_ab (first r1 with d(a, v1) >= d_ab ends it),
       then r2 = 0..inner-1 over v2 = N[b][r2]: `eval_pair`;
    3. pass B: r2 = 0.. while d(b, v2) < d_ab, then r1 = 0..inner-1 skipping those with
       d(a, v1) < d_ab: `eval_pair`.
  `eval_pair` (`three_opt_eval_cyclic_pair`, `:155-256`) takes the positions relative to i
  (rel = (p - i) mod n) and considers, in this order: cases 4, 5, 6 when 2 <= rel1 < rel2;
  the one-city relocation (case 5 at (p1 - 1, p1)) when 2 <= rel1 == rel2; case 7 when
  2 <= rel2 < rel1. Each is given in cyclic cut order (i, j_cyc, k_cyc) and turned into
  sorted cuts i0 < j0 < k0 by the rotation of `three_opt_consider_cyclic` (`:84-148`).
- Exhaustive scan of anchor i (`:385-447`): j = i+1..n-2, then case 1 at (i, j, j) when
  j > i + 1, then k = j+1..n-1 with cases 2 (k > j + 1), 3 (not i == 0 and k == n - 1),
  4, 5, 6, 7.
- batch (`three_opt_batch.cu`): the block minimum of the B thread bests
  (`three_opt_reduce_block_min`, `:485-530`: pairwise t vs t + s for s = B/2 .. 64 taking
  the right one only when strictly smaller, then t = 1..min(B, 64)-1 in order, strictly
  smaller again), applied when negative.
- multi_move (`three_opt_multi_move.cu`): up to min(B, n // 2) times, the smallest
  negative thread best (lowest thread on ties) is applied and cleared, and every other
  thread best whose cut span [i0, k0] meets [mi, mk] is dropped.
- a move applies the reversals [i0+1, j0] (cases 1, 4, 5, 7), [j0+1, k0] (2, 4, 5, 6),
  then [i0+1, k0] (3, 5, 6, 7) (`three_opt_apply_reconnection`, `:463-483`).
- every pass is one launch, `max_iterations` of them; a pass without an improving move
  changes nothing, so refinement may stop there.

Moves are returned as `(delta, i0, j0, k0, case)`; the thread bests are also exposed for
tests of the reduction.
"""

from __future__ import annotations

import numpy as np

NO_MOVE = (0, -1, -1, -1, 0)


def virtual_threads(threads_per_block: int, n: int) -> int:
  """Threads per tour of the reference's grid kernels (`gpu_three_opt.py:478-479`)."""
  v = max(1, min(int(threads_per_block), max(1, int(n))))
  p = 1 << (v.bit_length() - 1)
  return max(1, min(p, 256))


def _rotate(i: int, jc: int, kc: int, case: int) -> tuple[int, int, int, int]:
  """Cyclic cuts (i -> jc -> kc) as sorted linear cuts (`three_opt_consider_cyclic`)."""
  if i < jc < kc:
    return i, jc, kc, case
  if kc < i < jc:
    return kc, i, jc, {4: 6, 6: 7, 7: 4}.get(case, 5)
  return jc, kc, i, {4: 7, 7: 6, 6: 4}.get(case, 5)


class _Best:
  __slots__ = ("delta", "move")

  def __init__(self):
    self.delta = 0
    self.move = NO_MOVE

  def consider(self, delta: int, i0: int, j0: int, k0: int, case: int) -> None:
    if delta < self.delta:
      self.delta = delta
      self.move = (delta, i0, j0, k0, case)


def _eval_pair(best: _Best, i, n, d_ab, p1, d_av1, p2, d_bv2, t, edge, D):
  rel1 = (p1 - i) % n
  rel2 = (p2 - i) % n
  base = d_av1 + d_bv2 - d_ab
  if rel1 >= 2 and rel1 < rel2:
    # case 4: j = p1 (c = v1), k = p2 (e = v2), third new edge (d, f)
    jc, kc = p1, p2
    dl = base - edge[jc] - edge[kc] + int(D[t[(jc + 1) % n], t[(kc + 1) % n]])
    if dl < best.delta:
      best.consider(dl, *_rotate(i, jc, kc, 4))
    # case 5: j = p1 - 1 (d = v1), k = p2 (e = v2), third new edge (c, f)
    jc, kc = (p1 - 1) % n, p2
    dl = base - edge[jc] - edge[kc] + int(D[t[jc], t[(kc + 1) % n]])
    if dl < best.delta:
      best.consider(dl, *_rotate(i, jc, kc, 5))
    # case 6: j = p1 - 1 (d = v1), k = p2 - 1 (f = v2), third new edge (c, e)
    jc, kc = (p1 - 1) % n, (p2 - 1) % n
    dl = base - edge[jc] - edge[kc] + int(D[t[jc], t[kc]])
    if dl < best.delta:
      best.consider(dl, *_rotate(i, jc, kc, 6))
  elif rel1 >= 2 and rel1 == rel2:
    # v1 == v2: move that one city between a and b (case 5 at j = p1 - 1, k = p1)
    jc, kc = (p1 - 1) % n, p1
    dl = base - edge[jc] - edge[kc] + int(D[t[jc], t[(kc + 1) % n]])
    if dl < best.delta:
      best.consider(dl, *_rotate(i, jc, kc, 5))
  elif rel2 >= 2 and rel2 < rel1:
    # case 7: j = p2 - 1 (d = v2), k = p1 (e = v1), third new edge (c, f)
    jc, kc = (p2 - 1) % n, p1
    dl = base - edge[jc] - edge[kc] + int(D[t[jc], t[(kc + 1) % n]])
    if dl < best.delta:
      best.consider(dl, *_rotate(i, jc, kc, 7))


def _scan_candidate_anchor(best: _Best, i, t, pos, edge, D, cand, inner):
  n = len(t)
  k = cand.shape[1]
  a, b = int(t[i]), int(t[(i + 1) % n])
  d_ab = int(edge[i])
  ca, cb = cand[a], cand[b]
  for r1 in range(k):  # 2-opt seeds
    v1 = int(ca[r1])
    p1 = int(pos[v1])
    if p1 > i + 1 and not (i == 0 and p1 == n - 1):
      dn = int(t[(p1 + 1) % n])
      dl = int(D[a, v1]) - d_ab - int(edge[p1]) + int(D[b, dn])
      best.consider(dl, i, p1, p1, 1)
  for r1 in range(k):  # pass A
    v1 = int(ca[r1])
    d_av1 = int(D[a, v1])
    if d_av1 >= d_ab:
      break
    p1 = int(pos[v1])
    for r2 in range(inner):
      v2 = int(cb[r2])
      _eval_pair(best, i, n, d_ab, p1, d_av1, int(pos[v2]), int(D[b, v2]), t, edge, D)
  for r2 in range(k):  # pass B
    v2 = int(cb[r2])
    d_bv2 = int(D[b, v2])
    if d_bv2 >= d_ab:
      break
    p2 = int(pos[v2])
    for r1 in range(inner):
      v1 = int(ca[r1])
      d_av1 = int(D[a, v1])
      if d_av1 < d_ab:
        continue
      _eval_pair(best, i, n, d_ab, int(pos[v1]), d_av1, p2, d_bv2, t, edge, D)


def _scan_exhaustive_anchor(best: _Best, i, t, edge, D):
  n = len(t)
  kmax = n - 1
  if i > kmax - 2:
    return
  a, b = int(t[i]), int(t[i + 1])
  d_ab = int(edge[i])
  for j in range(i + 1, kmax):
    c, d = int(t[j]), int(t[j + 1])
    d_cd = int(edge[j])
    if j > i + 1:
      best.consider(int(D[a, c]) + int(D[b, d]) - d_ab - d_cd, i, j, j, 1)
    old_ab_cd = d_ab + d_cd
    for k in range(j + 1, kmax + 1):
      e, f = int(t[k]), int(t[(k + 1) % n])
      old3 = old_ab_cd + int(edge[k])
      if k > j + 1:
        best.consider(int(D[c, e]) + int(D[d, f]) - d_cd - int(edge[k]), i, j, k, 2)
      if not (i == 0 and k == n - 1):
        best.consider(int(D[a, e]) + int(D[b, f]) - d_ab - int(edge[k]), i, j, k, 3)
      best.consider(int(D[a, c]) + int(D[b, e]) + int(D[d, f]) - old3, i, j, k, 4)
      best.consider(int(D[a, d]) + int(D[b, e]) + int(D[c, f]) - old3, i, j, k, 5)
      best.consider(int(D[a, d]) + int(D[c, e]) + int(D[b, f]) - old3, i, j, k, 6)
      best.consider(int(D[a, e]) + int(D[b, d]) + int(D[c, f]) - old3, i, j, k, 7)


def thread_bests(tour, D, cand, inner_k, B: int) -> list[tuple[int, int, int, int, int]]:
  """Best move of each of the B threads in one pass (`NO_MOVE` when none improves)."""
  t = np.asarray(tour, dtype=np.int64)
  n = len(t)
  edge = D[t, np.roll(t, -1)].astype(np.int64)
  out = []
  if cand is not None:
    cand = np.asarray(cand)
    k = cand.shape[1]
    inner = min(int(inner_k), k) if inner_k and inner_k > 0 else k
    pos = np.empty(n, dtype=np.int64)
    pos[t] = np.arange(n)
  for tid in range(B):
    best = _Best()
    for i in range(tid, n, B):
      if cand is not None:
        _scan_candidate_anchor(best, i, t, pos, edge, D, cand, inner)
      else:
        _scan_exhaustive_anchor(best, i, t, edge, D)
    out.append(best.move)
  return out


def block_min(bests) -> tuple[int, int, int, int, int]:
  """`three_opt_reduce_block_min` over the thread bests."""
  v = list(bests)
  B = len(v)
  s = B // 2
  while s > 32:
    for tid in range(s):
      if tid + s < B and v[tid + s][0] < v[tid][0]:
        v[tid] = v[tid + s]
    s >>= 1
  best = v[0]
  for tt in range(1, min(B, 64)):
    if v[tt][0] < best[0]:
      best = v[tt]
  return best


def apply_move(tour: np.ndarray, move) -> None:
  """In place: the up-to-three reversals of `three_opt_apply_reconnection`."""
  _, i, j, k, case = move
  if case in (1, 4, 5, 7):
    tour[i + 1:j + 1] = tour[i + 1:j + 1][::-1].copy()
  if case in (2, 4, 5, 6):
    tour[j + 1:k + 1] = tour[j + 1:k + 1][::-1].copy()
  if case in (3, 5, 6, 7):
    tour[i + 1:k + 1] = tour[i + 1:k + 1][::-1].copy()


def one_pass(tour, D, cand, inner_k, B: int, mode: str) -> int:
  """One launch on `tour` (in place); returns the number of moves applied."""
  bests = thread_bests(tour, D, cand, inner_k, B)
  if mode == "batch":
    m = block_min(bests)
    if m[0] < 0:
      apply_move(tour, m)
      return 1
    return 0
  n = len(tour)
  deltas = [b[0] for b in bests]
  applied = 0
  for _ in range(min(B, n // 2)):
    best_t, best_d = -1, 0
    for tt in range(B):
      if deltas[tt] < best_d:
        best_d, best_t = deltas[tt], tt
    if best_t < 0:
      break
    m = bests[best_t]
    deltas[best_t] = 0
    apply_move(tour, m)
    applied += 1
    mi, mk = m[1], m[3]
    for tt in range(B):
      if deltas[tt] < 0 and not (bests[tt][3] < mi or mk < bests[tt][1]):
        deltas[tt] = 0
  return applied


def refine(tour, D, cand, inner_k, threads_per_block: int, mode: str, max_iterations: int):
  """`max_iterations` launches on a copy; returns `(tour, (passes, moves))`, where passes
  counts launches up to and including the first one that applies nothing."""
  t = np.array(tour, dtype=np.int32, copy=True)
  n = len(t)
  if n < 4 or max_iterations <= 0:
    return t, (0, 0)
  B = virtual_threads(threads_per_block, n)
  D = np.asarray(D, dtype=np.int64)
  passes = moves = 0
  for _ in range(max_iterations):
    passes += 1
    got = one_pass(t, D, cand, inner_k, B, mode)
    moves += got
    if got == 0:
      break
  return t, (passes, moves)
