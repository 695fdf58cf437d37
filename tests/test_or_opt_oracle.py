"""The Or-opt oracle (`oracle/or_opt.py`) pinned against itself: its vectorised pass against
the plain-loop restatement, and every applied delta against the change of tour length.
The reference has no Or-opt, so these self-consistency checks are its pin."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import distances as odist
from oracle import or_opt as oo


def _lattice(w, h, step=10.0):
  return np.array([[x * step, y * step] for x in range(w) for y in range(h)], dtype=np.float64)


def _tour(rng, n):
  return np.concatenate([[0], 1 + rng.permutation(n - 1)]).astype(np.int32)


@pytest.mark.parametrize("n", [3, 4, 5, 6, 9, 17, 33])
def test_vectorised_pass_equals_loops_and_delta_is_exact(n):
  rng = np.random.default_rng(n)
  coords = rng.uniform(0, 100, (n, 2))
  D = odist.euc2d_matrix(coords)
  for k in sorted({1, 2, min(5, n - 1), n - 1}):
    cand = odist.candidate_list(k, coords=coords)
    for _ in range(6):
      t = _tour(rng, n)
      for S in (1, 2, 3):
        mv, valid = oo.best_move(t, D, cand, S)
        assert mv == oo.best_move_loops(t, D, cand, S)
        assert valid >= 0
        if mv[1] >= 0:
          t2 = oo.apply_move(t, cand, *mv[1:])
          assert sorted(t2.tolist()) == list(range(n)) and t2[0] == t[0]
          assert oo.tour_length(t2, D) - oo.tour_length(t, D) == mv[0] < 0


def test_lattice_ties_follow_the_key_order():
  """On a lattice many moves share the best delta: both restatements take the smallest key."""
  coords = _lattice(5, 6)
  D = odist.euc2d_matrix(coords)
  cand = odist.candidate_list(6, coords=coords)
  rng = np.random.default_rng(3)
  ties = 0
  for _ in range(20):
    t = _tour(rng, len(coords))
    mv, _ = oo.best_move(t, D, cand, 3)
    assert mv == oo.best_move_loops(t, D, cand, 3)
    # count the moves that tie with the chosen one
    n = len(t)
    pos = np.empty(n, dtype=np.int64)
    pos[t] = np.arange(n)
    same = 0
    for i in range(1, n):
      for L in range(1, 4):
        if i + L - 1 > n - 1:
          continue
        for r in range(cand.shape[1]):
          for o in ((0, 1) if L >= 2 else (0,)):
            x = t[i] if o == 0 else t[i + L - 1]
            j = pos[cand[x][r]]
            if i - 1 <= j <= i + L - 1:
              continue
            t2 = oo.apply_move(t, cand, i, L, r, o)
            same += oo.tour_length(t2, D) - oo.tour_length(t, D) == mv[0]
    ties += same > 1
  assert ties > 0


def test_refine_is_monotone_and_counts_passes():
  rng = np.random.default_rng(11)
  coords = rng.uniform(0, 1000, (120, 2))
  D = odist.euc2d_matrix(coords)
  cand = odist.candidate_list(8, coords=coords)
  t = _tour(rng, 120)
  out, passes, moves, evaluated = oo.refine(t, D, cand, 10**6)
  assert passes == moves + 1  # the last pass finds nothing
  assert oo.best_move(out, D, cand, 3)[0][1] == -1
  assert oo.tour_length(out, D) < oo.tour_length(t, D)
  part, p5, m5, _ = oo.refine(t, D, cand, 5)
  assert (p5, m5) == (5, 5)
  assert np.array_equal(oo.refine(part, D, cand, 10**6)[0], out)  # passes compose


def test_three_opt_local_optima_admit_no_improving_or_opt_move():
  """Every Or-opt move removes three edges and reconnects them without a reversal or with
  the segment reversed, i.e. it is one of the seven 3-opt reconnections. A tour refined to a
  local optimum by the 3-opt oracle (pinned to the reference's CPU 3-opt) therefore admits
  no improving Or-opt move, even with full candidate lists."""
  from oracle import three_opt as o3

  rng = np.random.default_rng(21)
  for n in (8, 13, 21, 28):
    coords = rng.uniform(0, 500, (n, 2))
    D = odist.euc2d_matrix(coords)
    full = odist.candidate_list(n - 1, coords=coords)
    t = _tour(rng, n)
    opt, _ = o3.refine(t, D, 10**6)
    assert o3.best_move(opt, D)[0] == 0  # a 3-opt local optimum
    for S in (1, 2, 3):
      assert oo.best_move(opt, D, full, S)[0][1] == -1, (n, S)
    # while a random tour does have improving Or-opt moves
    assert oo.best_move(t, D, full, 3)[0][1] >= 0
