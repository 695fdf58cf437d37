"""NumPy restatement of the reference's population operators (TSP, open permutations).

- `sample_distinct_pairs`: `src/utils/route_helpers.py:74-108`.
- `tournament_select`: `SelectionCPUTournament.select_batch`,
  `src/algorithms/strategies/selection/tournament_selection.py:98-128`.
- `pmx_child` / `pmx_batch`: `CrossoverCPUPermPartiallyMapped._apply_pmx` and
  `crossover_batch`, `src/algorithms/strategies/crossover/pmx_crossover.py:49-105, 128-171`.
- `inversion_batch`: `MutationCPUPermInversion.mutate_batch`,
  `src/algorithms/strategies/mutation/inversion_mutation.py:65-99`.
- `tour_cost`: `evaluate_tour_cpu`, `src/algorithms/strategies/evaluation/tour_cost.py:17-29`.
- `survivors`: `GeneticAlgorithm._select_survivors_assessed` for feasible tours,
  `src/algorithms/metaheuristics/genetic_algorithm.py:618-706`.
- `elite_indices`: `EliteOnlyLocalSearchStep.run`, `src/algorithms/pipeline_steps.py:153-163`.
- `splitmix64_*`, `draw_row_seeds`, `nn_row`, `nn_init`: `src/utils/splitmix64.py:21-51` and
  `src/algorithms/strategies/initialization/nearest_neighbor_init.py:31-132`.

Every random draw is taken from the generator passed in, in the reference's order.
Test infrastructure only (see the package docstring).
"""

from __future__ import annotations

import numpy as np


def sample_distinct_pairs(rng: np.random.Generator, num_pairs: int, low: int, high: int) -> np.ndarray:
  """Ordered distinct pairs from `[low, high)` via `v = v' + (v' >= u)`."""
  if high - low < 2:
    raise ValueError(f"Need at least two distinct integers in [{low}, {high})")
  if num_pairs <= 0:
    return np.empty((0, 2), dtype=np.int32)
  first = rng.integers(low, high, size=num_pairs, dtype=np.int32)
  shifted = rng.integers(low, high - 1, size=num_pairs, dtype=np.int32)
  second = shifted + (shifted >= first).astype(np.int32)
  return np.stack((first, second), axis=1).astype(np.int32, copy=False)


def tournament_draw(rng, pop_size: int, num_parents: int, k: int) -> np.ndarray:
  """The `(num_parents, k)` competitor draw (`tournament_selection.py:113`)."""
  return rng.integers(0, pop_size, size=(num_parents, k), dtype=np.int32)


def tournament_winners(fitness: np.ndarray, cand: np.ndarray) -> np.ndarray:
  """First argmin of fitness over each row of competitors (`:125-127`)."""
  fit = np.asarray(fitness, dtype=np.float64)
  cols = np.argmin(fit[cand], axis=1)
  return cand[np.arange(cand.shape[0]), cols]


def tournament_select(rng, routes: np.ndarray, fitness: np.ndarray, num_parents: int | None, k: int) -> np.ndarray:
  pop = np.asarray(routes)
  n_sel = len(pop) if num_parents is None else num_parents
  cand = tournament_draw(rng, len(pop), n_sel, k)
  return pop[tournament_winners(fitness, cand)].copy()


def pmx_child(p1: np.ndarray, p2: np.ndarray, c1: int, c2: int) -> np.ndarray:
  """One PMX child for an open permutation (`pmx_crossover.py:49-105`, `is_closed=False`)."""
  n = len(p1)
  if n <= 1:
    return p1.copy()
  if c1 > c2:
    c1, c2 = c2, c1
  child = np.full(n, -1, dtype=np.int32)
  child[c1 : c2 + 1] = p1[c1 : c2 + 1]
  max_node = max(n, int(p1.max()) + 1, int(p2.max()) + 1)
  inv_p2 = np.full(max_node, -1, dtype=np.int32)
  inv_p2[p2] = np.arange(n, dtype=np.int32)
  in_seg = np.zeros(max_node, dtype=bool)
  in_seg[p1[c1 : c2 + 1]] = True
  seg_len = c2 - c1 + 1
  for idx in range(c1, c2 + 1):
    val = int(p2[idx])
    if val >= 0 and not in_seg[val]:
      pos = idx
      steps = 0
      while c1 <= pos <= c2 and steps <= seg_len:
        mv = int(p1[pos])
        if mv < 0:
          break
        nxt = int(inv_p2[mv])
        if nxt < 0:
          break
        pos = nxt
        steps += 1
      if 0 <= pos < n and (pos < c1 or pos > c2):
        child[pos] = val
  unmapped = child == -1
  child[unmapped] = p2[unmapped]
  return child


def pmx_cuts(rng, num_routes: int, n: int) -> np.ndarray:
  """The `(num_routes // 2, 2)` cut draw (`pmx_crossover.py:153-155`)."""
  return sample_distinct_pairs(rng, num_routes // 2, 0, n)


def pmx_apply(batch: np.ndarray, pairs: np.ndarray) -> np.ndarray:
  """Children of pairs `(2k, 2k+1)` sharing cuts; odd tail copied (`:157-171`)."""
  batch = np.asarray(batch, dtype=np.int32)
  out = np.empty_like(batch)
  for kk in range(len(batch) // 2):
    i = 2 * kk
    c1 = int(min(pairs[kk, 0], pairs[kk, 1]))
    c2 = int(max(pairs[kk, 0], pairs[kk, 1]))
    out[i] = pmx_child(batch[i], batch[i + 1], c1, c2)
    out[i + 1] = pmx_child(batch[i + 1], batch[i], c1, c2)
  if len(batch) % 2 == 1:
    out[-1] = batch[-1]
  return out


def pmx_batch(rng, batch: np.ndarray) -> np.ndarray:
  batch = np.asarray(batch, dtype=np.int32)
  if batch.ndim == 1 or len(batch) < 2 or batch.shape[1] < 2:
    return batch.copy()
  return pmx_apply(batch, pmx_cuts(rng, len(batch), batch.shape[1]))


def ox_child(p1: np.ndarray, p2: np.ndarray, c1: int, c2: int) -> np.ndarray:
  """One Order Crossover child of open permutations (`order_crossover.py:52-83`,
  `is_closed=False`): the child keeps p1[c1..c2]; the free positions c2+1, ..., n-1, 0,
  ..., c1-1 take, in this order, the genes of p2 read from index c2+1 onward (wrapping)
  that are not in the kept segment."""
  n = len(p1)
  if n <= 1:
    return p1.copy()
  if c1 > c2:
    c1, c2 = c2, c1
  child = np.full(n, -1, dtype=np.int32)
  child[c1 : c2 + 1] = p1[c1 : c2 + 1]
  kept = set(int(v) for v in p1[c1 : c2 + 1])
  dst = (c2 + 1) % n
  for t in range(n):
    gene = int(p2[(c2 + 1 + t) % n])
    if gene in kept:
      continue
    while child[dst] != -1:  # only the kept segment is pre-filled
      dst = (dst + 1) % n
    child[dst] = gene
    dst = (dst + 1) % n
  return child


def ox_apply(batch: np.ndarray, pairs: np.ndarray) -> np.ndarray:
  """OX children of pairs `(2k, 2k+1)` sharing cuts; odd tail copied (`order_crossover.py:150-168`)."""
  batch = np.asarray(batch, dtype=np.int32)
  out = np.empty_like(batch)
  for kk in range(len(batch) // 2):
    i = 2 * kk
    c1 = int(min(pairs[kk, 0], pairs[kk, 1]))
    c2 = int(max(pairs[kk, 0], pairs[kk, 1]))
    out[i] = ox_child(batch[i], batch[i + 1], c1, c2)
    out[i + 1] = ox_child(batch[i + 1], batch[i], c1, c2)
  if len(batch) % 2 == 1:
    out[-1] = batch[-1]
  return out


def ox_batch(rng, batch: np.ndarray) -> np.ndarray:
  """`CrossoverCPUPermOrder.crossover_batch` (`order_crossover.py:127-168`): the cut pairs
  are drawn exactly as PMX draws them."""
  batch = np.asarray(batch, dtype=np.int32)
  if batch.ndim == 1 or len(batch) < 2 or batch.shape[1] < 2:
    return batch.copy()
  return ox_apply(batch, pmx_cuts(rng, len(batch), batch.shape[1]))


def swap_apply(batch: np.ndarray, rate: float, u, p1, p2) -> np.ndarray:
  """Swap of positions p1[r], p2[r] in every row with u[r] < rate (`swap_mutation.py:94-99`)."""
  out = np.asarray(batch, dtype=np.int32).copy()
  for r in np.flatnonzero(np.asarray(u) < rate):
    a, b = int(p1[r]), int(p2[r])
    out[r, a], out[r, b] = out[r, b], out[r, a]
  return out


def swap_batch(rng, batch: np.ndarray, rate: float) -> np.ndarray:
  """`MutationCPUPermSwap.mutate_batch` (`swap_mutation.py:65-99`, uniform positions): the
  draws are those of inversion (u, then a distinct position pair per row)."""
  batch = np.asarray(batch, dtype=np.int32)
  if batch.shape[1] < 2:
    return batch.copy()
  u, p1, p2 = inversion_draw(rng, len(batch), batch.shape[1])
  return swap_apply(batch, rate, u, p1, p2)


def inversion_draw(rng, num_routes: int, n: int):
  """`u = random(N)` then the position pairs (`inversion_mutation.py:82-91`)."""
  u = rng.random(num_routes)
  pairs = sample_distinct_pairs(rng, num_routes, 0, n)
  return u, pairs[:, 0].copy(), pairs[:, 1].copy()


def inversion_apply(batch: np.ndarray, rate: float, u, p1, p2) -> np.ndarray:
  out = np.array(batch, dtype=np.int32, copy=True)
  for i in np.flatnonzero(u < rate):
    s = int(min(p1[i], p2[i]))
    e = int(max(p1[i], p2[i]))
    out[i, s : e + 1] = out[i, s : e + 1][::-1]
  return out


def inversion_batch(rng, batch: np.ndarray, rate: float) -> np.ndarray:
  batch = np.asarray(batch, dtype=np.int32)
  if batch.shape[1] < 2:
    return batch.copy()
  u, p1, p2 = inversion_draw(rng, len(batch), batch.shape[1])
  return inversion_apply(batch, rate, u, p1, p2)


def tour_cost(batch: np.ndarray, D: np.ndarray, return_to_depot: bool = True) -> np.ndarray:
  """Closed-tour cost in float64 (`tour_cost.py:17-29`)."""
  batch = np.asarray(batch)
  if batch.ndim == 1:
    batch = batch.reshape(1, -1)
  nrows, n = batch.shape
  if nrows == 0 or n <= 1:
    return np.zeros(nrows, dtype=np.float64)
  flat = D.ravel()
  stride = D.shape[1]
  costs = flat[batch[:, :-1] * stride + batch[:, 1:]].sum(axis=1, dtype=np.float64)
  if return_to_depot:
    costs += flat[batch[:, -1] * stride + batch[:, 0]]
  return costs


def survivors(old_pop, old_fit, new_pop, new_fit, population_size: int):
  """Stable `(mu + lambda)` survival on `lexsort` of the objective (`genetic_algorithm.py:628-706`)."""
  pop = np.vstack([old_pop, new_pop])
  obj = np.concatenate([np.asarray(old_fit, np.float64), np.asarray(new_fit, np.float64)])
  zeros = np.zeros_like(obj)
  idx = np.lexsort(np.vstack([obj, zeros, zeros]))[:population_size]
  return pop[idx], obj[idx], idx


def elite_indices(fitness: np.ndarray, k: int) -> np.ndarray:
  """`argsort(fitness)[:k]` with NumPy's default (unstable) sort (`pipeline_steps.py:163`)."""
  return np.argsort(fitness)[: min(k, len(fitness))]


MASK64 = 0xFFFFFFFFFFFFFFFF


def splitmix64_bounded(state: int, bound: int) -> tuple[int, int]:
  """One SplitMix64 step and the high-32 bounded draw (`splitmix64.py:38-51`)."""
  s = (state + 0x9E3779B97F4A7C15) & MASK64
  z = ((s ^ (s >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
  z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
  z = (z ^ (z >> 31)) & MASK64
  return s, ((z >> 32) * bound) >> 32


def draw_row_seeds(rng, population_size: int) -> np.ndarray:
  """`splitmix64.py:21-25`."""
  if population_size <= 0:
    return np.empty(0, dtype=np.uint64)
  return rng.integers(0, np.iinfo(np.int64).max, size=population_size, dtype=np.int64).view(np.uint64)


def nn_row(customers: np.ndarray, cand: np.ndarray, seed: int) -> np.ndarray:
  """GRASP nearest-neighbour row (`nearest_neighbor_init.py:31-99`)."""
  n = int(customers.size)
  if n == 0:
    return np.empty(0, dtype=np.int32)
  max_node = int(customers.max())
  rows = int(cand.shape[0])
  k = int(cand.shape[1]) if cand.ndim == 2 else 0
  unv = customers.astype(np.int64).copy()
  pos = np.full(max_node + 1, -1, dtype=np.int64)
  pos[unv] = np.arange(n)
  st = int(seed)
  rem = n
  out = np.empty(n, dtype=np.int32)
  st, s = splitmix64_bounded(st, rem)
  cur = int(unv[s])
  out[0] = cur
  last = rem - 1
  ln = int(unv[last])
  unv[s] = ln
  unv[last] = cur
  pos[ln] = s
  pos[cur] = last
  rem = last
  order = list(range(k))
  for step_i in range(1, n):
    chosen = -1
    if 0 <= cur < rows and k > 0:
      order = list(range(k))
      crow = cand[cur]
      for i in range(k):
        st, off = splitmix64_bounded(st, k - i)
        j = i + off
        order[i], order[j] = order[j], order[i]
        nb = int(crow[order[i]])
        if 0 <= nb <= max_node:
          p = int(pos[nb])
          if 0 <= p < rem:
            chosen = nb
            break
    if chosen < 0:
      st, u = splitmix64_bounded(st, rem)
      chosen = int(unv[u])
    out[step_i] = chosen
    p = int(pos[chosen])
    last = rem - 1
    ln = int(unv[last])
    unv[p] = ln
    unv[last] = chosen
    pos[ln] = p
    pos[chosen] = last
    rem = last
    cur = chosen
  return out


def random_init(rng, customers, population_size: int) -> np.ndarray:
  """`InitializationCPUPermRandom.initialize` (`random_init.py:30-55`): row seeds as for the
  nearest-neighbour init, then per row a Fisher-Yates shuffle of `customers` from the
  last position down to 1, position i swapped with a SplitMix64 draw in [0, i]. The
  SplitMix64 state advances by its constant increment each step, so step t of a row uses
  state seed + t * increment; all rows advance together here."""
  cust = np.asarray(customers, dtype=np.int32)
  seeds = draw_row_seeds(rng, population_size)
  n = cust.size
  pop = np.tile(cust, (population_size, 1)).astype(np.int32)
  if population_size == 0 or n == 0:
    return pop.reshape(population_size, n)
  rows = np.arange(population_size)
  state = seeds.astype(np.uint64)
  with np.errstate(over="ignore"):
    for i in range(n - 1, 0, -1):
      state = state + np.uint64(0x9E3779B97F4A7C15)
      z = (state ^ (state >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
      z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
      z = z ^ (z >> np.uint64(31))
      j = (((z >> np.uint64(32)) * np.uint64(i + 1)) >> np.uint64(32)).astype(np.intp)
      a = pop[:, i].copy()
      pop[:, i] = pop[rows, j]
      pop[rows, j] = a
  return pop


def nn_init(rng, customers, population_size: int, cand: np.ndarray) -> np.ndarray:
  """`InitializationCPUTourNearestNeighbor.initialize` (`nearest_neighbor_init.py:109-132`)."""
  cust = np.asarray(customers, dtype=np.int32)
  seeds = draw_row_seeds(rng, population_size)
  if population_size == 0 or cust.size == 0:
    return np.empty((population_size, cust.size), dtype=np.int32)
  return np.stack([nn_row(cust, cand, int(s)) for s in seeds]).astype(np.int32)
