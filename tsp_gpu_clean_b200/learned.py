"""Learned 2-opt candidate lists: an edge-scoring MLP trained on the GPU.

For each city u the pool is its `pool_k` nearest neighbours; a 5 -> 64 -> 64 -> 1 MLP
(BF16 weights, FP32 accumulation, hand-written kernels in `csrc/mlp.cu`) scores every
pool edge from features that plain k-NN ranking ignores (both ranks of the edge, the
direction, the local density scale), and the `k` best-scoring neighbours form the
candidate table handed to 2-opt. Plain k-NN stays the fallback and the yardstick.

Training data: edges of good tours of generated instances. Each training instance gets
nearest-neighbour starts refined to a 2-opt local optimum (best mode, k-NN candidates),
optionally followed by a few generations of the fused memetic GA; the edges of the best
tour are the positives, the other pool edges the negatives.
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import native
from .device import auto_threads, ptr, require_gpu, stream_handle, torch


@dataclass
class InstanceTensors:
  coords: "torch.Tensor"   # (n, 2) float64
  dist: "torch.Tensor | None"  # (n, n) int32 or None (coordinates only)
  pool: "torch.Tensor"     # (n, pool_k) int32
  n: int


def _call(name, *args):
  native.call(name, *args)


def device_instance(coords: np.ndarray, pool_k: int, with_matrix: bool = True) -> InstanceTensors:
  """Coordinates on the device, the EUC_2D matrix (when asked) and the k-NN pool."""
  require_gpu()
  c = torch.from_numpy(np.ascontiguousarray(coords, dtype=np.float64)).cuda()
  n = int(c.shape[0])
  d = None
  if with_matrix:
    d = torch.empty((n, n), dtype=torch.int32, device="cuda")
    _call("tspb_euc2d_matrix", ptr(c), n, ptr(d), n, stream_handle())
  pool = torch.empty((n, pool_k), dtype=torch.int32, device="cuda")
  _call("tspb_knn", ptr(d), n if d is not None else 0, ptr(c) if d is None else None, n, pool_k, ptr(pool),
        stream_handle())
  return InstanceTensors(c, d, pool, n)


def _edge_features(inst: InstanceTensors, tour_pos: "torch.Tensor | None"):
  pk = int(inst.pool.shape[1])
  E = inst.n * pk
  x = torch.empty((E, 16), dtype=torch.int16, device="cuda")
  y = torch.empty(E, dtype=torch.float32, device="cuda") if tour_pos is not None else None
  _call("tspb_edge_features", ptr(inst.coords), inst.n, ptr(inst.pool), pk, ptr(inst.dist),
        inst.n if inst.dist is not None else 0, ptr(tour_pos), ptr(x), ptr(y), stream_handle())
  return x, y


def two_opt_table(inst: InstanceTensors, tours: "torch.Tensor", table: "torch.Tensor", mode: str = "best",
                  max_iterations: int = 10**9) -> tuple["torch.Tensor", np.ndarray]:
  """2-opt of `tours` (in place copy) with an explicit candidate table; returns (tours, stats)."""
  n = inst.n
  k = int(table.shape[1])
  cd = torch.empty((n, k), dtype=torch.int32, device="cuda")
  _call("tspb_candidate_distances", ptr(table), n, k, ptr(inst.dist), n if inst.dist is not None else 0,
        ptr(inst.coords) if inst.dist is None else None, ptr(cd), stream_handle())
  packed = torch.empty((n, k), dtype=torch.int32, device="cuda")
  over = torch.zeros(1, dtype=torch.int32, device="cuda")
  use_packed = n <= 0xFFFF
  if use_packed:
    _call("tspb_candidate_pack", ptr(table), ptr(cd), n, k, ptr(packed), ptr(over), stream_handle())
  t = tours.contiguous().clone()
  num = int(t.shape[0])
  threads = auto_threads(num)
  lib = native.load_library()
  ws_bytes = int(lib.tspb_two_opt_workspace_bytes(num, n, k, native.MODE_CODES[mode], threads))
  ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
  stats = torch.zeros((num, 4), dtype=torch.int64, device="cuda")
  status = torch.zeros(num, dtype=torch.int32, device="cuda")
  if use_packed and int(over.item()) != 0:
    use_packed = False
  native.check("tspb_two_opt", lib.tspb_two_opt(
    ptr(t), num, n, ptr(inst.dist), n if inst.dist is not None else 0, ptr(inst.coords) if inst.dist is None else None,
    ptr(table), ptr(cd), None, None, ptr(packed) if use_packed else None, k,
    native.MODE_CODES[mode] | native.TSPB_MODE_SYMMETRIC, int(max_iterations),  # EUC_2D: symmetric
    threads, ptr(stats), ptr(status), ptr(ws), ws_bytes, stream_handle()))
  if int(status.max().item()) != 0:
    raise RuntimeError("2-opt rejected a start tour")
  return t, stats.cpu().numpy()


def tour_lengths(inst: InstanceTensors, tours: "torch.Tensor") -> np.ndarray:
  out = torch.empty(int(tours.shape[0]), dtype=torch.float64, device="cuda")
  _call("tspb_tour_cost", ptr(tours), int(tours.shape[0]), inst.n, ptr(inst.dist), inst.n if inst.dist is not None else 0,
        ptr(inst.coords) if inst.dist is None else None, 1, ptr(out), stream_handle())
  return out.cpu().numpy()


def double_bridge(tour: "torch.Tensor", count: int, gen: "torch.Generator") -> "torch.Tensor":
  """`count` copies of `tour`, each with one random double-bridge kick: cuts 0 < p1 < p2 <
  p3 < n turn A B C D into A C B D (four edges replaced; position 0 stays first)."""
  n = int(tour.shape[0])
  dev = tour.device
  cuts = torch.randint(1, n, (count, 3), generator=gen)
  while True:  # three distinct cuts per row
    cuts, _ = torch.sort(cuts, dim=1)
    dup = (cuts[:, 0] == cuts[:, 1]) | (cuts[:, 1] == cuts[:, 2])
    if not bool(dup.any()):
      break
    cuts[dup] = torch.randint(1, n, (int(dup.sum()), 3), generator=gen)
  p1, p2, p3 = (cuts[:, c:c + 1].to(dev) for c in range(3))
  j = torch.arange(n, device=dev).unsqueeze(0).expand(count, n)
  lc = p3 - p2
  src = torch.where(j < p1, j, torch.where(j < p1 + lc, p2 + (j - p1), torch.where(j < p3, p1 + (j - p1 - lc), j)))
  return tour.long()[src].to(torch.int32).contiguous()


def iterated_two_opt(inst: InstanceTensors, starts: "torch.Tensor", table: "torch.Tensor", budget_s: float,
                     kicks: int, seed: int, spent_s: float = 0.0) -> dict:
  """Iterated 2-opt with double-bridge kicks under a device-time budget.

  The starts are refined to a 2-opt local optimum (best mode, this candidate table); then,
  while the CUDA-event time used is below `budget_s`, the best tour so far gets `kicks`
  kicked copies, all refined in one launch, and the shortest replaces it when shorter.
  `spent_s` is time already used (for example building the table). Returns the best
  length, the time used and the rounds run."""
  gen = torch.Generator().manual_seed(seed)

  def timed(fn):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1) / 1e3

  (t, _), used = timed(lambda: two_opt_table(inst, starts, table, mode="best"))
  used += spent_s
  lengths = tour_lengths(inst, t)
  best_i = int(np.argmin(lengths))
  best, best_len = t[best_i].clone(), float(lengths[best_i])
  rounds = 0
  while used < budget_s:
    def one_round():
      kicked = double_bridge(best, kicks, gen)
      out, _ = two_opt_table(inst, kicked, table, mode="best")
      return out, tour_lengths(inst, out)
    (out, ls), dt = timed(one_round)
    used += dt
    rounds += 1
    i = int(np.argmin(ls))
    if float(ls[i]) < best_len:
      best, best_len = out[i].clone(), float(ls[i])
  return {"length": best_len, "used_s": used, "rounds": rounds, "tour": best}


def random_starts(n: int, count: int, seed: int) -> "torch.Tensor":
  rng = np.random.default_rng(seed)
  return torch.from_numpy(np.stack([rng.permutation(n) for _ in range(count)]).astype(np.int32)).cuda()


def nn_starts(inst: InstanceTensors, count: int, seed: int) -> "torch.Tensor":
  """GRASP nearest-neighbour starts over the pool (the NN-init kernel with the k-NN pool)."""
  n = inst.n
  k = min(5, int(inst.pool.shape[1]))
  cand = inst.pool[:, :k].contiguous()
  seeds = np.random.default_rng(seed).integers(0, np.iinfo(np.int64).max, size=count, dtype=np.int64)
  d_seeds = torch.from_numpy(seeds).cuda()
  cust = torch.arange(n, dtype=torch.int32, device="cuda")
  need = count * (2 * n + k) * 4
  ws = torch.empty(need // 4 + 1, dtype=torch.int32, device="cuda")
  out = torch.empty((count, n), dtype=torch.int32, device="cuda")
  _call("tspb_nn_init", ptr(cust), n, ptr(cand), n, k, ptr(d_seeds), count, n - 1, ptr(ws), need, ptr(out), stream_handle())
  return out


class EdgeScorer:
  """The MLP parameters (FP32 masters on the device) and their Adam state."""

  def __init__(self, seed: int = 0) -> None:
    require_gpu()
    lib = native.load_library()
    self.count = int(lib.tspb_mlp_param_count())
    rng = np.random.default_rng(seed)
    p = np.zeros(self.count, dtype=np.float32)
    H, KX = 64, 16
    o_w1, o_b1 = 0, KX * H
    o_w2, o_b2 = o_b1 + H, o_b1 + H + H * H
    o_w3, o_b3 = o_b2 + H, o_b2 + 2 * H
    p[o_w1 : o_w1 + 5 * H] = rng.normal(0, np.sqrt(2 / 5), 5 * H)
    p[o_w2 : o_w2 + H * H] = rng.normal(0, np.sqrt(2 / H), H * H)
    p[o_w3 : o_w3 + H] = rng.normal(0, np.sqrt(1 / H), H)
    p[o_b3] = -2.0  # positives are ~2 of every pool_k edges
    self.params = torch.from_numpy(p).cuda()
    self.grad = torch.zeros_like(self.params)
    self.m = torch.zeros_like(self.params)
    self.v = torch.zeros_like(self.params)
    self.step = 0
    #: gradient on the tcgen05 tensor cores (accumulators in tensor memory); False: the
    #: mma.sync kernel with the same rounding points except dh1, kept as its cross-check
    self.tensor_cores = True
    self._status = torch.zeros(1, dtype=torch.int32, device="cuda")

  def logits(self, x: "torch.Tensor") -> "torch.Tensor":
    E = int(x.shape[0])
    out = torch.empty(E, dtype=torch.float32, device="cuda")
    _call("tspb_mlp_infer", ptr(self.params), ptr(x), E, ptr(out), stream_handle())
    return out

  def train_step(self, x: "torch.Tensor", y: "torch.Tensor", lr: float = 3e-3) -> float:
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    E = int(x.shape[0])
    if self.tensor_cores:
      _call("tspb_mlp_train_grad_tc", ptr(self.params), ptr(x), ptr(y), E, ptr(self.grad), ptr(loss),
            ptr(self._status), stream_handle())
    else:
      _call("tspb_mlp_train_grad", ptr(self.params), ptr(x), ptr(y), E, ptr(self.grad), ptr(loss), stream_handle())
    self.step += 1
    _call("tspb_mlp_adam", ptr(self.params), ptr(self.grad), ptr(self.m), ptr(self.v), self.step, lr, 0.9, 0.999, 1e-8,
          0.0, stream_handle())
    if self.tensor_cores and int(self._status.item()) != 0:
      raise RuntimeError(f"tspb_mlp_train_grad_tc: {native.status_text(int(self._status.item()))}")
    return float(loss.item()) / max(E, 1)


class LearnedCandidates:
  """Train the scorer on good tours; emit learned top-k candidate tables."""

  def __init__(self, pool_k: int = 30, seed: int = 0) -> None:
    self.pool_k = pool_k
    self.scorer = EdgeScorer(seed)
    self.train_log: list[float] = []

  # ---------------------------------------------------------------- data
  def label_tour(self, inst: InstanceTensors, starts: int = 4, seed: int = 0, ga_generations: int = 0):
    """Best 2-opt local optimum (k-NN 20 candidates) of `starts` nearest-neighbour starts."""
    knn = inst.pool[:, : min(20, self.pool_k)].contiguous()
    tours, _ = two_opt_table(inst, nn_starts(inst, starts, seed), knn, mode="best")
    lengths = tour_lengths(inst, tours)
    best = tours[int(np.argmin(lengths))]
    if ga_generations > 0:
      best = self._ga_refine(inst, best, ga_generations, seed)
    return best

  def _ga_refine(self, inst, tour, generations, seed):
    from .fused import FusedMemeticSolver, LocalSearchConfig
    from .problem import Problem, ProblemContext

    coords = inst.coords.cpu().numpy()
    ctx = ProblemContext(Problem.from_coordinates(coords), seed=seed,
                         candidate_cache={5: inst.pool[:, :5].cpu().numpy(), 20: inst.pool[:, :20].cpu().numpy()})
    solver = FusedMemeticSolver(population_size=16, mutation_rate=0.1, elite_count=4, post_init=True,
                                local_search=LocalSearchConfig("best", 50, 20), chunk=8)
    best, _ = solver.evolve(ctx, list(range(inst.n)), generations, patience=10**9)
    cur = tour_lengths(inst, tour[None, :])[0]
    cand = torch.from_numpy(best).cuda()
    return cand if tour_lengths(inst, cand[None, :])[0] < cur else tour

  def training_edges(self, inst: InstanceTensors, tour: "torch.Tensor"):
    pos = torch.empty(inst.n, dtype=torch.int32, device="cuda")
    pos[tour.long()] = torch.arange(inst.n, dtype=torch.int32, device="cuda")
    return _edge_features(inst, pos)

  # ---------------------------------------------------------------- training
  def fit(self, xs: list, ys: list, epochs: int = 3, batch: int = 1 << 16, lr: float = 3e-3, seed: int = 0) -> float:
    X = torch.cat(xs)
    Y = torch.cat(ys)
    E = int(X.shape[0])
    nb = max(1, (E + batch - 1) // batch)
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    for ep in range(epochs):
      for b in rng.permutation(nb):
        s, e = int(b) * batch, min(E, (int(b) + 1) * batch)
        self.train_log.append(self.scorer.train_step(X[s:e], Y[s:e], lr))
    torch.cuda.synchronize()
    return time.perf_counter() - t0

  # ---------------------------------------------------------------- inference
  def table(self, inst: InstanceTensors, k: int) -> "torch.Tensor":
    x, _ = _edge_features(inst, None)
    logits = self.scorer.logits(x)
    out = torch.empty((inst.n, k), dtype=torch.int32, device="cuda")
    _call("tspb_select_topk", ptr(inst.pool), ptr(logits), inst.n, int(inst.pool.shape[1]), k, ptr(out), stream_handle())
    return out


def edge_recall(table: "torch.Tensor", tour: "torch.Tensor") -> float:
  """Fraction of the tour's edges (u, next u) whose endpoint is in u's candidate row, both directions."""
  n = int(tour.shape[0])
  t = tour.long()
  nxt = torch.roll(t, -1)
  prv = torch.roll(t, 1)
  rows = table[t.long()].long()
  hit_n = (rows == nxt[:, None]).any(dim=1)
  hit_p = (rows == prv[:, None]).any(dim=1)
  return float((hit_n.float().mean() + hit_p.float().mean()).item() / 2.0)
