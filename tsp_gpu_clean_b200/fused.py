"""Device-resident memetic GA with every generation replayed from a captured CUDA graph.

`FusedMemeticSolver.evolve` computes exactly what the reference's

    GeneticAlgorithm(population_size=P, mutation_rate=rate,
                     initialization=InitializationCPUTourNearestNeighbor(k=nn_k),
                     selection=SelectionCPUTournament(k=tournament_k),
                     crossover=CrossoverCPUPermPartiallyMapped(), mutation=MutationCPUPermInversion(),
                     evaluation=EvaluationCPUCost(), local_search=LocalSearchCPUTourTwoOpt(...),
                     local_search_stage="none",
                     pipeline=[PostInitLocalSearchStep(...), EliteOnlyLocalSearchStep(..., elite_count=k)])
    .evolve(context, customers, max_generations, patience=...)

computes (`src/algorithms/metaheuristics/genetic_algorithm.py:789-965`,
`src/algorithms/pipeline_steps.py:85-195`): same final population, fitness, best tour,
convergence history and final RNG state.

How: the row seeds and every generation's random draws are taken from `context.rng` in
the reference's order before the loop (no draw depends on tour data) and uploaded as a
tape. One generation is five launches - fused offspring (tournament + PMX + inversion +
length), survival, elite 2-opt on survivor rows [0, k), elite re-cost, best tracking -
captured once per population buffer parity into a CUDA graph and replayed in chunks.

Elites: survivors come out sorted by (fitness, index), so `argsort(fitness)[:k]` is the
first k rows unless the k-th and (k+1)-th fitness tie; then membership follows NumPy's
unstable sort, which only the host can reproduce. Once duplicate tours fill the
population such ties are common (46 of 50 generations of the 100-city run). The
survival kernel pauses the run on a tie (device flag; every later launch of the chunk is
a no-op); the host reads the fitness vector, takes `np.argsort`, runs that generation's
elite step and resumes, with the replay chunk shrinking to one generation after a pause
and doubling back while no tie occurs.
Early stop: the tracking kernel sets a device stop flag when patience runs out; later
launches (the 2-opt through `tspb_two_opt_gated`) become no-ops, and the RNG is rewound
to its state after the last generation that ran.
"""

from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass
from typing import Any

import numpy as np

from . import native
from .device import auto_threads, candidate_list, operands_for, ptr, require_gpu, stream_handle, torch
from .problem import resolve_rng
from .routes import sample_distinct_pairs
from .strategies.initialization import InitializationB200TourNearestNeighbor


class GeneratorStates:
  """Generator state after each generation of a natively drawn tape, as bit_generator.state
  dicts on demand."""

  def __init__(self, raw):
    self.raw = raw

  def __len__(self) -> int:
    return len(self.raw)

  def __getitem__(self, g: int) -> dict:
    return self.raw[g].to_state()


def draw_generation_tape(rng: np.random.Generator, G: int, P: int, kt: int, n: int):
  """`draw_generation_tape_numpy`'s draws and end state, computed by libtspb's restatement
  of NumPy's PCG64 stream (`tspb_tape_draw_host`) when `rng` is a PCG64 generator, else
  by NumPy itself."""
  g = native.Pcg64.from_state(rng.bit_generator.state)
  if g is None or n < 2 or P < 2 or G <= 0:
    return draw_generation_tape_numpy(rng, G, P, kt, n)
  arrs = (np.empty((G, P, kt), np.int32), np.empty((G, P // 2), np.int32), np.empty((G, P // 2), np.int32),
          np.empty((G, P), np.float64), np.empty((G, P), np.int32), np.empty((G, P), np.int32))
  raw = (native.Pcg64 * G)()
  native.call("tspb_tape_draw_host", ctypes.byref(g), G, P, kt, n,
              *[a.ctypes.data_as(ctypes.c_void_p) for a in arrs], raw)
  rng.bit_generator.state = g.to_state()
  return arrs, GeneratorStates(raw)


def draw_generation_tape_numpy(rng: np.random.Generator, G: int, P: int, kt: int, n: int):
  """Random draws of G generations from `rng` in the reference's order.

  Per generation: tournament contestants (P, kt) (`tournament_selection.py:113`), PMX cut
  pairs for P/2 pairs (`pmx_crossover.py:155`), inversion u (P) (`inversion_mutation.py:82`)
  and inversion position pairs (P) (`route_helpers.py:214`). Returns the six tape arrays
  (tourn, cut_a, cut_b, u, inv_a, inv_b), each with a leading G axis, and the generator
  state after each generation (to rewind the generator after an early stop).
  """
  tourn = np.empty((G, P, kt), dtype=np.int32)
  cut_a = np.empty((G, P // 2), dtype=np.int32)
  cut_b = np.empty((G, P // 2), dtype=np.int32)
  u = np.empty((G, P), dtype=np.float64)
  inv_a = np.empty((G, P), dtype=np.int32)
  inv_b = np.empty((G, P), dtype=np.int32)
  states = []
  for g in range(G):
    tourn[g] = rng.integers(0, P, size=(P, kt), dtype=np.int32)
    pairs = sample_distinct_pairs(rng, P // 2, 0, n)
    cut_a[g], cut_b[g] = pairs[:, 0], pairs[:, 1]
    u[g] = rng.random(P)
    pos = sample_distinct_pairs(rng, P, 0, n)
    inv_a[g], inv_b[g] = pos[:, 0], pos[:, 1]
    states.append(rng.bit_generator.state)
  return (tourn, cut_a, cut_b, u, inv_a, inv_b), states


def trailing_stall(history: list) -> int:
  """Generations since the last strict improvement: the best-so-far history changes only on
  an improvement larger than 1e-6, so this is the count of trailing unchanged entries."""
  k = 0
  for a, b in zip(reversed(history[:-1]), reversed(history[1:])):
    if a != b:
      break
    k += 1
  return k


@dataclass
class LocalSearchConfig:
  mode: str = "best"
  max_iterations: int = 10
  candidate_k: int | None = 20
  threads: int = 0  # 0: chosen per launch from the batch size


class FusedMemeticSolver:
  def __init__(self, population_size: int = 128, mutation_rate: float = 0.05, tournament_k: int = 5, nn_k: int = 5,
               local_search: LocalSearchConfig | None = None, elite_count: int = 16, post_init: bool = True,
               use_graph: bool = True, chunk: int = 16, max_matrix_dimension: int | None = None,
               engine: str = "batch", crossover: str = "pmx", mutation: str = "inversion", init: str = "nn",
               local_search_stage: str = "none") -> None:
    if population_size < 2:
      raise ValueError("population_size must be >= 2")
    if engine not in ("batch", "single"):
      raise ValueError("engine must be 'batch' (the multi-instance engine with one run) or 'single'")
    if crossover not in ("pmx", "ox") or mutation not in ("inversion", "swap"):
      raise ValueError("crossover must be 'pmx' or 'ox', mutation 'inversion' or 'swap'")
    if init not in ("nn", "random") or local_search_stage not in ("none", "post_mutation"):
      raise ValueError("init must be 'nn' or 'random', local_search_stage 'none' or 'post_mutation'")
    if engine == "single" and (crossover, mutation, init, local_search_stage) != ("pmx", "inversion", "nn", "none"):
      raise ValueError("the single-run engine runs NN init, PMX and inversion with the elite/post-init steps; "
                       "use engine='batch' for OX, swap, random init or the post_mutation stage")
    self.engine = engine
    self.crossover, self.mutation = crossover, mutation
    self.init, self.stage = init, local_search_stage
    self.P = population_size
    self.rate = mutation_rate
    self.kt = tournament_k
    self.nn_k = nn_k
    self.ls = local_search if local_search is not None else LocalSearchConfig()
    self.host_elite_generations = 0
    self.elite = min(elite_count, population_size) if elite_count else 0
    self.post_init = post_init
    self.use_graph = use_graph
    self.chunk = max(1, chunk)
    self.max_matrix_dimension = max_matrix_dimension
    self.kernel_launches = 0
    self.last_timing: dict[str, float] = {}

  # -------------------------------------------------------------------------- tape
  def _draw_tape(self, rng: np.random.Generator, G: int, n: int):
    return draw_generation_tape(rng, G, self.P, self.kt, n)

  # -------------------------------------------------------------------------- launches
  def _two_opt(self, rows_ptr, num, skip=None):
    ls = self.ls
    lib = native.load_library()
    mode = native.MODE_CODES[ls.mode] | (native.TSPB_MODE_SYMMETRIC if self.symmetric else 0)
    threads = int(ls.threads) if ls.threads else auto_threads(num)
    rc = lib.tspb_two_opt_gated(ptr(skip if skip is not None else self.d_zero), rows_ptr, num, self.n, ptr(self.dist),
                                self.stride, ptr(self.coords), ptr(self.cand), ptr(self.cand_dist), None, None,
                                ptr(self.packed), self.k, mode, int(ls.max_iterations), threads, None,
                                ptr(self.ls_status), ptr(self.ws), self.ws_bytes, stream_handle())
    native.check("tspb_two_opt_gated", rc)

  def _generation(self, parity: int) -> None:
    """Enqueue one generation reading buffer `parity`, writing buffer `1 - parity`."""
    lib = native.load_library()
    src, dst = self.pop[parity], self.pop[1 - parity]
    fsrc, fdst = self.fit[parity], self.fit[1 - parity]
    t = self.tape
    sh = stream_handle()
    native.check("offspring", lib.tspb_generation_offspring(
      ptr(src), ptr(fsrc), self.P, self.n, self.kt, ptr(t[0]), ptr(t[1]), ptr(t[2]), ptr(t[3]), ptr(t[4]), ptr(t[5]),
      float(self.rate), ptr(self.dist), self.stride, ptr(self.coords), ptr(self.gen), ptr(self.stopped), ptr(self.off),
      ptr(self.off_fit), sh))
    native.check("survival", lib.tspb_generation_survival(
      ptr(src), ptr(fsrc), ptr(self.off), ptr(self.off_fit), self.P, self.n, self.elite, ptr(self.gen), ptr(self.stopped),
      ptr(self.order), ptr(dst), ptr(fdst), ptr(self.ties), sh))
    if self.elite:
      self._two_opt(ptr(dst), self.elite, skip=self.stopped)
      native.check("elite_cost", lib.tspb_generation_elite_cost(
        ptr(dst), self.elite, self.n, ptr(self.dist), self.stride, ptr(self.coords), ptr(self.stopped), ptr(fdst), sh))
    native.check("track", lib.tspb_generation_track(
      ptr(fdst), ptr(dst), self.P, self.n, ptr(self.gen), ptr(self.stopped), ptr(self.stall), int(self.patience),
      ptr(self.best_cost), ptr(self.best_tour), ptr(self.history), ptr(self.done), sh))
    self.kernel_launches += 7 if self.elite else 4

  def _host_elites(self, gen: int) -> None:
    """Elite step of paused generation `gen`: membership from the host `np.argsort`."""
    lib = native.load_library()
    dst = self.pop[(gen + 1) % 2]
    fdst = self.fit[(gen + 1) % 2]
    sh = stream_handle()
    self.stopped.zero_()
    idx = np.argsort(fdst.cpu().numpy())[: self.elite].astype(np.int32)  # pipeline_steps.py:163
    d_idx = torch.from_numpy(idx).cuda()
    tmp = self.elite_tmp
    native.call("tspb_gather_rows", ptr(dst), self.P, self.n, ptr(d_idx), self.elite, ptr(tmp), sh)
    self._two_opt(ptr(tmp), self.elite)
    costs = self.elite_costs
    native.call("tspb_tour_cost", ptr(tmp), self.elite, self.n, ptr(self.dist), self.stride, ptr(self.coords), 1,
                ptr(costs), sh)
    native.call("tspb_scatter_rows", ptr(tmp), self.elite, self.n, ptr(d_idx), ptr(dst), self.P, sh)
    fdst[d_idx.long()] = costs
    native.check("track", lib.tspb_generation_track(
      ptr(fdst), ptr(dst), self.P, self.n, ptr(self.gen), ptr(self.stopped), ptr(self.stall), int(self.patience),
      ptr(self.best_cost), ptr(self.best_tour), ptr(self.history), ptr(self.done), sh))
    self.kernel_launches += 5
    self.host_elite_generations += 1

  # -------------------------------------------------------------------------- evolve
  def evolve(self, context: Any, customers: Any, max_generations: int, patience: int | None = None,
             optimal_cost: float | None = None):
    """One GA run; returns (best_tour, stats) like `GeneticAlgorithm.evolve`
    (`genetic_algorithm.py:789-965`). `optimal_cost` (batch engine) stops the run when its
    best reaches the known optimum or comes within 1 % of it."""
    require_gpu()
    t_start = time.perf_counter()
    n = len(customers)
    if n < 4 or n != int(context.dimension) or list(customers) != list(range(n)):
      raise ValueError("FusedMemeticSolver needs the full tour customers = range(dimension) with dimension >= 4")
    if self.engine == "batch":
      return self._evolve_batch(context, max_generations, patience, optimal_cost)
    if optimal_cost is not None and optimal_cost > 0:
      raise NotImplementedError("the single-run engine has no optimal-cost stop; use engine='batch'")
    if patience is None:
      patience = int(2 * math.sqrt(n))
    self.n, self.patience = n, patience
    P, G = self.P, int(max_generations)
    rng = resolve_rng(context, None)
    self.kernel_launches = 0

    # initial population and fitness (draws the row seeds first, like the reference)
    pop0 = InitializationB200TourNearestNeighbor(k=self.nn_k, return_gpu=True).initialize(list(customers), P, context)
    ops = operands_for(context)
    self.dist, self.stride, self.coords = ops.distance_args(n, self.max_matrix_dimension)
    self.symmetric = self.dist is not None and ops.symmetric
    self.cand = self.cand_dist = self.packed = None
    self.k = 0
    ls = self.ls
    if ls.candidate_k:
      tabs = ops.candidates(int(ls.candidate_k), candidate_list(context, int(ls.candidate_k)), n,
                            self.max_matrix_dimension)
      self.cand, self.cand_dist, self.packed, self.k = tabs.cand, tabs.cand_dist, tabs.packed, tabs.k
    lib = native.load_library()
    rows_max = max(self.elite, P if self.post_init else 0, 1)
    self.ws_bytes = int(lib.tspb_two_opt_workspace_bytes(rows_max, n, self.k, native.MODE_CODES[ls.mode], 128))
    self.ws = torch.empty(max(self.ws_bytes, 1), dtype=torch.uint8, device="cuda")
    self.ls_status = torch.zeros(rows_max, dtype=torch.int32, device="cuda")
    self.d_zero = torch.zeros(1, dtype=torch.int32, device="cuda")

    self.pop = [pop0.contiguous(), torch.empty_like(pop0)]
    self.fit = [torch.empty(P, dtype=torch.float64, device="cuda") for _ in range(2)]
    native.call("tspb_tour_cost", ptr(self.pop[0]), P, n, ptr(self.dist), self.stride, ptr(self.coords), 1,
                ptr(self.fit[0]), stream_handle())
    self.off = torch.empty_like(pop0)
    self.off_fit = torch.empty(P, dtype=torch.float64, device="cuda")
    self.order = torch.empty(P, dtype=torch.int32, device="cuda")
    fit0 = self.fit[0].cpu().numpy()
    i0 = int(np.argmin(fit0))
    initial_best = float(fit0[i0])
    self.best_cost = torch.tensor([initial_best], dtype=torch.float64, device="cuda")
    self.best_tour = self.pop[0][i0].clone()
    self.history = torch.zeros(G + 1, dtype=torch.float64, device="cuda")
    self.history[0] = initial_best
    self.gen = torch.zeros(1, dtype=torch.int32, device="cuda")
    self.stopped = torch.zeros(1, dtype=torch.int32, device="cuda")
    self.stall = torch.zeros(1, dtype=torch.int32, device="cuda")
    self.done = torch.zeros(1, dtype=torch.int32, device="cuda")
    self.ties = torch.zeros(max(G, 1), dtype=torch.int32, device="cuda")
    self.elite_tmp = torch.empty((max(self.elite, 1), n), dtype=torch.int32, device="cuda")
    self.elite_costs = torch.empty(max(self.elite, 1), dtype=torch.float64, device="cuda")

    tape_host, states = self._draw_tape(rng, G, n)
    self.tape = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in tape_host]
    torch.cuda.synchronize()
    t_setup = time.perf_counter()

    # generation 1 starts with the post-init refinement of the whole population
    if self.post_init and G > 0:
      self._two_opt(ptr(self.pop[0]), P)
      native.call("tspb_tour_cost", ptr(self.pop[0]), P, n, ptr(self.dist), self.stride, ptr(self.coords), 1,
                  ptr(self.fit[0]), stream_handle())
      self.kernel_launches += 2

    graphs = self._capture() if (self.use_graph and G > 0) else None
    per_gen = 7 if self.elite else 4
    self.kernel_launches = 2 if (self.post_init and G > 0) else 0
    torch.cuda.synchronize()
    t_loop = time.perf_counter()
    ev_start = torch.cuda.Event(enable_timing=True)
    ev_end = torch.cuda.Event(enable_timing=True)
    ev_start.record()
    g = 0
    chunk = self.chunk
    self.host_elite_generations = 0
    while g < G:
      c = min(chunk, G - g)
      for q in range(c):
        if graphs is not None:
          graphs[(g + q) % 2].replay()
          self.kernel_launches += per_gen
        else:
          self._generation((g + q) % 2)
      state = int(self.stopped.item())  # synchronises the chunk
      if state == 2:  # paused on an elite-edge tie at generation gt
        gt = int(self.gen.item())
        self._host_elites(gt)
        g = gt + 1
        chunk = 1
        if int(self.stopped.item()) == 1:
          break
        continue
      if state == 1:
        break
      g += c
      chunk = min(2 * chunk, self.chunk)
    ev_end.record()
    torch.cuda.synchronize()
    t_end = time.perf_counter()
    loop_ms = ev_start.elapsed_time(ev_end)
    if int(self.ls_status.max().item()) != 0:
      raise RuntimeError("2-opt kernel reported a bad tour inside the fused GA")

    done = int(self.done.item())
    if 0 < done < G:
      rng.bit_generator.state = states[done - 1]
    final_parity = done % 2 if done else 0
    self.final_population = self.pop[final_parity]
    self.final_fitness = self.fit[final_parity]
    history = self.history[: done + 1].cpu().numpy().tolist()
    best_cost = float(self.best_cost.item())
    best_tour = self.best_tour.cpu().numpy().astype(np.int32)
    self.last_timing = {"setup_s": t_setup - t_start, "loop_s": t_end - t_loop, "total_s": t_end - t_start,
                        "loop_ms_device": loop_ms, "generations": done}
    stats = {
      "initial_fitness": initial_best,
      "best_fitness": best_cost,
      "best_is_feasible": True,
      "generations_completed": done,
      # patience can also run out exactly at the last generation (genetic_algorithm.py:906-910)
      "stopped_early": done < G or trailing_stall(history) >= patience,
      "stop_reason": "no_improvements" if done < G or trailing_stall(history) >= patience else "max_generations",
      "convergence_history": history,
      "kernel_launches": self.kernel_launches,
      "host_elite_generations": self.host_elite_generations,
    }
    return best_tour, stats

  def _evolve_batch(self, context: Any, max_generations: int, patience: int | None, optimal_cost: float | None):
    """The run as a one-instance batch (`batch.FusedBatchSolver`): the persistent 2-opt,
    converged-row skipping and device-settled elite ties of the batch engine, same results."""
    from .batch import FusedBatchSolver

    solver = FusedBatchSolver(population_size=self.P, mutation_rate=self.rate, tournament_k=self.kt, nn_k=self.nn_k,
                              local_search=self.ls, elite_count=self.elite, post_init=self.post_init,
                              max_matrix_dimension=self.max_matrix_dimension, use_graph=self.use_graph,
                              chunk=self.chunk, crossover=self.crossover, mutation=self.mutation, init=self.init,
                              local_search_stage=self.stage)
    (best, stats), = solver.evolve([context], max_generations, patience=patience, optimal_cost=optimal_cost)
    self.final_population = solver.final_population[0]
    self.final_fitness = solver.final_fitness[0]
    self.last_timing = solver.last_timing
    self.kernel_launches = solver.kernel_launches
    self.host_elite_generations = stats["host_elite_generations"]
    self.two_opt_totals = solver.two_opt_totals
    stats = dict(stats, kernel_launches=solver.kernel_launches)
    return best, stats

  # -------------------------------------------------------------------------- graph, snapshots
  def _capture(self):
    # Warm every launch path outside capture with the stop flag set (all kernels no-op).
    self.stopped.fill_(1)
    self._generation(0)
    self._generation(1)
    torch.cuda.synchronize()
    self.stopped.fill_(0)
    from .batch import capture_graph

    return [capture_graph(lambda p=parity: self._generation(p)) for parity in (0, 1)]
