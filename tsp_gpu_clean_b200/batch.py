"""Uneven multi-instance batch: many memetic-GA runs advanced by one CUDA graph per generation.

`FusedBatchSolver.evolve(contexts, G)` runs, for every context, exactly the GA that
`FusedMemeticSolver.evolve(context, range(n), G)` runs on it alone - the reference's

    GeneticAlgorithm(population_size=P, mutation_rate=rate,
                     initialization=InitializationCPUTourNearestNeighbor(k=nn_k),
                     selection=SelectionCPUTournament(k=tournament_k),
                     crossover=CrossoverCPUPermPartiallyMapped(), mutation=MutationCPUPermInversion(),
                     evaluation=EvaluationCPUCost(), local_search=LocalSearchCPUTourTwoOpt(...),
                     local_search_stage="none",
                     pipeline=[PostInitLocalSearchStep(...), EliteOnlyLocalSearchStep(..., elite_count=k)])
    .evolve(context, customers, max_generations, patience=...)

(`src/algorithms/metaheuristics/genetic_algorithm.py:789-965`,
`src/algorithms/pipeline_steps.py:85-195`) - with every instance's result (final
population, fitness, best tour, convergence history, generator state) identical to the
single run's.

Layout in HBM: the populations of all instances sit in two flat int32 buffers at
per-instance offsets (P x n rows each), fitness in (I, P) float64 arrays, the tapes of all
runs in (I, G, ...) arrays, one {generation, state, stall, done} control block per run and
one "converged" byte per row (a converged 2-opt local optimum is not refined again: the
refinement would change nothing). Instances with n above `max_matrix_dimension` keep no
matrix: their distances are rebuilt from FP64 coordinates in every kernel.

Scheduling: instances are grouped into size buckets; each bucket gets its own offspring
launch and its own persistent elite 2-opt launch (CTA size picked by `BatchAutotuner`).
One captured graph holds the whole generation for every run (offspring, survival rank
with the elite-edge tie check, survivor gather, elite 2-opt, tracking) and is replayed in
chunks between host checks.

Elite-edge ties (the elite set then follows NumPy's unstable argsort): when every tied
row is converged, each argsort choice refines only rows that do not change, so the run
goes on on the device. Otherwise the run pauses; at the next check the host takes
`np.argsort` of its fitness, and the run finishes that generation in the RESUME phase
(its own 2-opt and tracking launches) at the start of the next replay. Only that first
replay after a host resume carries the phase: its graph is captured when a run first
pauses.
"""

from __future__ import annotations

import ctypes
import math
import time
import weakref
from dataclasses import dataclass, field
from typing import Any, Sequence

import numpy as np

from . import native
from .autotune import BatchAutotuner
from .device import (candidate_list, check_packed, checked_budget, operands_for, ptr, require_gpu, stream_handle, torch,
                     upload_coordinates)
from .fused import LocalSearchConfig, draw_generation_tape
from .problem import resolve_rng
from .strategies.initialization import draw_row_seeds

#: Upper n of the default size buckets (the last bucket takes every larger instance).
DEFAULT_BUCKET_BOUNDS = (128, 256, 512, 1024, 2048, 4096)
TWO_OPT_THREADS = (64, 128, 256, 512, 1024)
#: Runs from which the tape is drawn on the device (one thread per run) instead of the host.
DEVICE_TAPE_MIN_RUNS = 32
OFFSPRING_THREADS = (64, 128, 256)


class LaunchGraph:
  """An executable CUDA graph of this library's launches (`tspb_graph_*`), replayed on the
  current stream. The captured launches keep their buffers' addresses: the buffers must
  outlive the graph."""

  def __init__(self, handle: int):
    self._handle = handle
    self._fin = weakref.finalize(self, LaunchGraph._free, handle)

  @staticmethod
  def _free(handle: int) -> None:
    native.load_library().tspb_graph_destroy(handle)

  def replay(self) -> None:
    native.check("tspb_graph_launch", native.load_library().tspb_graph_launch(self._handle, stream_handle()))

  def release(self) -> None:
    self._fin()


def capture_graph(enqueue) -> LaunchGraph:
  """A CUDA graph of the launches `enqueue()` makes, captured on a side stream by the
  library itself (`tspb_graph_capture_begin/end`). Only the library's own kernels are
  recorded and nothing is allocated during capture, so torch's graph machinery (a private
  allocator pool per graph, set up in `CUDAGraph.capture_begin`, which stalled the host
  for 10-50 ms in some calls) is not involved."""
  lib = native.load_library()
  stream = torch.cuda.Stream()
  stream.wait_stream(torch.cuda.current_stream())
  handle = ctypes.c_void_p()
  with torch.cuda.stream(stream):
    sh = stream_handle()
    native.check("tspb_graph_capture_begin", lib.tspb_graph_capture_begin(sh))
    try:
      enqueue()
    finally:
      rc = lib.tspb_graph_capture_end(sh, ctypes.byref(handle))
  native.check("tspb_graph_capture_end", rc)
  torch.cuda.current_stream().wait_stream(stream)
  torch.cuda.synchronize()
  return LaunchGraph(handle.value)


_DEFAULT_TUNER: BatchAutotuner | None = None


def default_tuner() -> BatchAutotuner:
  """The process-wide tuner (its cache spans every solver of the process)."""
  global _DEFAULT_TUNER
  if _DEFAULT_TUNER is None:
    _DEFAULT_TUNER = BatchAutotuner()
  return _DEFAULT_TUNER


@dataclass
class Bucket:
  """Instances of one size class and the launch shapes chosen for them."""

  lo: int
  hi: int
  coords: bool
  items: list[int] = field(default_factory=list)
  max_n: int = 0
  grouped: bool = False  # every item's k % 4 == 0 and its packed table 16-byte aligned
  can_rebuild: bool = False  # every item has coordinates: the tuner may pick them over the matrix
  incremental: bool = False  # the 2-opt runs with the reverse k-NN index (TSPB_BATCH_INCREMENTAL)
  pair: bool = False  # every row is refined by a two-CTA cluster (TSPB_BATCH_PAIR, best mode)
  two_opt_threads: int = 128
  offspring_threads: int = 128
  d_items: Any = None
  queue: Any = None


# Operators of the generation: PMX (pmx_crossover.py) or OX (order_crossover.py) with
# inversion (inversion_mutation.py) or swap (swap_mutation.py) mutation. All four draw the
# same random numbers, so one tape serves every combination.
CROSSOVER_CODES = {"pmx": native.TSPB_XOVER_PMX, "ox": native.TSPB_XOVER_OX}
MUTATION_CODES = {"inversion": native.TSPB_MUT_INVERSION, "swap": native.TSPB_MUT_SWAP}


# Terminal states of a run that stopped early and the reference's stop_reason for each
# (genetic_algorithm.py:894-910); a run in state DONE ran every generation.
STOP_REASONS = {native.TSPB_BATCH_HIT_OPTIMAL: "hit_optimal", native.TSPB_BATCH_NEAR_OPTIMAL: "within_1pct_optimal",
                native.TSPB_BATCH_STOPPED: "no_improvements"}


def elite_rows(fitness: np.ndarray, elite: int) -> np.ndarray:
  """Rows of `argsort(fitness)[:elite]` for every row of an (m, P) fitness array.

  `EliteOnlyLocalSearchStep` takes `np.argsort(fitness)[:k]` (`pipeline_steps.py:163`);
  NumPy sorts each row of a 2-D array along the last axis with the same routine it uses
  for a 1-D array, so the rows agree with the per-run call, ties included.
  """
  return np.argsort(fitness, axis=1)[:, :elite].astype(np.int32)


class FusedBatchSolver:
  def __init__(self, population_size: int = 64, mutation_rate: float = 0.05, tournament_k: int = 5, nn_k: int = 5,
               local_search: LocalSearchConfig | None = None, elite_count: int = 8, post_init: bool = True,
               max_matrix_dimension: int | None = 4096, use_graph: bool = True,
               tuner: BatchAutotuner | None = None, bucket_bounds: Sequence[int] = DEFAULT_BUCKET_BOUNDS,
               chunk: int = 16, skip_converged: bool = True, concurrent_buckets: bool = True,
               crossover: str = "pmx", mutation: str = "inversion", init: str = "nn",
               local_search_stage: str = "none", incremental: str = "off", pair: str = "auto") -> None:
    if population_size < 2:
      raise ValueError("population_size must be >= 2")
    if init not in ("nn", "random"):
      raise ValueError("init must be 'nn' (nearest neighbour) or 'random' (uniform permutations)")
    if local_search_stage not in ("none", "post_mutation"):
      raise ValueError("local_search_stage must be 'none' or 'post_mutation'")
    self.init, self.stage = init, local_search_stage
    # 2-opt with the reverse k-NN index: best mode recomputes only the rows a move can
    # change, first mode restarts from the move's row; "auto" lets the tuner measure both.
    # Off by default: it lost on every workload measured (a 2000-city GA refining 64
    # elites, a 1002-city GA refining every child), and trying it doubles the tuner's
    # 2-opt probes.
    if incremental not in ("auto", "on", "off"):
      raise ValueError("incremental must be 'auto', 'on' or 'off'")
    self.incremental = incremental
    # best-mode 2-opt of a row by a two-CTA cluster (both CTAs apply every move, each scans
    # half of every pass): pays off when a phase has fewer rows than SMs, e.g. the elites of
    # one run; "auto" lets the tuner measure it beside the one-CTA kernel
    if pair not in ("auto", "on", "off"):
      raise ValueError("pair must be 'auto', 'on' or 'off'")
    self.pair = pair
    if crossover not in CROSSOVER_CODES:
      raise ValueError(f"crossover must be one of {sorted(CROSSOVER_CODES)}")
    if mutation not in MUTATION_CODES:
      raise ValueError(f"mutation must be one of {sorted(MUTATION_CODES)}")
    self.crossover, self.mutation = crossover, mutation
    self.P = int(population_size)
    self.rate = float(mutation_rate)
    self.kt = int(tournament_k)
    self.nn_k = int(nn_k)
    self.ls = local_search if local_search is not None else LocalSearchConfig()
    if self.ls.mode not in ("best", "batch", "first"):
      raise ValueError("the batch 2-opt supports best/batch and first modes")
    if not self.ls.candidate_k:
      raise ValueError("the batch 2-opt runs in candidate mode (candidate_k >= 1)")
    self.elite = min(int(elite_count), self.P) if elite_count else 0
    self.post_init = bool(post_init)
    self.max_matrix_dimension = max_matrix_dimension
    self.use_graph = bool(use_graph)
    self.chunk = max(1, int(chunk))
    self.skip_converged = bool(skip_converged)
    self.concurrent_buckets = bool(concurrent_buckets)
    self._side: list = []
    self.tuner = tuner if tuner is not None else default_tuner()
    self.bucket_bounds = tuple(sorted(int(b) for b in bucket_bounds))
    self.kernel_launches = 0
    self.replays = 0
    self.last_timing: dict[str, float] = {}
    self.buckets: list[Bucket] = []

  # ------------------------------------------------------------------------ setup
  def _make_buckets(self, ns: list[int], coords_flags: list[bool]) -> list[Bucket]:
    buckets: dict[tuple[int, bool], Bucket] = {}
    bounds = self.bucket_bounds
    for i, (n, c) in enumerate(zip(ns, coords_flags)):
      hi_idx = next((j for j, b in enumerate(bounds) if n <= b), len(bounds))
      lo = bounds[hi_idx - 1] + 1 if hi_idx > 0 else 4
      hi = bounds[hi_idx] if hi_idx < len(bounds) else 1 << 16
      b = buckets.setdefault((hi_idx, c), Bucket(lo=lo, hi=hi, coords=c))
      b.items.append(i)
    out = []
    for key in sorted(buckets, key=lambda kc: (-kc[0], kc[1])):
      b = buckets[key]
      b.items.sort(key=lambda i: (-ns[i], i))  # largest first: the persistent queue is LPT
      b.max_n = max(ns[i] for i in b.items)
      out.append(b)
    return out

  def _state(self) -> native.BatchState:
    s = native.BatchState()
    s.num_instances = self.I
    s.P = self.P
    s.kt = self.kt
    s.elite = self.elite
    s.G = self.G
    s.rows_max = self.P
    s.mutation_rate = self.rate
    s.inst = self.d_inst.data_ptr()
    s.pop[0] = self.pop[0].data_ptr()
    s.pop[1] = self.pop[1].data_ptr()
    s.fit[0] = self.fit[0].data_ptr()
    s.fit[1] = self.fit[1].data_ptr()
    s.off = self.off.data_ptr()
    s.off_fit = self.off_fit.data_ptr()
    s.order = self.order.data_ptr()
    t = self.tape
    s.tape_tourn, s.tape_cut_a, s.tape_cut_b = t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr()
    s.tape_u, s.tape_inv_a, s.tape_inv_b = t[3].data_ptr(), t[4].data_ptr(), t[5].data_ptr()
    s.ctl = self.ctl.data_ptr()
    s.best_cost = self.best_cost.data_ptr()
    s.best_tour = self.best_tour.data_ptr()
    s.history = self.history.data_ptr()
    s.ties = self.ties.data_ptr()
    s.host_elites = self.host_elites.data_ptr()
    s.ls_status = self.ls_status.data_ptr()
    s.ls_stats = self.ls_stats.data_ptr()
    if self.skip_converged:
      s.clean[0] = self.clean[0].data_ptr()
      s.clean[1] = self.clean[1].data_ptr()
      s.off_clean = self.off_clean.data_ptr()
    s.crossover = CROSSOVER_CODES[self.crossover]
    s.mutation = MUTATION_CODES[self.mutation]
    return s

  # ------------------------------------------------------------------------ launches
  @property
  def _mode(self) -> int:
    return native.MODE_CODES[self.ls.mode]

  @staticmethod
  def _flags(bucket: Bucket) -> int:
    return ((native.TSPB_BATCH_COORDS if bucket.coords else 0) | (native.TSPB_BATCH_GROUPED if bucket.grouped else 0)
            | (native.TSPB_BATCH_INCREMENTAL if bucket.incremental else 0)
            | (native.TSPB_BATCH_PAIR if bucket.pair else 0))

  def _two_opt(self, st_ref, bucket: Bucket, phase: int, threads: int | None = None) -> None:
    rc = native.load_library().tspb_batch_two_opt(
      st_ref, ptr(bucket.d_items), len(bucket.items), bucket.max_n, self._flags(bucket), phase, self._mode,
      int(self.ls.max_iterations), int(threads or bucket.two_opt_threads), 0, ptr(bucket.queue), stream_handle())
    native.check("tspb_batch_two_opt", rc)
    self.kernel_launches += 1

  def _offspring(self, st_ref, bucket: Bucket, threads: int | None = None) -> None:
    rc = native.load_library().tspb_batch_offspring(st_ref, ptr(bucket.d_items), len(bucket.items), bucket.max_n,
                                                    int(threads or bucket.offspring_threads), stream_handle())
    native.check("tspb_batch_offspring", rc)
    self.kernel_launches += 1

  def _per_bucket(self, fn) -> None:
    """fn(bucket) for every bucket; with concurrent buckets each runs on its own side
    stream forked from and joined back to the current stream (parallel graph branches)."""
    if not self.concurrent_buckets or len(self.buckets) < 2:
      for b in self.buckets:
        fn(b)
      return
    main = torch.cuda.current_stream()
    while len(self._side) < len(self.buckets):
      self._side.append(torch.cuda.Stream())
    for s, b in zip(self._side, self.buckets):
      s.wait_stream(main)
      with torch.cuda.stream(s):
        fn(b)
    for s in self._side[: len(self.buckets)]:
      main.wait_stream(s)

  @property
  def _post_mutation(self) -> bool:
    return self.stage == "post_mutation"

  @property
  def _ls_rows(self) -> int:
    """Rows per instance of the generation's main 2-opt phase (the tuner's work shape)."""
    return self.P if self._post_mutation else self.elite

  def _generation(self, resume: bool = True) -> None:
    """Enqueue one replay: finish RESUME runs (only the host sets that state, so `resume`
    is needed only right after a host check that resumed runs), then one generation of
    every RUN run."""
    lib = native.load_library()
    st = ctypes.byref(self.state)
    sh = stream_handle()
    R, U, O = native.TSPB_BATCH_PHASE_RESUME, native.TSPB_BATCH_PHASE_RUN, native.TSPB_BATCH_PHASE_OFFSPRING
    # the 2-opt kernel stores each refined row's fitness itself (no separate cost pass)
    if self.elite and resume:
      self._per_bucket(lambda b: self._two_opt(st, b, R))
      native.check("tspb_batch_track", lib.tspb_batch_track(st, R, sh))
      self.kernel_launches += 1

    def children(b: Bucket) -> None:
      self._offspring(st, b)
      if self._post_mutation:  # LocalSearchStep(target="offspring") before evaluation
        self._two_opt(st, b, O)

    self._per_bucket(children)
    native.check("tspb_batch_survival", lib.tspb_batch_survival(st, sh))
    self.kernel_launches += self._survival_launches()
    if self.elite:
      self._per_bucket(lambda b: self._two_opt(st, b, U))
    native.check("tspb_batch_track", lib.tspb_batch_track(st, U, sh))
    self.kernel_launches += 1

  @staticmethod
  def _survival_launches() -> int:
    """Kernels of tspb_batch_survival: the rank (with the elite-edge tie check), then the
    survivor gather."""
    return 2

  def _launches_per_replay(self, resume: bool = False) -> int:
    nb = len(self.buckets)
    per = nb + self._survival_launches() + 1  # offspring per bucket, survival, track
    if self.elite:
      per += nb  # the elite 2-opt per bucket
      if resume:
        per += nb + 1  # the RESUME phase's 2-opt per bucket and its track
    if self._post_mutation:
      per += nb  # offspring 2-opt per bucket
    return per

  # ------------------------------------------------------------------------ autotuning
  def _tune(self) -> None:
    """CTA sizes per bucket from the tuner (measured once per shape, then cached)."""
    lib = native.load_library()
    name = torch.cuda.get_device_name()
    for b in self.buckets:
      if self._ls_rows:
        units = len(b.items) * self._ls_rows
        pairable = b.grouped and self.ls.mode in ("best", "batch")
        key = self.tuner.key(name, "two_opt", mode=self.ls.mode, k=self.k, iters=int(self.ls.max_iterations),
                             lo=b.lo, hi=b.hi, coords=b.coords, rebuild=b.can_rebuild, units=units,
                             inc=self.incremental if b.grouped else "off", pair=self.pair if pairable else "off")
        # candidate = 8 * threads + 4 * pair + 2 * incremental + source (1: distances rebuilt
        # from coordinates); a pair runs without the incremental row keys
        incs = {"auto": (0, 1), "on": (1,), "off": (0,)}[self.incremental] if b.grouped else (0,)
        pairs = {"auto": (0, 1), "on": (1,), "off": (0,)}[self.pair] if pairable else (0,)
        sources = (0, 1) if (b.can_rebuild and not b.coords) else ((1,) if b.coords else (0,))

        def fits(t, inc, pr):
          flags = ((native.TSPB_BATCH_GROUPED if b.grouped else 0) | (native.TSPB_BATCH_INCREMENTAL if inc else 0)
                   | (native.TSPB_BATCH_PAIR if pr else 0))
          return lib.tspb_batch_two_opt_occupancy(b.max_n, self._mode, t, flags) > 0

        cands = [8 * t + 4 * pr + 2 * inc + src for t in TWO_OPT_THREADS for pr in pairs for inc in incs
                 for src in sources if not (pr and inc) and fits(t, inc, pr)]
        if not cands:
          raise ValueError(f"instances of n={b.max_n} do not fit the batch 2-opt's shared memory")
        choice = self.tuner.choose(key, cands,
                                   lambda c, b=b: self._probe_two_opt(b, c // 8, bool(c & 1), bool(c & 2),
                                                                      bool(c & 4)))
        b.two_opt_threads = choice // 8
        b.pair = bool(choice & 4)
        b.incremental = bool(choice & 2)
        if choice & 1 and not b.coords:
          self._rebuild_from_coordinates(b)
      if self.G:
        key = self.tuner.key(name, "offspring", lo=b.lo, hi=b.hi, coords=b.coords, units=len(b.items) * self.P)
        b.offspring_threads = self.tuner.choose(key, list(OFFSPRING_THREADS),
                                                lambda t, b=b: self._probe_offspring(b, t))

  @staticmethod
  def _timed(fn, reps: int = 3) -> float:
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    fn()  # warm-up (also sets the kernel attributes)
    torch.cuda.synchronize()
    start.record()
    for _ in range(reps):
      fn()
    end.record()
    end.synchronize()
    return start.elapsed_time(end) / reps

  def _rebuild_from_coordinates(self, b: Bucket) -> None:
    """The bucket's instances drop their matrix: every kernel rebuilds their distances from
    the FP64 coordinates (the same values, bit for bit)."""
    for i in b.items:
      self.h_inst[i].dist = None
      self.h_inst[i].dist_stride = 0
    self.d_inst.copy_(torch.frombuffer(bytearray(self.h_inst), dtype=torch.uint8))
    b.coords = True

  def _probe_two_opt(self, b: Bucket, threads: int, rebuild: bool = False, incremental: bool = False,
                     pair: bool = False) -> float:
    """The generation's 2-opt work shape for one bucket on scratch copies of the initial
    tours: the first `elite` rows of every instance (every row with the post_mutation
    stage), refined for up to max_iterations passes, with the bucket's matrices or
    (rebuild) distances rebuilt from coordinates, and with or without the reverse k-NN
    index (incremental)."""
    e = max(self._ls_rows, 2)  # the probe batch needs P >= 2
    ns = self.ns
    offs = np.zeros(self.I, dtype=np.int64)
    offs[1:] = np.cumsum([e * n for n in ns])[:-1]
    scratch = torch.empty(max(int(e * sum(ns)), 1), dtype=torch.int32, device="cuda")
    inst = (native.BatchInstance * self.I)()
    ctypes.memmove(inst, self.h_inst, ctypes.sizeof(inst))
    for i in range(self.I):
      inst[i].pop_offset = int(offs[i])
      if rebuild:
        inst[i].dist = None
        inst[i].dist_stride = 0
    d_inst = torch.frombuffer(bytearray(inst), dtype=torch.uint8).cuda()
    flags = ((native.TSPB_BATCH_COORDS if (b.coords or rebuild) else 0)
             | (native.TSPB_BATCH_GROUPED if b.grouped else 0) | (native.TSPB_BATCH_INCREMENTAL if incremental else 0)
             | (native.TSPB_BATCH_PAIR if pair else 0))
    status = torch.zeros((self.I, e), dtype=torch.int32, device="cuda")
    st = self._state()
    st.P = e
    st.rows_max = e
    st.inst = d_inst.data_ptr()
    st.ls_status = status.data_ptr()
    st.ls_stats = None
    st.pop[0] = st.pop[1] = scratch.data_ptr()
    st.clean[0] = st.clean[1] = None  # measure the full refinement work
    st.off_clean = None
    st_ref = ctypes.byref(st)
    lib = native.load_library()
    src = [self.pop[0][self.pop_offsets[i]: self.pop_offsets[i] + e * ns[i]] for i in b.items]
    dst = [scratch[int(offs[i]): int(offs[i]) + e * ns[i]] for i in b.items]

    def fill():
      for d, s_ in zip(dst, src):
        d.copy_(s_)

    def run():
      fill()
      rc = lib.tspb_batch_two_opt(st_ref, ptr(b.d_items), len(b.items), b.max_n, flags,
                                  native.TSPB_BATCH_PHASE_POSTINIT, self._mode, int(self.ls.max_iterations), threads, 0,
                                  ptr(b.queue), stream_handle())
      native.check("tspb_batch_two_opt", rc)

    fill_ms = self._timed(fill)
    ms = self._timed(run)
    if int(status.max().item()) != 0:
      raise RuntimeError("2-opt probe reported a bad tour")
    return max(ms - fill_ms, 0.0)

  def _probe_offspring(self, b: Bucket, threads: int) -> float:
    # offspring writes only the scratch rows `off`, `off_fit`, `off_clean`: safe on the live state
    st_ref = ctypes.byref(self.state)
    return self._timed(lambda: self._offspring(st_ref, b, threads))

  def _host_tapes(self, rngs: list, ns: list[int]) -> bool:
    """Whether this batch draws its tapes on the host (a few runs; any bit generator)."""
    gens_pcg = all(native.Pcg64.from_state(r.bit_generator.state) is not None for r in rngs)
    return self.G > 0 and not (gens_pcg and self.I >= DEVICE_TAPE_MIN_RUNS)

  def _start_host_tapes(self, rngs: list, ns: list[int]):
    """Start the host draws of every run's tape in a thread; None when the device draws."""
    if not self._host_tapes(rngs, ns):
      return None
    import threading

    G, P, kt = self.G, self.P, self.kt
    job = {"tapes": [None] * len(rngs), "error": None}

    def work():
      try:
        for i, (r, n) in enumerate(zip(rngs, ns)):
          job["tapes"][i] = draw_generation_tape(r, G, P, kt, n)
      except BaseException as exc:  # re-raised by the caller
        job["error"] = exc

    job["thread"] = threading.Thread(target=work, daemon=True)
    job["thread"].start()
    return job

  def _draw_tapes(self, rngs: list, ns: list[int], job=None) -> None:
    """Every run's random tape, drawn on the device by `tspb_tape_draw` (one thread per run,
    NumPy's PCG64 stream restated) when every generator is PCG64, else by NumPy on the host.
    Each generator ends in the state it has after the reference draws G generations."""
    I, G, P, kt = self.I, self.G, self.P, self.kt
    dev = "cuda"
    self.tape = [torch.empty((I, G, P, kt), dtype=torch.int32, device=dev),
                 torch.empty((I, G, P // 2), dtype=torch.int32, device=dev),
                 torch.empty((I, G, P // 2), dtype=torch.int32, device=dev),
                 torch.empty((I, G, P), dtype=torch.float64, device=dev),
                 torch.empty((I, G, P), dtype=torch.int32, device=dev),
                 torch.empty((I, G, P), dtype=torch.int32, device=dev)]
    self._dev_states = None
    self.states = []
    if G == 0:
      return
    if job is not None:  # the host draws already running: no generator is read before they end
      job["thread"].join()
      if job["error"] is not None:
        raise job["error"]
      self._store_host_tapes(job["tapes"])
      return
    gens = [native.Pcg64.from_state(r.bit_generator.state) for r in rngs]
    # one device thread per run pays only with many runs; a few runs draw faster on the host
    if all(g is not None for g in gens) and I >= DEVICE_TAPE_MIN_RUNS:
      h_gens = (native.Pcg64 * I)(*gens)
      d_gens = torch.frombuffer(bytearray(h_gens), dtype=torch.uint8).cuda()
      d_ns = torch.tensor(ns, dtype=torch.int32, device=dev)
      self._dev_states = torch.empty(I * G * ctypes.sizeof(native.Pcg64), dtype=torch.uint8, device=dev)
      native.call("tspb_tape_draw", ptr(d_gens), ptr(d_ns), I, G, P, kt, *[ptr(t) for t in self.tape],
                  ptr(self._dev_states), stream_handle())
      self.kernel_launches += 1
      final = (native.Pcg64 * I).from_buffer_copy(d_gens.cpu().numpy().tobytes())
      for r, g in zip(rngs, final):
        r.bit_generator.state = g.to_state()
      return
    self._store_host_tapes([draw_generation_tape(r, G, P, kt, n) for r, n in zip(rngs, ns)])

  def _store_host_tapes(self, drawn) -> None:
    """Copy the host-drawn tapes (one (arrays, states) pair per run) to the device tape."""
    host = [np.empty(tuple(t.shape), dtype=np.float64 if t.dtype == torch.float64 else np.int32) for t in self.tape]
    for i, (tape, states) in enumerate(drawn):
      for h, a in zip(host, tape):
        h[i] = a
      self.states.append(states)
    for t, h in zip(self.tape, host):
      t.copy_(torch.from_numpy(h))

  def _state_after(self, i: int, g: int) -> dict:
    """Generator state of run i after generation g (0-based)."""
    if self._dev_states is None:
      return self.states[i][g]
    sz = ctypes.sizeof(native.Pcg64)
    off = (i * self.G + g) * sz
    return native.Pcg64.from_buffer_copy(self._dev_states[off: off + sz].cpu().numpy().tobytes()).to_state()

  def _nn_init(self, h_jobs, seeds_all: np.ndarray, tables: list, ns: list[int]) -> None:
    """GRASP nearest-neighbour populations of every instance in one launch
    (`tspb_nn_init_jobs_smem`, or `tspb_nn_init_jobs` for rows too large for shared memory;
    each row as `InitializationCPUTourNearestNeighbor` builds it)."""
    P = self.P
    ks = [int(t.shape[1]) if t.ndim == 2 else 0 for t in tables]
    cand_off = np.zeros(self.I + 1, dtype=np.int64)
    cand_off[1:] = np.cumsum([n * k for n, k in zip(ns, ks)])
    flat = np.zeros(max(int(cand_off[-1]), 1), dtype=np.int32)
    for i, t in enumerate(tables):
      flat[cand_off[i]: cand_off[i + 1]] = t.reshape(-1)
    d_cand = torch.from_numpy(flat).cuda()
    d_seeds = torch.from_numpy(seeds_all.view(np.int64)).cuda()
    for i, (n, k) in enumerate(zip(ns, ks)):
      job = h_jobs[i]
      job.n, job.k, job.rows = n, k, P
      job.cand = d_cand.data_ptr() + int(cand_off[i]) * 4
      job.seeds = d_seeds.data_ptr() + i * P * 8
      job.out = self.pop[0].data_ptr() + self.pop_offsets[i] * 4
    d_jobs = torch.frombuffer(bytearray(h_jobs), dtype=torch.uint8).cuda()
    # every row's working arrays in shared memory when they fit, else a global workspace
    rc = native.load_library().tspb_nn_init_jobs_smem(ptr(d_jobs), self.I, P, max(ns), max(ks), stream_handle())
    if rc == native.TSPB_ERR_UNSUPPORTED:
      ws_off = np.zeros(self.I + 1, dtype=np.int64)
      ws_off[1:] = np.cumsum([P * (2 * n + k) for n, k in zip(ns, ks)])
      d_ws = torch.empty(max(int(ws_off[-1]), 1), dtype=torch.int32, device="cuda")
      d_ws_off = torch.from_numpy(ws_off[:-1].copy()).cuda()
      native.call("tspb_nn_init_jobs", ptr(d_jobs), self.I, P, ptr(d_ws), ptr(d_ws_off), stream_handle())
    else:
      native.check("tspb_nn_init_jobs_smem", rc)
    torch.cuda.current_stream().synchronize()  # the host buffers above are released on return
    self.kernel_launches += 1

  def _random_init(self, h_jobs, seeds_all: np.ndarray, ns: list[int]) -> None:
    """Uniform random-permutation populations of every instance in one launch
    (`tspb_random_init_jobs`, each row as `InitializationCPUPermRandom` builds it)."""
    P = self.P
    d_seeds = torch.from_numpy(seeds_all.view(np.int64)).cuda()
    for i, n in enumerate(ns):
      job = h_jobs[i]
      job.n, job.k, job.rows = n, 0, P
      job.cand = None
      job.seeds = d_seeds.data_ptr() + i * P * 8
      job.out = self.pop[0].data_ptr() + self.pop_offsets[i] * 4
    d_jobs = torch.frombuffer(bytearray(h_jobs), dtype=torch.uint8).cuda()
    native.call("tspb_random_init_jobs", ptr(d_jobs), self.I, P, max(ns), stream_handle())
    torch.cuda.current_stream().synchronize()  # the host buffers above are released on return
    self.kernel_launches += 1

  # ------------------------------------------------------------------------ evolve
  def evolve(self, contexts: Sequence[Any], max_generations: int, patience: Any = None, optimal_cost: Any = None):
    """Run every context's GA; returns a list of (best_tour, stats) in context order.

    `patience`: one value for every run, or one per context; None means the reference's
    default int(2 * sqrt(n)) (`genetic_algorithm.py:815-816`). `optimal_cost`: None, one
    value or one per context; a run whose best reaches it, or comes within 1 % of it,
    stops early (`genetic_algorithm.py:894-905`)."""
    require_gpu()
    t_start = time.perf_counter()
    P, G, k = self.P, int(max_generations), int(self.ls.candidate_k)
    self.G, self.I, self.k = G, len(contexts), k
    self.kernel_launches = 0
    self.replays = 0
    if self.I == 0:
      return []
    ns = [int(c.dimension) for c in contexts]
    if min(ns) < 4:
      raise ValueError("every instance needs dimension >= 4")
    self.ns = ns
    rngs = [resolve_rng(c, None) for c in contexts]
    prefix = np.zeros(self.I + 1, dtype=np.int64)
    prefix[1:] = np.cumsum(ns)
    self.pop_offsets = [int(P * prefix[i]) for i in range(self.I)]
    total = int(prefix[-1])

    # device buffers
    dev = "cuda"
    self.pop = [torch.empty(P * total, dtype=torch.int32, device=dev) for _ in range(2)]
    self.off = torch.empty(P * total, dtype=torch.int32, device=dev)
    self.fit = [torch.zeros((self.I, P), dtype=torch.float64, device=dev) for _ in range(2)]
    self.off_fit = torch.zeros((self.I, P), dtype=torch.float64, device=dev)
    self.order = torch.zeros((self.I, P), dtype=torch.int32, device=dev)
    self.ctl = torch.zeros((self.I, 4), dtype=torch.int32, device=dev)
    self.best_cost = torch.zeros(self.I, dtype=torch.float64, device=dev)
    self.best_tour = torch.zeros(total, dtype=torch.int32, device=dev)
    self.history = torch.zeros((self.I, G + 1), dtype=torch.float64, device=dev)
    self.ties = torch.zeros((self.I, max(G, 1)), dtype=torch.int32, device=dev)
    self.host_elites = torch.zeros((self.I, max(self.elite, 1)), dtype=torch.int32, device=dev)
    self.ls_status = torch.zeros((self.I, P), dtype=torch.int32, device=dev)
    self.ls_stats = torch.zeros((self.I, P, 4), dtype=torch.int64, device=dev)
    self.clean = [torch.zeros((self.I, P), dtype=torch.uint8, device=dev) for _ in range(2)]
    self.off_clean = torch.zeros((self.I, P), dtype=torch.uint8, device=dev)

    # per instance: NN row seeds (drawn first, like the reference), operands, tape
    h_inst = (native.BatchInstance * self.I)()
    h_jobs = (native.NNJob * self.I)()
    seeds_all = np.empty((self.I, P), dtype=np.uint64)
    nn_tables = []

    self._keep = []
    coords_flags = []
    rebuildable = []
    t_ops = t_tape = 0.0
    all_tabs = []
    for i, rng in enumerate(rngs):
      seeds_all[i] = draw_row_seeds(rng, P)  # nearest_neighbor_init.py:118-121, random_init.py:42
    # every generator's next draws are its generations' tape: a few runs draw it on the
    # host, in a thread (the C++ draw releases the GIL) while the operands are built here
    tape_job = self._start_host_tapes(rngs, ns)
    t0 = time.perf_counter()
    # all coordinates in one upload, and one free-memory check for all the matrices to build
    all_ops = [operands_for(ctx) for ctx in contexts]
    upload_coordinates([o for o in all_ops if o._euc2d_on_device()])
    need, seen = 0, set()
    for o, n in zip(all_ops, ns):
      key = id(o._shared) if o._shared is not None else id(o)  # contexts of one Problem share a matrix
      if key not in seen and not o.use_coords(n, self.max_matrix_dimension) and not o.has_dist():
        need += n * n * 4
      seen.add(key)
    budget = checked_budget(need, f"distance matrices of {self.I} instances")
    budget.__enter__()
    t_ops += time.perf_counter() - t0
    try:
      for i, (ctx, n, rng) in enumerate(zip(contexts, ns, rngs)):
        if self.init == "nn":
          nn_tables.append(np.ascontiguousarray(candidate_list(ctx, self.nn_k), dtype=np.int32))
        t0 = time.perf_counter()
        ops = operands_for(ctx)
        dist, stride, coords = ops.distance_args(n, self.max_matrix_dimension)
        tabs = ops.candidates(k, candidate_list(ctx, k), n, self.max_matrix_dimension)
        if tabs.packed_words is None:
          raise ValueError(f"instance {i}: k-NN table does not pack into 16-bit ids and distances")
        all_tabs.append(tabs)
        t_ops += time.perf_counter() - t0
        self._keep.append((dist, coords, tabs))
        inst = h_inst[i]
        inst.n = n
        inst.k = tabs.k
        inst.pop_offset = self.pop_offsets[i]
        inst.node_offset = int(prefix[i])
        inst.dist = dist.data_ptr() if dist is not None else None
        inst.dist_stride = int(stride)
        has_xy = ops._euc2d_on_device() or coords is not None
        xy = coords if coords is not None else (ops.coords() if has_xy else None)
        inst.coords = xy.data_ptr() if xy is not None else None
        rebuildable.append(xy is not None)
        self._keep.append(xy)
        inst.cand_packed = tabs.packed_words.data_ptr()
        inst.rev_off = tabs.rev_off.data_ptr()
        inst.rev_idx = tabs.rev_idx.data_ptr()
        pat = patience[i] if isinstance(patience, (list, tuple, np.ndarray)) else patience
        inst.patience = int(pat) if pat is not None else int(2 * math.sqrt(n))
        opt = optimal_cost[i] if isinstance(optimal_cost, (list, tuple, np.ndarray)) else optimal_cost
        inst.optimal = float(opt) if opt is not None and opt > 0 else 0.0
        coords_flags.append(dist is None)
    finally:
      budget.__exit__(None, None, None)
    t0 = time.perf_counter()
    check_packed(all_tabs)  # every instance's pack-overflow flag in one sync
    bad = [i for i, t in enumerate(all_tabs) if t.packed is None]
    if bad:
      raise ValueError(f"instance {bad[0]}: k-NN table does not pack into 16-bit ids and distances")
    t_ops += time.perf_counter() - t0
    t0 = time.perf_counter()
    if self.init == "nn":
      self._nn_init(h_jobs, seeds_all, nn_tables, ns)
    else:
      self._random_init(h_jobs, seeds_all, ns)
    t1 = time.perf_counter()
    self._draw_tapes(rngs, ns, tape_job)  # after the row seeds, like the reference
    t_nn, t_tape = t1 - t0, time.perf_counter() - t1
    self.h_inst = h_inst
    self.d_inst = torch.frombuffer(bytearray(h_inst), dtype=torch.uint8).cuda()
    self.state = self._state()
    st = ctypes.byref(self.state)
    lib = native.load_library()
    sh = stream_handle()

    self.buckets = self._make_buckets(ns, coords_flags)
    for b in self.buckets:
      b.grouped = all(h_inst[i].k % 4 == 0 and h_inst[i].cand_packed % 16 == 0 for i in b.items)
      b.can_rebuild = all(rebuildable[i] for i in b.items)
      b.d_items = torch.tensor(b.items, dtype=torch.int32, device=dev)
      b.queue = torch.zeros(1, dtype=torch.int32, device=dev)

    # initial fitness and best (before the post-init refinement, like the reference)
    native.check("tspb_batch_init", lib.tspb_batch_init(st, 0, 1, sh))
    torch.cuda.synchronize()
    t_setup = time.perf_counter()
    self._tune()
    torch.cuda.synchronize()
    t_tuned = time.perf_counter()
    self.kernel_launches = 2  # tspb_batch_init: the rows' fitness, then the initial best
    initial_best = self.best_cost.cpu().numpy().copy()
    if self.post_init and G > 0:
      for b in self.buckets:
        self._two_opt(st, b, native.TSPB_BATCH_PHASE_POSTINIT)
      native.check("tspb_batch_init", lib.tspb_batch_init(st, 0, 0, sh))
      self.kernel_launches += 1
    stats_before = self.ls_stats.sum(dim=(0, 1)).cpu().numpy()
    t_postinit = time.perf_counter()

    # graphs[resume]: the replay with the RESUME phase is captured when a run first pauses
    graphs = {False: self._capture(False)} if (self.use_graph and G > 0) else None
    torch.cuda.synchronize()
    t_loop = time.perf_counter()
    t_prep = t_loop - t_tuned  # post-init refinement, graph capture
    ev_start = torch.cuda.Event(enable_timing=True)
    ev_end = torch.cuda.Event(enable_timing=True)
    ev_start.record()
    ctl_host = torch.empty((self.I, 4), dtype=torch.int32, pin_memory=True)
    # each round's snapshot also carries both fitness buffers, so a paused run's fitness
    # needs no further read; the host's answers go back through pinned buffers without a
    # sync (the next round's snapshot is ordered after them)
    fit_host = torch.empty((2, self.I, P), dtype=torch.float64, pin_memory=True)
    ctl_up = torch.empty((self.I, 4), dtype=torch.int32, pin_memory=True)
    he_up = torch.zeros((self.I, max(self.elite, 1)), dtype=torch.int32, pin_memory=True)
    he_host = he_up.numpy()
    ready = torch.cuda.Event()
    host_elite_gens = np.zeros(self.I, dtype=np.int64)
    live = (native.TSPB_BATCH_RUN, native.TSPB_BATCH_PAUSED, native.TSPB_BATCH_RESUME)
    # Every round (replays, then one host check) advances each live run by a generation
    # or leaves it paused for the host, who resumes it before the next round.
    rounds, max_rounds = 0, 2 * G + 2
    chunk, remaining = min(self.chunk, max(G, 1)), G
    c = None
    need_resume = False  # runs the host resumed wait for the next replay's RESUME phase
    while G > 0 and rounds < max_rounds:
      for q in range(max(1, min(chunk, remaining))):
        resume = need_resume and q == 0 and self.elite > 0
        if graphs is not None:
          if resume not in graphs:
            graphs[resume] = self._capture(resume, warm=False)
          graphs[resume].replay()
          self.kernel_launches += self._launches_per_replay(resume)
        else:
          self._generation(resume)
        self.replays += 1
      rounds += 1
      ctl_host.copy_(self.ctl, non_blocking=True)
      fit_host[0].copy_(self.fit[0], non_blocking=True)
      fit_host[1].copy_(self.fit[1], non_blocking=True)
      ready.record()
      ready.synchronize()
      c = ctl_host.numpy()
      paused = np.nonzero(c[:, 1] == native.TSPB_BATCH_PAUSED)[0]
      if paused.size:
        parity = (c[paused, 0] + 1) & 1
        fits = fit_host.numpy()[parity, paused]
        he_host[paused] = elite_rows(fits, self.elite)  # pipeline_steps.py:163
        self.host_elites.copy_(he_up, non_blocking=True)
        c = c.copy()
        c[paused, 1] = native.TSPB_BATCH_RESUME
        ctl_up.numpy()[...] = c
        self.ctl.copy_(ctl_up, non_blocking=True)
        host_elite_gens[paused] += 1
        chunk = max(1, chunk // 2)
      else:
        chunk = min(2 * chunk, self.chunk)
      need_resume = bool(paused.size)
      alive = np.isin(c[:, 1], live)
      if not alive.any():
        break
      remaining = G - int(c[alive, 0].min())
    ev_end.record()
    torch.cuda.synchronize()
    t_end = time.perf_counter()
    loop_ms = ev_start.elapsed_time(ev_end)
    if G > 0 and c is not None and np.isin(c[:, 1], live).any():
      raise RuntimeError("batch GA did not finish within its round bound")
    if int(self.ls_status.max().item()) != 0:
      raise RuntimeError(f"2-opt kernel reported status {int(self.ls_status.max().item())} inside the batch GA")

    # results
    ctl = self.ctl.cpu().numpy()
    best_cost = self.best_cost.cpu().numpy()
    best_tour = self.best_tour.cpu().numpy()
    history = self.history.cpu().numpy()
    ties = self.ties.cpu().numpy()
    stats_all = self.ls_stats.sum(dim=(0, 1)).cpu().numpy() - stats_before
    results = []
    self.final_population, self.final_fitness = [], []
    for i, rng in enumerate(rngs):
      done = int(ctl[i, 3]) if G > 0 else 0
      if 0 < done < G:
        rng.bit_generator.state = self._state_after(i, done - 1)
      parity = done % 2
      n = ns[i]
      self.final_population.append(self.pop[parity][self.pop_offsets[i]: self.pop_offsets[i] + P * n].view(P, n))
      self.final_fitness.append(self.fit[parity][i])
      results.append((best_tour[prefix[i]: prefix[i + 1]].astype(np.int32).copy(), {
        "initial_fitness": float(initial_best[i]),
        "best_fitness": float(best_cost[i]),
        "best_is_feasible": True,
        "generations_completed": done,
        "stopped_early": int(ctl[i, 1]) in STOP_REASONS,
        "stop_reason": STOP_REASONS.get(int(ctl[i, 1]), "max_generations"),
        "convergence_history": history[i, : done + 1].tolist(),
        "host_elite_generations": int(host_elite_gens[i]),
        "elite_edge_ties": int(ties[i, :done].sum()) if G > 0 else 0,
      }))
    # 2-opt work inside the generation loop (the post-init refinement excluded)
    self.two_opt_totals = {"passes": int(stats_all[0]), "pairs": int(stats_all[1]), "moves": int(stats_all[2]),
                           "evaluated": int(stats_all[3])}
    self.last_timing = {"setup_s": t_setup - t_start, "setup_operands_s": t_ops, "setup_tape_s": t_tape,
                        "setup_nn_init_s": t_nn, "tune_s": t_tuned - t_setup, "postinit_capture_s": t_prep,
                        "postinit_s": t_postinit - t_tuned, "capture_s": t_loop - t_postinit,
                        "results_s": time.perf_counter() - t_end, "loop_s": t_end - t_loop,
                        "total_s": t_end - t_start, "loop_ms_device": loop_ms,
                        "generations": int(ctl[:, 3].sum()) if G > 0 else 0, "replays": self.replays,
                        "rounds": rounds}
    return results

  # ------------------------------------------------------------------------ graph
  def _capture(self, resume: bool, warm: bool = True):
    """The graph of one replay, with or without the RESUME phase. `warm` first runs every
    launch path (the RESUME phase included) outside capture with every run parked, so all
    kernels no-op."""
    launches = self.kernel_launches
    if warm:
      saved = self.ctl.clone()
      self.ctl[:, 1] = native.TSPB_BATCH_DONE
      self._generation(True)
      torch.cuda.synchronize()
      self.ctl.copy_(saved)
    g = capture_graph(lambda: self._generation(resume))
    self.kernel_launches = launches
    return g
