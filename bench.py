"""Benchmark: batched 2-opt to a local optimum on B200 (2-opt deltas/s).

Workload (one step): 1024 random-permutation tours of a 1000-city, 20-cluster
Gaussian-mixture EUC_2D instance (sigma 30, [0, 1000]^2, int32 matrix), refined to a
local optimum with candidate_k=20, once in best mode and once in first mode. The
metric counts the (i, j) pairs the reference's CPU scan evaluates on the same tours
(oracle-equivalent 2-opt deltas), summed over every pass of every tour.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

- `value`: deltas/s with tours already resident in HBM, timed with CUDA events on the
  launching stream, L2 flushed (256 MiB write) between timed steps. The timed launches
  pass no stats buffer, so first mode runs without its pair-count bookkeeping; the pair
  count comes from one untimed launch of the same tours with stats (the kernel counts the
  pairs itself, and tests pin the count to the oracle), and every timed launch must
  return exactly that launch's tours.
- `e2e`: the same metric through `LocalSearchB200TourTwoOpt.improve_batch` on host
  NumPy tours (pinned H2D, kernel, D2H per call), timed with CUDA events.
- `parity`: a sample of the timed tours, spread over the batch, refined by the NumPy
  oracle in both modes on the host cores; tours, passes, pairs and moves must equal the
  GPU's, or the run exits non-zero after printing its line.
- `roofline`: the dominant launch against the two ceilings of an L2-resident scan, the
  L2 gather rate and the INT32 issue rate, both measured in the same run
  (`tsp_gpu_clean_b200.roofline`), with per-gain counter figures from one ncu capture.
- `detail.ga1000`: the memetic GA at n = 1000 (population 512, 100 generations, 64
  elites, best-mode 2-opt k = 20 x 10): device generations/s, end to end, and the NumPy
  GA on one host core.
- `--impl reference`: the reference CPU path (the NumPy oracle restatement of
  `LocalSearchCPUTourTwoOpt`) on the host cores, on a bounded sample of tours.
- N > 1 (torchrun): every rank refines its own 1024 tours (weak scaling, no
  collective on the data path); rank 0 prints the aggregate over ranks.
"""

from __future__ import annotations

import argparse
import gc
import hashlib
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)

from tsp_gpu_clean_b200 import instances  # noqa: E402

METRIC = "2-opt deltas/s"
UNIT = "deltas/s"
MODES = ("best", "first")
K_CAND = 20
#: Algorithmic work per 2-opt delta: three int32 distances d(a,c), d(b,d) and the retired
#: edges (12 B, the L2-side figure) and about 12 integer operations.
ALG_BYTES_PER_DELTA = 12
ALG_OPS_PER_DELTA = 12
L2_FLUSH_BYTES = 256 << 20
#: Per gain the scan kernel computed (128-thread CTAs, the uncounted launch of first mode,
#: the best-mode launch), from one ncu capture on the first 256 tours of the batch: warp
#: instructions executed (sm__inst_executed.sum), L2 sector bytes (lts__t_bytes.sum), and
#: DRAM bytes read + written scaled to a 1024-tour launch (the tours' 4 KB each is the part
#: that grows). A gain is computed only for entries whose lower bound could improve.
NCU_PER_GAIN: dict[str, dict[str, float]] = {
  "first": {"inst": 8.337, "lts_bytes": 32.52, "dram_bytes_per_launch": 8_486_144},
  "best": {"inst": 9.083, "lts_bytes": 31.95, "dram_bytes_per_launch": 8_617_472},
}
#: CPU parity sample: tours of the timed batch refined by the oracle (at least this many)
PARITY_TOURS = 16
GA_SUB_WORKLOAD = "ga1000"


# ----------------------------------------------------------------------------------- CPU
def _cpu_worker(args):
  """Refine one tour in best then first mode with the oracle.

  Returns ({mode: (tour, (passes, pairs, moves))}, seconds of refinement)."""
  coords, tour = args
  from oracle import distances, two_opt

  D = distances.euc2d_matrix(coords)
  cand = distances.candidate_list(K_CAND, coords=coords)
  t0 = time.perf_counter()
  out = {}
  for mode in MODES:
    t, st = two_opt.improve_batch(tour[None, :], D, cand, mode, 10**9)
    out[mode] = (t[0], tuple(int(v) for v in st[0]))
  return out, time.perf_counter() - t0


def _ref_worker(args):
  """Refine one tour in best then first mode with the reference's own CPU 2-opt (installed
  under baseline/_ref). Returns ({mode: (tour, (passes, pairs))}, seconds of refinement)."""
  coords, tour = args
  from baseline import reference_arm

  return reference_arm.two_opt_worker((coords, tour, MODES, K_CAND))


def cpu_path() -> tuple[str, object]:
  """The CPU 2-opt to time: the reference itself when it is installed, else the oracle port."""
  from baseline import reference_arm

  return ("reference", _ref_worker) if reference_arm.import_root() is not None else ("port", _cpu_worker)


def parity_indices(tours: int, count: int) -> list[int]:
  """`count` tour indices spread evenly over a batch of `tours` (first and last included)."""
  return sorted({int(round(v)) for v in np.linspace(0, tours - 1, min(count, tours))})


def cpu_sample(pool, tours_np: np.ndarray, indices, worker=_cpu_worker) -> dict:
  """CPU deltas/s over the given tours of the batch in parallel (one tour per process),
  with each tour's refined result per mode for the parity check."""
  coords, _ = instances.two_opt_workload(tours=1)
  t0 = time.perf_counter()
  res = pool.map(worker, [(coords, tours_np[i]) for i in indices])
  wall = time.perf_counter() - t0
  pairs = sum(st[1] for out, _ in res for _, st in out.values())
  return {"value": pairs / wall, "pairs": pairs, "wall_s": wall, "tours": len(indices),
          "tours_per_s": len(indices) * len(MODES) / wall, "indices": list(indices),
          "results": [out for out, _ in res]}


def cpu_one_core(pool, tours_np: np.ndarray, index: int, worker=_cpu_worker) -> dict:
  """The same CPU 2-opt on one tour with no other worker busy: deltas/s of one host core."""
  coords, _ = instances.two_opt_workload(tours=1)
  out, secs = pool.apply(worker, ((coords, tours_np[index]),))
  pairs = sum(st[1] for _, st in out.values())
  return {"value": pairs / secs, "pairs": pairs, "seconds": secs, "tours_per_s": len(MODES) / secs, "tour": index}


def refined_digest(results: list, modes=MODES) -> str:
  """sha256 over the refined tours of each sampled tour, mode by mode (equal digests from
  two arms mean identical refinements)."""
  h = hashlib.sha256()
  for out in results:
    for m in modes:
      h.update(np.ascontiguousarray(out[m][0], dtype=np.int32).tobytes())
  return h.hexdigest()


def check_parity(gpu: dict, cpu: dict, kind: str = "port") -> dict:
  """Compare the CPU refinements (the reference's or the oracle's) with the GPU's counted
  launch at the same indices."""
  bad = []
  for i, out in zip(cpu["indices"], cpu["results"]):
    for m, (tour, st) in out.items():
      g_tour, g_st = gpu[m]
      if not np.array_equal(g_tour[i], tour):
        bad.append(f"{m} tour {i}: tours differ")
      elif tuple(int(v) for v in g_st[i][: len(st)]) != tuple(st):
        bad.append(f"{m} tour {i}: (passes, pairs[, moves]) {tuple(int(v) for v in g_st[i][:len(st)])} vs {st}")
  n = len(cpu["indices"])
  total = len(next(iter(gpu.values()))[0])
  what = "the reference's CPU 2-opt" if kind == "reference" else "the oracle port"
  return {"ok": not bad, "text": (f"bit-exact against {what} on {n}/{total} tours (both modes: tours, passes, pairs)"
                                  if not bad else f"MISMATCH on {len(bad)} of {n * len(MODES)} refinements"),
          "mismatches": bad[:8]}


class GcWatch:
  """Time spent in Python's cyclic garbage collector while the block runs, per generation
  (collections pause the host thread that enqueues the GPU work)."""

  def __enter__(self):
    self.ms = [0.0, 0.0, 0.0]
    self.count = [0, 0, 0]
    self._t0 = None

    def cb(phase, info):
      if phase == "start":
        self._t0 = time.perf_counter()
      elif self._t0 is not None:
        g = int(info.get("generation", 0))
        self.ms[g] += 1e3 * (time.perf_counter() - self._t0)
        self.count[g] += 1
        self._t0 = None

    self._cb = cb
    gc.callbacks.append(cb)
    return self

  def __exit__(self, *exc):
    gc.callbacks.remove(self._cb)
    return False

  def summary(self) -> dict:
    return {"collections": self.count, "ms": [round(v, 2) for v in self.ms]}


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
  FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

  #: sampling period of nvidia-smi (ms); --clock-interval-ms changes it
  interval_ms = 200

  def __init__(self, device: int):
    self.device = device
    self.proc = None

  def __enter__(self):
    """Start sampling and wait for the first sample: nvidia-smi's start-up (NVML
    initialisation) then lies before the timed region instead of inside it."""
    import select

    self.first = []
    try:
      self.proc = subprocess.Popen(
        ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
        stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
      ready, _, _ = select.select([self.proc.stdout], [], [], 5.0)
      if ready:
        self.first.append(self.proc.stdout.readline())
    except Exception:
      self.proc = None
    return self

  def __exit__(self, *exc):
    self.lines = []
    if self.proc is not None:
      self.proc.terminate()
      try:
        out, _ = self.proc.communicate(timeout=5)
      except Exception:
        self.proc.kill()
        out = ""
      self.lines = [ln for ln in self.first + out.splitlines() if ln.strip()]

  def summary(self) -> dict:
    sm, mx, reasons = [], 0.0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in getattr(self, "lines", []):
      parts = [p.strip() for p in ln.split(",")]
      if len(parts) < 6:
        continue
      try:
        sm.append(float(parts[0]))
        mx = max(mx, float(parts[1]))
      except ValueError:
        continue
      for nm, v in zip(names, parts[2:6]):
        if v.lower().startswith("active"):
          reasons.add(nm)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
            "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------------- GPU
def _dist_env():
  world = int(os.environ.get("WORLD_SIZE", "1"))
  rank = int(os.environ.get("RANK", "0"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  return world, rank, local


def _init_ranks():
  """(world, rank) after binding this process to its GPU and, under torchrun, joining the
  NCCL process group (short timeout: ranks that wait for one another end with an error)."""
  import datetime

  import torch
  import torch.distributed as dist

  world, rank, local = _dist_env()
  torch.cuda.set_device(local)
  if world > 1 and not dist.is_initialized():
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
  return world, rank


def _barrier(world: int) -> None:
  if world > 1:
    import torch.distributed as dist

    dist.barrier()


def _finish_ranks(world: int) -> None:
  if world > 1:
    import torch.distributed as dist

    dist.destroy_process_group()


def aggregate(units: float, elapsed_s: float, world: int):
  """(sum of units over ranks, max elapsed over ranks); identity for one process."""
  if world <= 1:
    return units, elapsed_s
  import torch
  import torch.distributed as dist

  dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
  u = torch.tensor([units], dtype=torch.float64, device=dev)
  e = torch.tensor([elapsed_s], dtype=torch.float64, device=dev)
  dist.all_reduce(u, op=dist.ReduceOp.SUM)
  dist.all_reduce(e, op=dist.ReduceOp.MAX)
  return float(u.item()), float(e.item())


def two_opt_tours(count: int, rank: int) -> np.ndarray:
  """The workload's random tours of one rank (rank 0: the batch the CPU parity sample reads)."""
  return instances.random_tours(instances.TWO_OPT_N, count, instances.TWO_OPT_TOUR_SEED + 1000 * rank)


def _roofline(dominant: str, gains: int, launch_s: float, peaks: dict, tours: int, threads: int, kernel: str) -> dict:
  """The dominant launch against the L2-gather and INT32-issue ceilings measured in this run.

  Counter-based figures (instructions and L2 bytes per evaluated gain, from one ncu capture
  of the same kernel on this workload's tours) are used where they exist; otherwise the
  algorithmic ones (12 B and 12 integer operations per gain)."""
  per = NCU_PER_GAIN.get(dominant) if (kernel == "scan" and threads == 128) else None
  gps = gains / launch_s
  int_peak = peaks["int32_tops"]
  l2_peak = peaks["l2_sector_gbs"]
  alg = {"l2_gbs": gps * ALG_BYTES_PER_DELTA / 1e9, "int32_tops": gps * ALG_OPS_PER_DELTA / 1e12,
         "basis": f"{ALG_BYTES_PER_DELTA} B and {ALG_OPS_PER_DELTA} integer ops per evaluated gain"}
  alg["l2_frac_of_useful"] = alg["l2_gbs"] / peaks["l2_useful_gbs"]
  alg["int32_frac"] = alg["int32_tops"] / int_peak
  if per is not None:
    int_ach = gps * per["inst"] * 32 / 1e12  # warp instructions issued, as lane operations
    l2_ach = gps * per["lts_bytes"] / 1e9
    basis = (f"ncu per evaluated gain: {per['inst']:.2f} warp instructions, {per['lts_bytes']:.2f} L2 sector bytes; "
             f"x {gains} gains per launch / {launch_s * 1e3:.2f} ms")
  else:  # one 32-byte sector per gain (the matrix gather) and the algorithmic integer work
    int_ach, l2_ach = alg["int32_tops"], gps * 32 / 1e9
    basis = ("no ncu figure for this launch shape: one 32-byte L2 sector and " f"{ALG_OPS_PER_DELTA} integer ops "
             "per evaluated gain")
  l2 = {"achieved": l2_ach, "peak": l2_peak, "unit": "GB/s", "frac": l2_ach / l2_peak}
  i32 = {"achieved": int_ach, "peak": int_peak, "unit": "TOP/s", "frac": int_ach / int_peak}
  top = i32 if i32["frac"] >= l2["frac"] else l2
  traffic = None
  if per is not None and tours == instances.TWO_OPT_TOURS:
    traffic = per.get("dram_bytes_per_launch")
  return {"bound": "int32" if top is i32 else "l2", "achieved": top["achieved"], "peak": top["peak"],
          "unit": top["unit"], "frac": top["frac"], "traffic": traffic,
          "kernel": f"two_opt_{kernel}_kernel<{dominant}>", "peak_source": "measured in this run: " + peaks["method"],
          "basis": basis, "int32": i32, "l2": l2, "algorithmic": alg,
          "hbm_note": "DRAM traffic is the matrix, the packed k-NN table and the tours once per launch; HBM is "
                      "not the bound"}


def run_gpu(args, world: int, rank: int) -> dict:
  import torch

  from tsp_gpu_clean_b200 import native, roofline
  from tsp_gpu_clean_b200.device import operands_for, ptr, stream_handle
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext
  from tsp_gpu_clean_b200.strategies.local_search import LocalSearchB200TourTwoOpt

  local = int(os.environ.get("LOCAL_RANK", "0"))
  lib = native.load_library()
  coords, _ = instances.two_opt_workload(tours=1)
  tours_np = two_opt_tours(args.tours, rank)
  n = instances.TWO_OPT_N
  ctx = ProblemContext(Problem.from_coordinates(coords, "clustered1000"), seed=0)
  ops = operands_for(ctx)
  dist_t, stride, _ = ops.distance_args(n)
  coords_t = None
  if args.distances == "coords":  # the same int32 EUC_2D values, rebuilt in FP64 from L1-resident coordinates
    dist_t, stride, coords_t = None, 0, ops.coords()
  tabs = ops.candidates(K_CAND, ctx.get_cpu_candidate_list(K_CAND), n)
  k = tabs.k
  # the reverse index selects the cached kernel, or (with the packed table) the incremental
  # restart of the scan kernel's first mode
  use_rev = args.kernel == "cached" or (args.kernel == "scan" and args.first_restart == "incremental")
  rev_off = tabs.rev_off if use_rev else None
  rev_idx = tabs.rev_idx if use_rev else None
  packed = tabs.packed if args.kernel == "scan" else None
  pristine = torch.from_numpy(tours_np).cuda()
  modes = MODES if args.mode == "both" else (args.mode,)
  work = {m: torch.empty_like(pristine) for m in modes}
  stats = {m: torch.zeros((args.tours, 4), dtype=torch.int64, device="cuda") for m in modes}
  status = torch.zeros(args.tours, dtype=torch.int32, device="cuda")
  flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
  stream = torch.cuda.current_stream()

  sym = native.TSPB_MODE_SYMMETRIC if ops.symmetric else 0  # as the strategy decides it

  def launch(m, counted):
    rc = lib.tspb_two_opt(ptr(work[m]), args.tours, n, ptr(dist_t), stride, ptr(coords_t), ptr(tabs.cand),
                          ptr(tabs.cand_dist), ptr(rev_off), ptr(rev_idx), ptr(packed), k, native.MODE_CODES[m] | sym,
                          args.max_iter, args.threads, ptr(stats[m]) if counted else None, ptr(status), None, 0,
                          stream_handle())
    native.check("tspb_two_opt", rc)

  def check_status():
    bad = int(status.max().item())
    if bad != 0:
      raise RuntimeError(f"2-opt kernel reported {native.status_text(bad)}")

  # the counted launch (untimed): pair, pass, move and gain counts, and the tours every
  # timed launch must reproduce
  counted = {}
  for m in modes:
    work[m].copy_(pristine)
    launch(m, True)
  torch.cuda.synchronize()
  check_status()
  for m in modes:
    counted[m] = (work[m].cpu().numpy(), stats[m].cpu().numpy())

  def step(ev):
    for m in modes:
      work[m].copy_(pristine)
      ev[m][0].record(stream)
      launch(m, False)
      ev[m][1].record(stream)

  def new_events():
    return {m: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for m in modes}

  for _ in range(args.warmup):
    step(new_events())
  torch.cuda.synchronize()
  check_status()
  peaks = roofline.measure_peaks()  # the scan's ceilings on this device, before the timed region

  per_step = []
  _barrier(world)
  torch.cuda.synchronize()
  with ClockSampler(local) as clocks:
    for _ in range(args.steps):
      flush.fill_(1)
      ev = new_events()
      step(ev)
      per_step.append(ev)
    torch.cuda.synchronize()
  _barrier(world)
  check_status()
  for m in modes:
    if not np.array_equal(work[m].cpu().numpy(), counted[m][0]):
      raise RuntimeError(f"{m}: a timed launch returned other tours than the counted launch")
  kernel_ms = {m: sum(e[m][0].elapsed_time(e[m][1]) for e in per_step) for m in modes}
  total_ms = sum(kernel_ms.values())
  st = {m: counted[m][1] for m in modes}
  pairs_step = sum(int(st[m][:, 1].sum()) for m in modes)
  eval_step = sum(int(st[m][:, 3].sum()) for m in modes)
  units_all, elapsed = aggregate(pairs_step * args.steps, total_ms / 1e3, world)
  tours_all, _ = aggregate(args.tours * len(modes) * args.steps, total_ms / 1e3, world)
  value = units_all / elapsed

  # end to end: the public strategy call on host tours (pinned H2D + kernel + D2H); no
  # stats requested, like the timed launches; the counts are the counted launch's
  e2e_ms = 0.0
  strategies = {m: LocalSearchB200TourTwoOpt(max_iterations=args.max_iter, mode=m, candidate_k=K_CAND,
                                              threads_per_block=args.threads) for m in modes}
  for s_ in strategies.values():
    s_.kernel = args.kernel
    s_.incremental_first = args.first_restart == "incremental"
    s_.collect_stats = False
  for m in modes:
    strategies[m].improve_batch(tours_np, ctx)  # warm
  torch.cuda.synchronize()
  e2e_pairs = 0
  for _ in range(args.steps):
    for m in modes:
      e0 = torch.cuda.Event(enable_timing=True)
      e1 = torch.cuda.Event(enable_timing=True)
      e0.record(stream)
      out = strategies[m].improve_batch(tours_np, ctx)
      e1.record(stream)
      torch.cuda.synchronize()
      e2e_ms += e0.elapsed_time(e1)
      if not np.array_equal(out, counted[m][0]):
        raise RuntimeError(f"{m}: the public call returned other tours than the counted launch")
      e2e_pairs += int(st[m][:, 1].sum())
  e2e_units, e2e_elapsed = aggregate(e2e_pairs, e2e_ms / 1e3, world)
  del out

  dominant = max(modes, key=lambda m: kernel_ms[m])
  launches = args.steps * len(modes)
  dom_s = kernel_ms[dominant] / args.steps / 1e3
  dom_eval = int(st[dominant][:, 3].sum())
  return {
    "value": value,
    "ms_per_step": total_ms / args.steps,
    "kernel_ms_per_step": {m: kernel_ms[m] / args.steps for m in modes},
    "tours_per_s": tours_all / elapsed,
    "pairs_per_step": pairs_step,
    "evaluated_per_step": eval_step,
    "passes_per_step": {m: int(st[m][:, 0].sum()) for m in modes},
    "moves_per_step": {m: int(st[m][:, 2].sum()) for m in modes},
    "clocks": clocks.summary(),
    "e2e": {"value": e2e_units / e2e_elapsed, "unit": UNIT,
            "h2d_bytes_per_step": int(tours_np.nbytes * len(modes)),
            "d2h_bytes_per_step": int(tours_np.nbytes * len(modes) + 4 * len(modes))},  # tours + status max
    "gpu_launches": launches,
    "roofline": _roofline(dominant, dom_eval, dom_s, peaks, args.tours, args.threads, args.kernel),
    "peaks": peaks,
    "counted": counted,
    "tours_np": tours_np,
  }


GA_WORKLOADS = {
  # name: (n, population, generations, elite, post_init, instance seed, description)
  "ga100": (100, 128, 50, 16, True, 42, "memetic GA, 100 uniform cities, population 128, 50 generations, NN init k=5, "
                                        "tournament 5, PMX, inversion 0.05, 2-opt best k=20 x10 post-init and on 16 elites"),
  "ga1000": (1000, 512, 100, 64, False, 1000, "memetic GA, 1000 uniform cities, population 512, 100 generations, 64 elites "
                                               "2-opt best k=20 x10, tournament 5, PMX, inversion 0.05"),
  "ga2000": (2000, 512, 200, 64, False, 2000, "memetic GA, 2000 uniform cities, population 512, 200 generations, 64 elites "
                                               "2-opt best k=20 x10, tournament 5, PMX, inversion 0.05"),
  "chapter4": (1002, 256, 200, 0, False, 1002, "GA in the reference's published Chapter-4 configuration on a 1002-city "
                                               "uniform instance: population 256, random-permutation init, tournament 5, "
                                               "OX, swap 0.02, 2-opt best k=20 x10 on every child (post_mutation), "
                                               "200 generations"),
  "chapter4x30": (1002, 256, 200, 0, False, 1002, "the chapter4 workload's 30 repetitions (generators seeded 42..71) "
                                                  "advanced together as one batch"),
}
# Operators and stage of each GA workload (defaults: the memetic configuration of the path).
GA_DEFAULT_OPTIONS = {"rate": 0.05, "crossover": "pmx", "mutation": "inversion", "init": "nn", "stage": "none",
                      "reps": 1}
GA_OPTIONS = {
  "chapter4": {"rate": 0.02, "crossover": "ox", "mutation": "swap", "init": "random", "stage": "post_mutation"},
  "chapter4x30": {"rate": 0.02, "crossover": "ox", "mutation": "swap", "init": "random", "stage": "post_mutation",
                  "reps": 30},
}


def ga_options(name: str) -> dict:
  return {**GA_DEFAULT_OPTIONS, **GA_OPTIONS.get(name, {})}


def _ga_cpu_gens_per_s(name: str, sample_gens: int) -> dict:
  """GA generations/s on one core: the reference's own `GeneticAlgorithm.evolve` with its
  CPU strategies when it is installed (baseline/_ref), else the oracle GA (the NumPy
  restatement of the same GA, pinned to the reference's recorded runs)."""
  n, P, G, elite, post_init, seed, _ = GA_WORKLOADS[name]
  o = ga_options(name)
  coords = instances.uniform_instance(n, seed)
  if cpu_path()[0] == "reference":
    from baseline import reference_arm

    r = reference_arm.ga_gens_per_s(coords, P, elite, post_init, sample_gens, o)
    return {**r, "kind": "reference", "what": "the reference's GeneticAlgorithm.evolve with its CPU strategies"}
  from oracle import distances as odist
  from oracle import ga as oga

  D = odist.euc2d_matrix(coords)
  cache = {}

  def provider(k):
    if k not in cache:
      cache[k] = odist.candidate_list(k, coords=coords)
    return cache[k]

  cfg = oga.GAConfig(population_size=P, mutation_rate=o["rate"], nn_k=5, tournament_k=5,
                     local_search=oga.LocalSearchSpec("best", 10, 20), post_init=post_init, elite_count=elite or None,
                     local_search_stage=o["stage"], crossover=o["crossover"], mutation=o["mutation"], init=o["init"])
  provider(5), provider(20)
  t0 = time.perf_counter()
  oga.OracleGA(D, provider, cfg, np.random.default_rng(42)).evolve(0, patience=10**9)
  t1 = time.perf_counter()
  res = oga.OracleGA(D, provider, cfg, np.random.default_rng(42)).evolve(sample_gens, patience=10**9)
  t2 = time.perf_counter()
  loop = max((t2 - t1) - (t1 - t0), 1e-9)
  return {"value": sample_gens / loop, "gens": sample_gens, "loop_s": loop,
          "history": [float(v) for v in res[3]["convergence_history"]], "kind": "port", "what": "the NumPy GA"}


def _ga_cpu_sample(name: str, sample_gens: int) -> dict:
  """CPU baseline of a GA workload: one oracle run on one core, or for a workload of R
  repetitions R oracle runs over min(R, host cores) spawned processes (aggregate rate =
  R * sample generations over the mean per-process busy time)."""
  reps = ga_options(name)["reps"]
  if reps == 1:
    r = _ga_cpu_gens_per_s(name, sample_gens)
    return {"value": r["value"], "cores": 1, "loop_s": r["loop_s"], "history": r["history"], "kind": r["kind"],
            "sample": f"{sample_gens} generations of {r['what']} (init excluded), {r['loop_s']:.1f} s"}
  import multiprocessing as mp

  workers = max(1, min(reps, os.cpu_count() or 1, 64))
  with mp.get_context("spawn").Pool(workers) as pool:
    res = pool.starmap(_ga_cpu_gens_per_s, [(name, sample_gens)] * reps)
  busy = sum(r["loop_s"] for r in res) / workers
  return {"value": reps * sample_gens / busy, "cores": workers, "loop_s": busy, "kind": res[0]["kind"],
          "sample": f"{reps} runs x {sample_gens} generations of {res[0]['what']} (init excluded) on {workers} "
                    f"processes, {busy:.1f} s per process"}


def ga_measure(workload: str, warmup: int, steps: int, world: int, rank: int, engine: str = "batch", chunk: int = 16,
               no_graph: bool = False, batch_incremental: str = "off", generations: int | None = None,
               batch_pair: str = "auto") -> dict:
  """Device and end-to-end generations/s of one GA workload on this rank's GPU (the
  process group, if any, is the caller's)."""
  import torch

  from tsp_gpu_clean_b200.fused import FusedMemeticSolver, LocalSearchConfig
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  n, P, G, elite, post_init, seed, desc = GA_WORKLOADS[workload]
  G = generations or G
  o = ga_options(workload)
  reps = o["reps"]
  coords = instances.uniform_instance(n, seed)

  from tsp_gpu_clean_b200.autotune import BatchAutotuner
  from tsp_gpu_clean_b200.batch import FusedBatchSolver

  tuner = BatchAutotuner()
  if engine != "batch" and (reps > 1 or o != GA_DEFAULT_OPTIONS):
    raise SystemExit(f"--engine single does not run the {workload} workload")

  def run_once():
    # replicas per rank: the same instance, each run's generator seeded per rank and repetition
    # like the reference's runner: one problem, one candidate cache, a context per repetition
    problem, cache = Problem.from_coordinates(coords), {}
    ctxs = [ProblemContext(problem, seed=42 + r + reps * rank, candidate_cache=cache) for r in range(reps)]
    ls = LocalSearchConfig("best", 10, 20)
    gc.collect()  # the previous runs' garbage, outside the timed call
    t0 = time.perf_counter()
    if engine == "batch":
      solver = FusedBatchSolver(population_size=P, mutation_rate=o["rate"], tournament_k=5, nn_k=5, local_search=ls,
                                elite_count=elite, post_init=post_init, max_matrix_dimension=None, tuner=tuner,
                                chunk=chunk, use_graph=not no_graph, crossover=o["crossover"],
                                mutation=o["mutation"], init=o["init"], local_search_stage=o["stage"],
                                incremental=batch_incremental, pair=batch_pair)
      results = solver.evolve(ctxs, G, patience=10**9)
      stats = {"generations_completed": sum(st["generations_completed"] for _, st in results),
               "best_fitness": min(st["best_fitness"] for _, st in results),
               "history": results[0][1]["convergence_history"]}
    else:
      solver = FusedMemeticSolver(population_size=P, mutation_rate=0.05, tournament_k=5, nn_k=5, local_search=ls,
                                  elite_count=elite, post_init=post_init, chunk=chunk, engine="single",
                                  use_graph=not no_graph)
      best, stats = solver.evolve(ctxs[0], list(range(n)), G, patience=10**9)
      stats = {**stats, "history": stats["convergence_history"]}
    wall = time.perf_counter() - t0
    return solver, stats, wall

  for _ in range(warmup):
    run_once()
  torch.cuda.synchronize()
  _barrier(world)
  loop_ms, walls, launches, gens, phases = [], [], 0, 0, []
  with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks, GcWatch() as gcw:
    for _ in range(steps):
      solver = stats = None  # the previous run's buffers are released before the next timed call
      solver, stats, wall = run_once()
      loop_ms.append(solver.last_timing["loop_ms_device"])
      phases.append({k: round(solver.last_timing[k] * 1e3, 2) for k in ("setup_s", "postinit_s", "capture_s", "loop_s")
                     if k in solver.last_timing})
      walls.append(wall)
      launches += solver.kernel_launches
      gens += stats["generations_completed"]
  torch.cuda.synchronize()
  _barrier(world)
  units, loop_s = aggregate(gens, sum(loop_ms) / 1e3, world)
  e2e_units, wall_s = aggregate(gens, sum(walls), world)
  value = units / loop_s
  return {"value": value, "ms_per_step": 1e3 * loop_s / steps, "clocks": clocks.summary(), "world": world,
          "rank": rank,
          "e2e": {"value": e2e_units / wall_s, "unit": "generations/s", "h2d_bytes_per_step": int(reps * coords.nbytes),
                  "d2h_bytes_per_step": int(reps * (n * 4 + (G + 1) * 8 + P * n * 4))},
          "gpu_launches": launches, "desc": desc, "best": stats["best_fitness"], "history": stats["history"],
          "loop_ms_steps": [round(v, 3) for v in loop_ms], "walls_s": [round(w, 4) for w in walls],
          "phase_ms_steps": phases, "gc": gcw.summary(),
          "buckets": [{"n": [b.lo, b.hi], "two_opt_threads": b.two_opt_threads, "incremental": b.incremental, "pair": b.pair,
                       "offspring_threads": b.offspring_threads} for b in getattr(solver, "buckets", [])],
          "two_opt_totals": getattr(solver, "two_opt_totals", None),
          "timing": {k: round(v, 4) for k, v in solver.last_timing.items() if isinstance(v, (int, float))}}


def run_ga_bench(args) -> dict:
  from tsp_gpu_clean_b200.build import build_library

  world, rank = _init_ranks()
  build_library()
  try:
    return ga_measure(args.workload, args.warmup, args.steps, world, rank, engine=args.engine, chunk=args.chunk,
                      no_graph=args.no_graph, batch_incremental=args.batch_incremental, batch_pair=args.batch_pair)
  finally:
    _finish_ranks(world)


# ------------------------------------------------------------------------ uneven batch
UNEVEN_SEED = 4242
UNEVEN_DESC = ("uneven batch: {count} instances, n log-uniform in [50, 5000] (half uniform, half 10-50-cluster "
               "mixtures), population 64, {G} generations, NN init k=5, tournament 5, PMX, inversion 0.05, 2-opt best "
               "k=20 x10 post-init and on 8 elites; n > 4096 rebuilds distances from FP64 coordinates; one CUDA "
               "graph replay per generation")


def _knn_tables(c):
  from tsp_gpu_clean_b200.problem import compute_candidate_list

  return {5: compute_candidate_list(5, coords=c), 20: compute_candidate_list(20, coords=c)}


def _uneven_inputs(count: int, pool=None, seed: int = UNEVEN_SEED):
  """Coordinates of the batch and their host k-NN tables (k = 5 for the NN init, 20 for
  2-opt), computed once like a ProblemContext's candidate cache (on the host cores)."""
  coords = instances.uneven_batch(count, seed)
  order = sorted(range(count), key=lambda i: -len(coords[i]))  # largest first for the pool
  if pool is not None:
    tabs = pool.map(_knn_tables, [coords[i] for i in order], chunksize=1)
  else:
    tabs = [_knn_tables(coords[i]) for i in order]
  caches = [None] * count
  for i, t in zip(order, tabs):
    caches[i] = t
  return coords, caches


def _uneven_cpu_worker(args):
  """GA generations/s on one instance of the batch (init excluded): the reference's own
  GeneticAlgorithm.evolve with its CPU strategies when it is installed, else the oracle GA."""
  coords, cache, seed, gens = args
  if cpu_path()[0] == "reference":
    from baseline import reference_arm

    r = reference_arm.ga_gens_per_s(coords, 64, 8, True, gens, dict(GA_DEFAULT_OPTIONS), seed=seed)
    return gens, r["loop_s"], len(coords)
  from oracle import distances as odist
  from oracle import ga as oga

  D = odist.euc2d_matrix(coords)
  cfg = oga.GAConfig(population_size=64, mutation_rate=0.05, nn_k=5, tournament_k=5,
                     local_search=oga.LocalSearchSpec("best", 10, 20), post_init=True, elite_count=8)
  t0 = time.perf_counter()
  oga.OracleGA(D, cache.__getitem__, cfg, np.random.default_rng(seed)).evolve(0, patience=10**9)
  t1 = time.perf_counter()
  oga.OracleGA(D, cache.__getitem__, cfg, np.random.default_rng(seed)).evolve(gens, patience=10**9)
  t2 = time.perf_counter()
  return gens, max((t2 - t1) - (t1 - t0), 1e-9), len(coords)


def uneven_cpu_sample(pool, workers: int, coords, caches, gens: int) -> dict:
  """Aggregate CPU generations/s (the reference's GA, else the oracle's) over a
  size-stratified sample of the batch, one instance per process (evenly spaced instances
  in size order)."""
  order = sorted(range(len(coords)), key=lambda i: len(coords[i]))
  step = max(1, len(order) // workers)
  pick = [order[min(j * step + step // 2, len(order) - 1)] for j in range(min(workers, len(order)))]
  t0 = time.perf_counter()
  res = pool.map(_uneven_cpu_worker, [(coords[i], caches[i], 1000 + i, gens) for i in pick], chunksize=1)
  wall = time.perf_counter() - t0
  # each process runs one GA at a time; the aggregate is the sum of the per-process rates
  value = sum(g / t for g, t, _ in res)
  return {"value": value, "instances": len(pick), "sizes": [n for _, _, n in res], "wall_s": wall, "gens": gens,
          "kind": cpu_path()[0]}


def run_uneven_bench(args) -> dict:
  import torch

  from tsp_gpu_clean_b200.autotune import BatchAutotuner
  from tsp_gpu_clean_b200.batch import FusedBatchSolver
  from tsp_gpu_clean_b200.build import build_library
  from tsp_gpu_clean_b200.fused import LocalSearchConfig
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext

  world, rank = _init_ranks()
  build_library()
  coords, caches = args.uneven_inputs
  G = args.generations
  tuner = BatchAutotuner()

  def run_once():
    ctxs = [ProblemContext(Problem.from_coordinates(c), seed=1000 + i, candidate_cache=dict(caches[i]))
            for i, c in enumerate(coords)]
    solver = FusedBatchSolver(population_size=64, mutation_rate=0.05, tournament_k=5, nn_k=5,
                              local_search=LocalSearchConfig("best", 10, 20), elite_count=8, post_init=True,
                              max_matrix_dimension=4096, tuner=tuner, chunk=args.chunk,
                              use_graph=not args.no_graph, incremental=args.batch_incremental,
                              pair=args.batch_pair)
    gc.collect()  # the previous runs' garbage, outside the timed call
    t0 = time.perf_counter()
    res = solver.evolve(ctxs, G, patience=10**9)
    wall = time.perf_counter() - t0
    return solver, res, wall

  for _ in range(args.warmup):
    run_once()
  torch.cuda.synchronize()
  _barrier(world)
  loop_ms, walls, launches, gens, pairs, tune_s, pauses, ties = [], [], 0, 0, 0, 0.0, 0, 0
  phases = []
  with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks, GcWatch() as gcw:
    for _ in range(args.steps):
      solver = res = None  # the previous run's buffers are released before the next timed call
      mallocs = torch.cuda.memory_stats().get("segment.all.allocated", 0)
      solver, res, wall = run_once()
      loop_ms.append(solver.last_timing["loop_ms_device"])
      walls.append(wall)
      phases.append({**{k: round(solver.last_timing[k] * 1e3, 2)
                        for k in ("setup_s", "setup_operands_s", "postinit_s", "capture_s", "loop_s", "results_s")},
                     "device_mallocs": torch.cuda.memory_stats().get("segment.all.allocated", 0) - mallocs})
      launches += solver.kernel_launches
      gens += sum(st["generations_completed"] for _, st in res)
      pairs += solver.two_opt_totals["pairs"]
      tune_s += solver.last_timing["tune_s"]
      pauses += sum(st["host_elite_generations"] for _, st in res)
      ties += sum(st["elite_edge_ties"] for _, st in res)
  torch.cuda.synchronize()
  _barrier(world)
  all_gens, loop_s = aggregate(gens, sum(loop_ms) / 1e3, world)
  e2e_gens, wall_s = aggregate(gens, sum(walls), world)
  all_pairs, _ = aggregate(pairs, 0.0, world)
  _finish_ranks(world)
  total_n = sum(len(c) for c in coords)
  h2d = sum(c.nbytes for c in coords) + sum(len(c) * (5 + 20) * 4 for c in coords)
  h2d += len(coords) * G * 64 * (5 * 4 + 4 + 8 + 2 * 4)  # the tape
  d2h = total_n * 4 + len(coords) * (G + 1) * 8
  return {"value": all_gens / loop_s, "ms_per_step": 1e3 * loop_s / args.steps, "clocks": clocks.summary(),
          "world": world, "rank": rank,
          "e2e": {"value": e2e_gens / wall_s, "unit": "generations/s", "h2d_bytes_per_step": int(h2d * world),
                  "d2h_bytes_per_step": int(d2h * world)},
          "gpu_launches": launches,
          "detail": {"deltas_per_s": all_pairs / loop_s, "tours_evaluated_per_s": all_gens * (64 + 8) / loop_s,
                     "replays_per_step": solver.replays, "host_checks_per_step": solver.last_timing["rounds"],
                     "generations_per_step": gens // args.steps,
                     "elite_edge_ties_per_step": ties // args.steps, "host_pauses_per_step": pauses // args.steps,
                     "buckets": [{"n": [b.lo, b.hi], "coords": b.coords, "instances": len(b.items),
                                  "two_opt_threads": b.two_opt_threads, "incremental": b.incremental, "pair": b.pair,
                                  "offspring_threads": b.offspring_threads}
                                 for b in solver.buckets],
                     "setup_s": solver.last_timing["setup_s"], "tune_s_total": tune_s,
                     "last_run": {k: round(v, 4) for k, v in solver.last_timing.items() if isinstance(v, (int, float))},
                     "walls_s": [round(w, 4) for w in walls], "gc": gcw.summary(), "phase_ms_steps": phases,
                     "setup_parts_s": {k: round(solver.last_timing[k], 3)
                                       for k in ("setup_operands_s", "setup_tape_s", "setup_nn_init_s")}}}


def main_uneven(args) -> int:
  world, rank, _ = _dist_env()
  count, G = args.instances, args.generations
  config = {"workload": UNEVEN_DESC.format(count=count, G=G), "instances": count, "population": 64, "generations": G,
            "elite": 8, "seed": UNEVEN_SEED,
            "l2": "not flushed: the matrices of the batch (about 1.9 GB) exceed L2 and are re-read every generation"}
  workers = args.cpu_workers or min(os.cpu_count() or 1, 64)
  sample_gens = args.cpu_gens or 2
  if args.impl == "reference":
    if rank != 0:
      return 0
    with mp.get_context("spawn").Pool(workers) as pool:
      coords, caches = _uneven_inputs(count, pool)
      vals = [uneven_cpu_sample(pool, workers, coords, caches, sample_gens) for _ in range(max(1, args.steps))]
    value = statistics.mean(v["value"] for v in vals)
    line = {"metric": "generations/s (aggregate over instances)", "value": value, "unit": "generations/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * count * G / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic (seeded)", "impl": "reference", "config": config,
            "cpu_baseline": {"value": value, "unit": "generations/s", "cores": workers, "kind": vals[0]["kind"],
                             "sample": f"{vals[0]['instances']} size-stratified instances (n = {vals[0]['sizes']}), "
                                       f"{sample_gens} generations each, one process per instance"},
            "e2e": {"value": value, "unit": "generations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0
  # weak scaling: every rank gets its own batch of `count` instances (rank-specific seed)
  pool = mp.get_context("spawn").Pool(max(1, workers // max(world, 1)))  # before the first CUDA call
  args.uneven_inputs = _uneven_inputs(count, pool, seed=UNEVEN_SEED + 7919 * rank)
  if rank != 0 or world != 1 or args.no_cpu_baseline:
    pool.close()
    pool.join()
    pool = None
  res = run_uneven_bench(args)
  if res["rank"] != 0:
    return 0
  if res["world"] > 1:
    config["parallelism"] = f"{res['world']} ranks, each its own {count}-instance batch (weak scaling, no collective)"
  line = {"metric": "generations/s (aggregate over instances)", "value": res["value"], "unit": "generations/s",
          "n_gpus": res["world"], "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
          "data": "synthetic (seeded)", "config": config, "clocks": res["clocks"], "e2e": res["e2e"],
          "gpu_launches": res["gpu_launches"], "detail": res["detail"]}
  if pool is not None:
    coords, caches = args.uneven_inputs
    cpu = uneven_cpu_sample(pool, workers, coords, caches, sample_gens)
    pool.close()
    pool.join()
    line["cpu_baseline"] = {"value": cpu["value"], "unit": "generations/s", "cores": workers, "kind": cpu["kind"],
                            "sample": f"{cpu['instances']} size-stratified instances (n = {cpu['sizes']}), "
                                      f"{sample_gens} generations each, one process per instance, {cpu['wall_s']:.1f} s"}
  print(json.dumps(line))
  return 0


#: Algorithmic FLOPs of one edge's training gradient: the three row-wise products
#: (x W1 with K padded to 16, h1 W2, dh2 W2^T) and the sums over edges for dW2 and dW1.
MLP_FLOPS_PER_EDGE = 2 * (16 * 64 + 64 * 64 + 64 * 64 + 64 * 64 + 16 * 64)


def main_mlp_train(args) -> int:
  """Training-gradient throughput of the edge-scoring MLP: the tcgen05 kernel (accumulators
  in tensor memory) against the mma.sync kernel, on one synthetic batch of 65,536 edges
  (the training batch of the learned-candidate workload), CUDA-event timed."""
  import torch

  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.build import build_library
  from tsp_gpu_clean_b200.device import ptr, stream_handle
  from tsp_gpu_clean_b200.learned import EdgeScorer

  build_library()
  E = args.mlp_edges
  rng = np.random.default_rng(7)
  x = np.zeros((E, 16), dtype=np.float32)
  x[:, :5] = rng.uniform(-2, 2, (E, 5))
  xb = (x.view(np.uint32) >> 16).astype(np.uint16)  # truncation suffices for synthetic inputs
  dx = torch.from_numpy(xb.view(np.int16).copy()).cuda()
  dy = torch.from_numpy((rng.random(E) < 0.1).astype(np.float32)).cuda()
  sc = EdgeScorer(seed=1)
  grad = torch.zeros_like(sc.params)
  loss = torch.zeros(1, dtype=torch.float32, device="cuda")
  status = torch.zeros(1, dtype=torch.int32, device="cuda")
  lib = native.load_library()

  def launch(tc: bool):
    if tc:
      rc = lib.tspb_mlp_train_grad_tc(ptr(sc.params), ptr(dx), ptr(dy), E, ptr(grad), ptr(loss), ptr(status),
                                      stream_handle())
    else:
      rc = lib.tspb_mlp_train_grad(ptr(sc.params), ptr(dx), ptr(dy), E, ptr(grad), ptr(loss), stream_handle())
    native.check("mlp train", rc)

  res = {}
  for name, tc in (("tcgen05", True), ("mma_sync", False)):
    for _ in range(args.warmup):
      launch(tc)
    torch.cuda.synchronize()
    ms = []
    for _ in range(args.steps):
      e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
      e0.record()
      launch(tc)
      e1.record()
      e1.synchronize()
      ms.append(e0.elapsed_time(e1))
    res[name] = statistics.median(ms)
  if int(status.item()) != 0:
    raise RuntimeError("tcgen05 kernel reported a completion wait that ran out")
  peak = 1590.0  # dense BF16 TFLOP/s: MEASURED_PEAKS.json when present, else the pool's fallback
  src = "fallback"
  path = os.path.join(ROOT, "MEASURED_PEAKS.json")
  if os.path.exists(path):
    with open(path) as fh:
      d = json.load(fh)
    if "bf16_tflops" in d:
      peak, src = float(d["bf16_tflops"]), "measured"
  tf = {k: E * MLP_FLOPS_PER_EDGE / (v / 1e3) / 1e12 for k, v in res.items()}
  print(json.dumps({"metric": "MLP training-gradient edges/s", "value": E / (res["tcgen05"] / 1e3), "unit": "edges/s",
                    "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                    "dtype": "bf16 operands, fp32 accumulate", "data": "synthetic (seeded)",
                    "config": {"workload": "edge-scoring MLP 5(16)-64-64-1 training gradient, one batch", "edges": E},
                    "ms": res, "tflops": tf,
                    "roofline": {"bound": "tensor", "achieved": tf["tcgen05"], "peak": peak, "unit": "TFLOP/s",
                                 "frac": tf["tcgen05"] / peak, "peak_source": src,
                                 "basis": f"{MLP_FLOPS_PER_EDGE} algorithmic FLOPs per edge"}}))
  return 0


def run_learned_bench(args) -> dict:
  """Learned top-10 vs k-NN top-20 candidates for 2-opt at equal wall time.

  Train: `args.train_instances` generated instances (n log-uniform in [200, 2000], half
  uniform, half 10-50-cluster mixtures); labels are the edges of the best tour that the
  memetic GA produces on the instance (nearest-neighbour starts refined to a 2-opt local
  optimum, then `args.ga_label_generations` generations of the fused GA).
  Evaluate at n = 1000, 5000, 10000: both arms run iterated 2-opt under the same CUDA-event
  time budget (`args.ils_factor` times the k-NN arm's first descent): the same
  nearest-neighbour starts refined to a local optimum (best mode) with the arm's table, then
  rounds of `args.ils_kicks` double-bridge kicks of the best tour, refined in one launch.
  The learned arm's budget also pays for building its table (features, MLP, top-k). Gap =
  best length / best length found by any arm - 1. Learned lists of 12 and 14 entries are
  reported beside the 10-entry headline.
  """
  import torch

  from tsp_gpu_clean_b200 import learned
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  lc = learned.LearnedCandidates(pool_k=30, seed=0)
  rng = np.random.default_rng(2024)
  t0 = time.perf_counter()
  xs, ys = [], []
  for i in range(args.train_instances):
    n = int(round(np.exp(rng.uniform(np.log(200), np.log(2000)))))
    coords = (instances.uniform_instance(n, 10_000 + i) if i % 2 == 0
              else instances.clustered_instance(n, int(rng.integers(10, 51)), 30.0, 10_000 + i))
    inst = learned.device_instance(coords, 30)
    tour = lc.label_tour(inst, starts=4, seed=i, ga_generations=args.ga_label_generations)
    x, y = lc.training_edges(inst, tour)
    xs.append(x)
    ys.append(y)
  torch.cuda.synchronize()
  t_data = time.perf_counter() - t0
  t_train = lc.fit(xs, ys, epochs=3, batch=1 << 16, lr=3e-3)
  edges = sum(int(x.shape[0]) for x in xs)
  del xs, ys

  def timed(fn):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1) / 1e3

  sizes = (10, 12, 14)
  rows = []
  for n in (1000, 5000, 10000):
    for j in range(args.eval_instances):
      seed = 90_000 + 100 * n + j
      coords = instances.uniform_instance(n, seed) if j % 2 == 0 else instances.clustered_instance(n, 30, 30.0, seed)
      inst = learned.device_instance(coords, 30)
      starts = learned.nn_starts(inst, args.eval_starts, seed)
      knn20 = inst.pool[:, :20].contiguous()
      (t_k, _), descent_k = timed(lambda: learned.two_opt_table(inst, starts, knn20, mode="best"))
      budget = args.ils_factor * descent_k
      knn = learned.iterated_two_opt(inst, starts, knn20, budget, args.ils_kicks, seed)
      row = {"n": n, "budget_s": budget, "knn": knn["length"], "knn_rounds": knn["rounds"],
             "knn_recall": learned.edge_recall(knn20, knn["tour"])}
      for k in sizes:
        tab, t_tab = timed(lambda: lc.table(inst, k))
        got = learned.iterated_two_opt(inst, starts, tab, budget, args.ils_kicks, seed, spent_s=t_tab)
        row[f"learned{k}"] = got["length"]
        row[f"learned{k}_rounds"] = got["rounds"]
        row[f"learned{k}_table_s"] = t_tab
        row[f"learned{k}_recall_of_knn_tour"] = learned.edge_recall(tab, knn["tour"])
      ref = min(row["knn"], *(row[f"learned{k}"] for k in sizes))
      row["knn_gap"] = row["knn"] / ref - 1
      for k in sizes:
        row[f"learned{k}_gap"] = row[f"learned{k}"] / ref - 1
      rows.append(row)
  by_n = {}
  for n in (1000, 5000, 10000):
    rs = [r for r in rows if r["n"] == n]
    d = {"knn_gap_pct": 100 * float(np.mean([r["knn_gap"] for r in rs])),
         "budget_s": float(np.mean([r["budget_s"] for r in rs])),
         "knn_rounds": float(np.mean([r["knn_rounds"] for r in rs]))}
    for k in sizes:
      d[f"learned{k}_gap_pct"] = 100 * float(np.mean([r[f"learned{k}_gap"] for r in rs]))
      d[f"learned{k}_rounds"] = float(np.mean([r[f"learned{k}_rounds"] for r in rs]))
    by_n[str(n)] = d
  return {"value": 100 * float(np.mean([r["learned10_gap"] for r in rows])),
          "knn": 100 * float(np.mean([r["knn_gap"] for r in rows])),
          "by_list_size": {str(k): 100 * float(np.mean([r[f"learned{k}_gap"] for r in rows])) for k in sizes},
          "by_n": by_n,
          "train": {"instances": args.train_instances, "edges": edges, "data_s": t_data, "train_s": t_train,
                    "ga_label_generations": args.ga_label_generations,
                    "final_loss": float(np.mean(lc.train_log[-20:]))}}


# ------------------------------------------------------------------------ Or-opt
OR_OPT_PASSES = 50
OR_OPT_SEGMENT = 3
OR_OPT_BYTES_PER_ENTRY = 12  # candidate id + d(x, c) from the k-NN tables, one gathered d(y, e)
#: Per valid entry the Or-opt kernel evaluated (1024 tours, 128-thread CTAs), from one ncu
#: capture of the same launch on the first 256 tours: warp instructions executed and L2
#: sector bytes, and DRAM bytes scaled to a 1024-tour launch (the tours' 4 KB each grows).
OR_OPT_NCU_PER_ENTRY: dict | None = {"inst": 4.032, "lts_bytes": 32.51, "dram_bytes_per_launch": 8_488_960}
OR_OPT_CPU_TOURS = 6
OR_OPT_THREADS = 128  # fastest of 128 / 256 / 512 threads per CTA here


def _or_opt_cpu_sample(coords, cand, tours_np) -> dict:
  """Oracle Or-opt (NumPy, one core) on the first tours of the workload, same passes."""
  from oracle import distances as odist
  from oracle import or_opt as oo

  D = odist.euc2d_matrix(coords)
  t0 = time.perf_counter()
  evaluated = 0
  outs = []
  for t in tours_np[:OR_OPT_CPU_TOURS]:
    out, _, _, ev = oo.refine(t, D, cand, OR_OPT_PASSES, OR_OPT_SEGMENT)
    evaluated += ev
    outs.append(out)
  dt = time.perf_counter() - t0
  return {"value": evaluated / dt, "unit": "entries/s", "cores": 1, "kind": "port", "outs": outs,
          "sample": f"{OR_OPT_CPU_TOURS} of the tours, {OR_OPT_PASSES} passes each ({dt:.1f} s)"}


def main_or_opt(args) -> int:
  """Candidate Or-opt on the 1000-city 20-cluster instance: 1024 random tours, k=20,
  segments of up to 3 cities, 50 best-improvement passes per tour; metric = valid entries
  evaluated per second."""
  import torch

  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.build import build_library
  from tsp_gpu_clean_b200.device import operands_for, ptr, stream_handle
  from tsp_gpu_clean_b200.problem import Problem, ProblemContext
  from tsp_gpu_clean_b200.strategies.or_opt import LocalSearchB200OrOpt

  world, rank, _ = _dist_env()
  n = instances.TWO_OPT_N
  coords, _ = instances.two_opt_workload(tours=1)
  tours_np = instances.random_tours(n, args.tours, instances.TWO_OPT_TOUR_SEED + 1000 * rank)
  ctx = ProblemContext(Problem.from_coordinates(coords, "clustered1000"), seed=0)
  cand_np = ctx.get_cpu_candidate_list(K_CAND)
  config = {"workload": f"Or-opt (best improvement, candidate_k={K_CAND}, segments <= {OR_OPT_SEGMENT}, "
                        f"{OR_OPT_PASSES} passes) on random tours of the 1000-city 20-cluster EUC_2D instance",
            "tours": args.tours, "n": n, "k": K_CAND, "passes": OR_OPT_PASSES,
            "threads_per_cta": OR_OPT_THREADS, "l2": "flushed between timed steps (256 MiB write)"}
  metric = "Or-opt entries evaluated/s"
  if args.impl == "reference":
    if rank != 0:
      return 0
    cpu = _or_opt_cpu_sample(coords, cand_np, tours_np)
    print(json.dumps({"metric": metric, "value": cpu["value"], "unit": "entries/s", "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)", "impl": "reference",
                      "config": config,
                      "cpu_baseline": {k: v for k, v in cpu.items() if k != "outs"},
                      "e2e": {"value": cpu["value"], "unit": "entries/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}))
    return 0
  world, rank = _init_ranks()  # this rank's GPU and, under torchrun, the NCCL group
  build_library()
  lib = native.load_library()
  from tsp_gpu_clean_b200 import roofline

  peaks = roofline.measure_peaks()  # the kernel's ceilings on this device, before the timed region
  ops = operands_for(ctx)
  dist_t, stride, _ = ops.distance_args(n)
  tabs = ops.candidates(K_CAND, cand_np, n)
  pristine = torch.from_numpy(tours_np).cuda()
  work = torch.empty_like(pristine)
  stats = torch.zeros((args.tours, 3), dtype=torch.int64, device="cuda")
  status = torch.zeros(args.tours, dtype=torch.int32, device="cuda")
  flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

  def launch():
    native.check("tspb_or_opt", lib.tspb_or_opt(ptr(work), args.tours, n, ptr(dist_t), stride, None, ptr(tabs.cand),
                                                 ptr(tabs.cand_dist), ptr(tabs.packed), tabs.k, OR_OPT_SEGMENT,
                                                 OR_OPT_PASSES, OR_OPT_THREADS,
                                                 ptr(status), ptr(stats), stream_handle()))

  for _ in range(args.warmup):
    work.copy_(pristine)
    launch()
  torch.cuda.synchronize()
  _barrier(world)
  ms, evaluated, launches = [], 0, 0
  with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
    for _ in range(args.steps):
      work.copy_(pristine)
      flush.fill_(1)
      e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
      e0.record()
      launch()
      e1.record()
      torch.cuda.synchronize()
      ms.append(e0.elapsed_time(e1))
      evaluated += int(stats[:, 2].sum().item())
      launches += 1
  if int(status.max().item()) != 0:
    raise RuntimeError(f"Or-opt kernel reported {native.status_text(int(status.max().item()))}")
  device_out = work.cpu().numpy()
  _barrier(world)
  units, secs = aggregate(evaluated, sum(ms) / 1e3, world)
  # end to end through the strategy: host tours in, host tours out
  ls = LocalSearchB200OrOpt(max_iterations=OR_OPT_PASSES, candidate_k=K_CAND, max_segment=OR_OPT_SEGMENT)
  ls.improve_batch(tours_np[:2], ctx)
  walls, e2e_eval = [], 0
  with GcWatch() as gcw:
    for _ in range(args.steps):
      torch.cuda.synchronize()
      t0 = time.perf_counter()
      out = ls.improve_batch(tours_np, ctx)
      walls.append(time.perf_counter() - t0)
      e2e_eval += int(ls.last_stats[:, 2].sum())
  assert np.array_equal(out, device_out)
  e2e_units, e2e_s = aggregate(e2e_eval, sum(walls), world)
  _finish_ranks(world)
  if rank != 0:
    return 0
  line = {"metric": metric, "value": units / secs, "unit": "entries/s", "n_gpus": world, "steps": args.steps,
          "warmup": args.warmup, "ms_per_step": sum(ms) / len(ms), "higher_is_better": True, "scaling": "weak",
          "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)", "config": config,
          "clocks": clocks.summary(),
          "e2e": {"value": e2e_units / e2e_s, "unit": "entries/s", "h2d_bytes_per_step": int(tours_np.nbytes),
                  "d2h_bytes_per_step": int(tours_np.nbytes)},
          "gpu_launches": launches,
          "detail": {"e2e_walls_s": [round(w, 4) for w in walls], "e2e_gc": gcw.summary()}}
  line["detail"]["evaluated_per_step"] = evaluated // len(ms)
  # like the 2-opt scan, the kernel works on an L2-resident matrix and shared-memory tour
  # state: its ceilings are the L2 gather rate and the INT32 issue rate, measured here
  eps = evaluated / (sum(ms) / 1e3)
  per = OR_OPT_NCU_PER_ENTRY
  if per is not None:
    int_ach, l2_ach = eps * per["inst"] * 32 / 1e12, eps * per["lts_bytes"] / 1e9
    basis = (f"ncu per valid entry: {per['inst']:.2f} warp instructions, {per['lts_bytes']:.2f} L2 sector bytes")
  else:
    int_ach, l2_ach = eps * ALG_OPS_PER_DELTA / 1e12, eps * 32 / 1e9
    basis = f"no ncu figure: one 32-byte L2 sector and {ALG_OPS_PER_DELTA} integer ops per valid entry"
  i32 = {"achieved": int_ach, "peak": peaks["int32_tops"], "unit": "TOP/s", "frac": int_ach / peaks["int32_tops"]}
  l2 = {"achieved": l2_ach, "peak": peaks["l2_sector_gbs"], "unit": "GB/s", "frac": l2_ach / peaks["l2_sector_gbs"]}
  top = i32 if i32["frac"] >= l2["frac"] else l2
  line["roofline"] = {"bound": "int32" if top is i32 else "l2", "achieved": top["achieved"], "peak": top["peak"],
                      "unit": top["unit"], "frac": top["frac"],
                      "traffic": per.get("dram_bytes_per_launch") if per is not None else None,
                      "kernel": "or_opt_kernel", "peak_source": "measured in this run: " + peaks["method"],
                      "basis": basis, "int32": i32, "l2": l2,
                      "algorithmic": {"gbs": eps * OR_OPT_BYTES_PER_ENTRY / 1e9,
                                      "basis": f"{OR_OPT_BYTES_PER_ENTRY} B per valid entry"}}
  if world == 1 and not args.no_cpu_baseline:
    cpu = _or_opt_cpu_sample(coords, cand_np, tours_np)
    for t, o in enumerate(cpu["outs"]):
      assert np.array_equal(o, device_out[t]), t
    line["cpu_baseline"] = {k: v for k, v in cpu.items() if k != "outs"}
  print(json.dumps(line))
  return 0


def main(argv=None) -> int:
  ap = argparse.ArgumentParser()
  ap.add_argument("--gpus", type=int, default=1)
  ap.add_argument("--steps", type=int, default=3)
  ap.add_argument("--warmup", type=int, default=3)
  ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
  ap.add_argument("--tours", type=int, default=instances.TWO_OPT_TOURS)
  ap.add_argument("--max-iter", type=int, default=10**9,
                  help="2-opt: passes per tour (default: to a local optimum; fewer only for short profiling runs)")
  ap.add_argument("--mode", default="both", choices=["both", "best", "first"])
  ap.add_argument("--threads", type=int, default=128)
  ap.add_argument("--kernel", default="scan", choices=["scan", "scan_unpacked", "cached"])
  ap.add_argument("--distances", default="matrix", choices=["matrix", "coords"],
                  help="two_opt: read the int32 matrix, or rebuild each distance from FP64 coordinates")
  ap.add_argument("--first-restart", default="incremental", choices=["incremental", "full"],
                  help="first mode: restart each pass from the affected entries and row bi, or rescan from entry 0")
  ap.add_argument("--batch-incremental", default="off", choices=["auto", "on", "off"],
                  help="GA/uneven: 2-opt with the reverse k-NN index (best: only the rows a move can change are "
                       "recomputed; first: incremental restart); auto lets the tuner measure both; off (the "
                       "solver's default) uses the plain kernel")
  ap.add_argument("--batch-pair", default="auto", choices=["auto", "on", "off"],
                  help="GA/uneven: best-mode 2-opt of a row by a two-CTA cluster; auto lets the tuner measure it")
  ap.add_argument("--cpu-workers", type=int, default=0, help="0: all host cores, capped at 64")
  ap.add_argument("--no-cpu-baseline", action="store_true")
  ap.add_argument("--no-ga", action="store_true", help="two_opt: leave out the ga1000 sub-result")
  ap.add_argument("--workload", default="two_opt",
                  choices=["two_opt", "learned", "uneven", "or_opt", "mlp_train", *GA_WORKLOADS])
  ap.add_argument("--mlp-edges", type=int, default=1 << 16, help="mlp_train: edges in the batch")
  ap.add_argument("--instances", type=int, default=256, help="uneven: instances in the batch")
  ap.add_argument("--generations", type=int, default=100, help="uneven: generations")
  ap.add_argument("--train-instances", type=int, default=2000)
  ap.add_argument("--eval-instances", type=int, default=4)
  ap.add_argument("--eval-starts", type=int, default=8)
  ap.add_argument("--ga-label-generations", type=int, default=8,
                  help="learned: generations of the fused GA that refine each training instance's labels")
  ap.add_argument("--ils-factor", type=float, default=6.0,
                  help="learned: equal time budget per arm, in units of the k-NN arm's first descent")
  ap.add_argument("--ils-kicks", type=int, default=128, help="learned: double-bridge kicks per round")
  ap.add_argument("--chunk", type=int, default=16, help="GA: generations replayed between host checks")
  ap.add_argument("--no-graph", action="store_true",
                  help="GA/uneven: launch every generation directly instead of replaying a captured graph "
                       "(for kernel profilers, which do not follow launches inside a stream capture)")
  ap.add_argument("--engine", default="batch", choices=["single", "batch"],
                  help="GA: the multi-instance batch engine with one instance, or the one-run graph engine")
  ap.add_argument("--cpu-gens", type=int, default=0, help="GA: generations in the CPU sample (0: workload default)")
  ap.add_argument("--clock-interval-ms", type=int, default=200, help="nvidia-smi clock sampling period")
  args = ap.parse_args(argv)
  ClockSampler.interval_ms = max(20, int(args.clock_interval_ms))
  if args.workload == "learned":
    res = run_learned_bench(args)
    print(json.dumps({"metric": "tour gap @ equal wall time, learned top-10 vs k-NN top-20", "value": res["value"],
                      "unit": "% above best found", "n_gpus": 1, "higher_is_better": False, "data": "synthetic (seeded)",
                      "dtype": "bf16 weights / fp32 accumulate; int32 tours", "knn_gap_pct": res["knn"],
                      "by_list_size": res["by_list_size"], "by_n": res["by_n"], "train": res["train"],
                      "config": {"workload": "learned candidates: train on GA tours of generated instances n in "
                                             "[200, 2000], evaluate n = 1000, 5000, 10000 with iterated 2-opt (best "
                                             "mode, double-bridge kicks) under equal CUDA-event time per arm",
                                 "train_instances": args.train_instances, "eval_instances_per_n": args.eval_instances,
                                 "starts": args.eval_starts, "ils_factor": args.ils_factor,
                                 "ils_kicks": args.ils_kicks}}))
    return 0
  if args.workload == "uneven":
    return main_uneven(args)
  if args.workload == "mlp_train":
    return main_mlp_train(args)
  if args.workload == "or_opt":
    return main_or_opt(args)
  if args.workload != "two_opt":
    return main_ga(args)
  world, rank, _ = _dist_env()
  workers = args.cpu_workers or min(os.cpu_count() or 1, 64)
  config = {"workload": "2-opt to local optimum (best and first modes, candidate_k=20) on random tours of a "
                        "1000-city 20-cluster EUC_2D instance",
            "tours": args.tours, "n": instances.TWO_OPT_N, "k": K_CAND, "modes": list(MODES if args.mode == "both" else (args.mode,)),
            "l2": "flushed between timed steps (256 MiB write); the 4 MB matrix is L2-resident within a step",
            "threads_per_cta": args.threads, "kernel": args.kernel, "distances": args.distances,
            "first_restart": args.first_restart,
            "counting": "timed launches pass no stats buffer (first mode then skips its per-row pair-count "
                        "bookkeeping); the pair count is that of one untimed counted launch of the same tours, "
                        "whose tours every timed launch reproduces (checked)"}
  sample_gens = args.cpu_gens or 6
  tours_np = two_opt_tours(args.tours, rank)
  indices = parity_indices(args.tours, max(PARITY_TOURS, workers))

  if args.impl == "reference":
    if rank != 0:
      return 0
    kind, worker = cpu_path()
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
      small = instances.clustered_instance(60, 4, 30.0, 5)
      for w in range(args.warmup):  # imports and first calls in every worker, on a 60-city tour
        pool.map(worker, [(small, instances.random_tours(60, 1, w)[0])] * workers)
      vals = [cpu_sample(pool, tours_np, indices, worker) for _ in range(args.steps)]
      one = cpu_one_core(pool, tours_np, indices[0], worker)
      ga_cpu = pool.apply(_ga_cpu_gens_per_s, (GA_SUB_WORKLOAD, sample_gens))
    value = sum(v["pairs"] for v in vals) / sum(v["wall_s"] for v in vals)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(v["wall_s"] for v in vals) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded)", "impl": "reference", "config": config,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": kind,
                             "implementation": ("LocalSearchCPUTourTwoOpt.improve_batch of the installed reference "
                                                "(baseline/_ref)" if kind == "reference" else "oracle/two_opt.py"),
                             "sample": f"{len(indices)} tours of the batch per step over {workers} processes (one tour "
                                       "per task), best then first mode to a local optimum",
                             "refined_digest": refined_digest(vals[0]["results"]) if vals else None,
                             "tours_per_s": statistics.mean(v["tours_per_s"] for v in vals),
                             "one_core": {k: one[k] for k in ("value", "tours_per_s", "seconds")}},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "detail": {GA_SUB_WORKLOAD: {"metric": "generations/s", "cpu_one_core": ga_cpu["value"],
                                         "kind": ga_cpu["kind"],
                                         "sample": f"{sample_gens} generations of {ga_cpu['what']} on one core, "
                                                   f"{ga_cpu['loop_s']:.1f} s (init excluded)"}}}
    print(json.dumps(line))
    return 0

  pool = None
  kind, worker = cpu_path()
  if rank == 0 and world == 1 and not args.no_cpu_baseline:
    pool = mp.get_context("spawn").Pool(workers)  # before the first CUDA call
  from tsp_gpu_clean_b200.build import build_library

  world, rank = _init_ranks()
  build_library()
  res = run_gpu(args, world, rank)
  ga = None
  if not args.no_ga:
    ga = ga_measure(GA_SUB_WORKLOAD, max(args.warmup, 1), max(args.steps, 3), world, rank)
  _finish_ranks(world)
  cpu = one = ga_cpu = parity = ga_parity = None
  if pool is not None:
    cpu = cpu_sample(pool, res["tours_np"], indices, worker)
    parity = check_parity(res["counted"], cpu, kind)
    one = cpu_one_core(pool, res["tours_np"], indices[0], worker)
    if ga is not None:
      ga_cpu = pool.apply(_ga_cpu_gens_per_s, (GA_SUB_WORKLOAD, sample_gens))
    pool.close()
    pool.join()
  if rank != 0:
    return 0
  line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
          "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
          "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)", "config": config,
          "clocks": res["clocks"], "e2e": res["e2e"], "gpu_launches": res["gpu_launches"],
          "roofline": res["roofline"],
          "detail": {"kernel_ms_per_step": res["kernel_ms_per_step"], "pairs_per_step": res["pairs_per_step"],
                     "evaluated_per_step": res["evaluated_per_step"], "passes_per_step": res["passes_per_step"],
                     "moves_per_step": res["moves_per_step"], "tours_per_s": res["tours_per_s"],
                     "peaks": res["peaks"]}}
  line["detail"]["refined_digest"] = {
    "indices": list(indices),
    "sha256": refined_digest([{m: (res["counted"][m][0][i],) for m in res["counted"]} for i in indices],
                             [m for m in MODES if m in res["counted"]])}
  if parity is not None:
    line["parity"] = parity["text"]
    if parity["mismatches"]:
      line["detail"]["parity_mismatches"] = parity["mismatches"]
  if cpu is not None:
    line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": workers, "kind": kind,
                            "implementation": ("LocalSearchCPUTourTwoOpt.improve_batch of the installed reference "
                                               "(baseline/_ref)" if kind == "reference" else "oracle/two_opt.py"),
                            "sample": f"{cpu['tours']} tours of the timed batch (indices spread over it, one per "
                                      f"process), best then first mode to a local optimum, {cpu['wall_s']:.1f} s wall",
                            "tours_per_s": cpu["tours_per_s"],
                            "one_core": {"value": one["value"], "tours_per_s": one["tours_per_s"],
                                         "seconds": one["seconds"], "tour": one["tour"]}}
  if ga is not None:
    sub = {"workload": ga["desc"], "metric": "generations/s", "value": ga["value"], "e2e": ga["e2e"]["value"],
           "ms_per_run": ga["ms_per_step"], "walls_s": ga["walls_s"], "clocks": ga["clocks"],
           "gpu_launches": ga["gpu_launches"]}
    if ga_cpu is not None:
      sub["cpu_one_core"] = ga_cpu["value"]
      sub["cpu_kind"] = ga_cpu["kind"]
      sub["cpu_sample"] = f"{sample_gens} generations of {ga_cpu['what']} on one core, {ga_cpu['loop_s']:.1f} s"
      sub["vs_cpu_one_core"] = {"device": ga["value"] / ga_cpu["value"], "e2e": ga["e2e"]["value"] / ga_cpu["value"]}
      # the first generations of the same seeded run on the device, against the oracle's
      short = ga_measure(GA_SUB_WORKLOAD, 0, 1, 1, 0, generations=sample_gens) if world == 1 else None
      if short is not None:
        ok = [float(v) for v in short["history"]] == ga_cpu["history"]
        sub["parity"] = (f"best-fitness history of the first {sample_gens} generations equal to that of "
                         f"{ga_cpu['what']}" if ok else f"MISMATCH of the best-fitness history against {ga_cpu['what']}")
        if not ok:
          parity = {"ok": False}
    line["detail"][GA_SUB_WORKLOAD] = sub
  print(json.dumps(line))
  if parity is not None and not parity["ok"]:
    return 1
  return 0


def main_ga(args) -> int:
  world, rank, _ = _dist_env()
  n, P, G, elite, post_init, seed, desc = GA_WORKLOADS[args.workload]
  sample = args.cpu_gens or {"ga100": 50, "ga1000": 6, "ga2000": 4, "chapter4": 3, "chapter4x30": 3}[args.workload]
  o = ga_options(args.workload)
  config = {"workload": desc, "n": n, "population": P, "generations": G, "elite": elite,
            "operators": {k: v for k, v in o.items() if k != "reps"}, "runs": o["reps"],
            "l2": "working set (matrix + population) below L2 for n <= 2000; not flushed between generations"}
  if args.workload.startswith("chapter4"):
    config["published_context"] = ("the reference publishes 35.0 generations/s for this configuration on pr1002 "
                                   "(FullGPUModular, GTX 1050 Mobile); the instance here is a seeded synthetic "
                                   "stand-in of the same size, patience disabled")
  if args.impl == "reference":
    if rank != 0:
      return 0
    vals = [_ga_cpu_sample(args.workload, sample) for _ in range(max(1, args.steps))]
    value = sum(v["value"] * v["loop_s"] for v in vals) / sum(v["loop_s"] for v in vals)
    line = {"metric": "generations/s", "value": value, "unit": "generations/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value * G, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)", "impl": "reference",
            "config": config,
            "cpu_baseline": {"value": value, "unit": "generations/s", "cores": vals[0]["cores"],
                             "kind": vals[0]["kind"], "sample": f"per step: {vals[0]['sample']}"},
            "e2e": {"value": value, "unit": "generations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0
  res = run_ga_bench(args)
  if res["rank"] != 0:
    return 0
  line = {"metric": "generations/s", "value": res["value"], "unit": "generations/s", "n_gpus": res["world"],
          "steps": args.steps,
          "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
          "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)", "config": config, "clocks": res["clocks"],
          "e2e": res["e2e"], "gpu_launches": res["gpu_launches"],
          "detail": {"best_fitness": res["best"], "engine": args.engine, "last_run": res["timing"],
                     "loop_ms_steps": res["loop_ms_steps"], "walls_s": res["walls_s"],
                     "phase_ms_steps": res["phase_ms_steps"], "gc": res["gc"], "buckets": res["buckets"],
                     "two_opt_totals": res["two_opt_totals"]}}
  if res["world"] > 1:
    config["parallelism"] = f"{res['world']} independent replicas (one GA run per GPU, generator seeded per rank)"
  if not args.no_cpu_baseline and res["world"] == 1:
    cpu = _ga_cpu_sample(args.workload, sample)
    line["cpu_baseline"] = {"value": cpu["value"], "unit": "generations/s", "cores": cpu["cores"], "kind": cpu["kind"],
                            "sample": cpu["sample"]}
  print(json.dumps(line))
  return 0


if __name__ == "__main__":
  sys.exit(main())
