"""ctypes binding of libtspb.so (the C ABI declared in include/tspb.h).

The library is loaded from this package directory (built in-tree by
`tsp_gpu_clean_b200.build`). There is no CPU fallback: when the library is
missing or no CUDA device is present, callers get `GPUUnavailableError`.
"""

from __future__ import annotations

import ctypes
import os
import threading

from .errors import GPUUnavailableError, KernelError, NotPermutationError, VRAMInsufficientError

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libtspb.so")

TSPB_OK = 0
TSPB_ERR_ARG = 1
TSPB_ERR_CUDA = 2
TSPB_ERR_NOT_PERMUTATION = 3
TSPB_ERR_RANGE = 4
TSPB_ERR_UNSUPPORTED = 5
TSPB_ERR_WORKSPACE = 6
TSPB_ERR_BUDGET = 7
TSPB_ERR_DEVICE_MEMORY = 8

MODE_CODES = {"best": 0, "batch": 0, "first": 1, "multi_move": 2}
#: OR-ed into a 2-opt mode code: the distances are symmetric (include/tspb.h)
TSPB_MODE_SYMMETRIC = 0x100

_p = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_sz = ctypes.c_size_t
_f64 = ctypes.c_double

#: name -> (restype, argtypes); one entry per declaration in include/tspb.h.
SIGNATURES: dict[str, tuple] = {
  "tspb_version": (ctypes.c_int, []),
  "tspb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
  "tspb_set_watchdog_cycles": (_i64, [_i64]),
  "tspb_three_opt_grid": (ctypes.c_int, [_p, _i32, _i32, _p, _i64, _p, _p, _p, _i32, _i32, _i32, _i32, _i64, _p, _p, _p]),
  "tspb_three_opt_grid_threads": (ctypes.c_int, [_i32, _i32]),
  "tspb_microbench_l2_gather": (ctypes.c_int, [_p, _i64, _i32, _i32, _p, _p]),
  "tspb_microbench_int32": (ctypes.c_int, [_i32, _i32, _i32, _p, _p]),
  "tspb_graph_capture_begin": (ctypes.c_int, [_p]),
  "tspb_graph_capture_end": (ctypes.c_int, [_p, ctypes.POINTER(ctypes.c_void_p)]),
  "tspb_graph_launch": (ctypes.c_int, [_p, _p]),
  "tspb_graph_destroy": (ctypes.c_int, [_p]),
  "tspb_two_opt_workspace_bytes": (_sz, [_i32, _i32, _i32, _i32, _i32]),
  "tspb_two_opt": (ctypes.c_int, [_p, _i32, _i32, _p, _i64, _p, _p, _p, _p, _p, _p, _i32, _i32, _i64, _i32, _p, _p, _p, _sz, _p]),
  "tspb_two_opt_gated": (ctypes.c_int, [_p, _p, _i32, _i32, _p, _i64, _p, _p, _p, _p, _p, _p, _i32, _i32, _i64, _i32, _p,
                                         _p, _p, _sz, _p]),
  "tspb_candidate_pack": (ctypes.c_int, [_p, _p, _i32, _i32, _p, _p, _p]),
  "tspb_two_opt_multi_move_static": (ctypes.c_int, [_p, _i32, _i32, _p, _i64, _p, _p, _p, _i32, _i64, _i32, _p, _p, _p]),
  "tspb_candidate_reverse_index": (ctypes.c_int, [_p, _i32, _i32, _p, _p, _p, _p]),
  "tspb_candidate_distances": (ctypes.c_int, [_p, _i32, _i32, _p, _i64, _p, _p, _p]),
  "tspb_tour_cost": (ctypes.c_int, [_p, _i32, _i32, _p, _i64, _p, _i32, _p, _p]),
  "tspb_tournament": (ctypes.c_int, [_p, _i32, _p, _i32, _i32, _p, _p]),
  "tspb_gather_rows": (ctypes.c_int, [_p, _i32, _i32, _p, _i32, _p, _p]),
  "tspb_pmx": (ctypes.c_int, [_p, _i32, _i32, _p, _p, _p, _p, _p]),
  "tspb_scatter_rows": (ctypes.c_int, [_p, _i32, _i32, _p, _p, _i32, _p]),
  "tspb_inversion": (ctypes.c_int, [_p, _i32, _i32, _p, _f64, _p, _p, _p]),
  "tspb_ox": (ctypes.c_int, [_p, _i32, _i32, _p, _p, _p, _p, _p]),
  "tspb_swap": (ctypes.c_int, [_p, _i32, _i32, _p, _f64, _p, _p, _p]),
  "tspb_stable_rank": (ctypes.c_int, [_p, _i32, _i32, _p, _p]),
  "tspb_validate_perm": (ctypes.c_int, [_p, _i32, _i32, _p, _p]),
  "tspb_euc2d_matrix": (ctypes.c_int, [_p, _i32, _p, _i64, _p]),
  "tspb_generation_offspring": (ctypes.c_int, [_p, _p, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p, _f64, _p, _i64, _p, _p,
                                                _p, _p, _p, _p]),
  "tspb_generation_survival": (ctypes.c_int, [_p, _p, _p, _p, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p, _p]),
  "tspb_generation_elite_cost": (ctypes.c_int, [_p, _i32, _i32, _p, _i64, _p, _p, _p, _p]),
  "tspb_generation_track": (ctypes.c_int, [_p, _p, _i32, _i32, _p, _p, _p, _i64, _p, _p, _p, _p, _p]),
  "tspb_knn": (ctypes.c_int, [_p, _i64, _p, _i32, _i32, _p, _p]),
  "tspb_knn_ties": (ctypes.c_int, [_p, _i64, _p, _i32, _i32, _p, _p, _p]),
  "tspb_mlp_param_count": (ctypes.c_int, []),
  "tspb_edge_features": (ctypes.c_int, [_p, _i32, _p, _i32, _p, _i64, _p, _p, _p, _p]),
  "tspb_mlp_infer": (ctypes.c_int, [_p, _p, _i64, _p, _p]),
  "tspb_mlp_train_grad": (ctypes.c_int, [_p, _p, _p, _i64, _p, _p, _p]),
  "tspb_mlp_train_grad_tc": (ctypes.c_int, [_p, _p, _p, _i64, _p, _p, _p, _p]),
  "tspb_mlp_adam": (ctypes.c_int, [_p, _p, _p, _p, _i32, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                   ctypes.c_float, _p]),
  "tspb_select_topk": (ctypes.c_int, [_p, _p, _i32, _i32, _i32, _p, _p]),
  "tspb_nn_init": (ctypes.c_int, [_p, _i32, _p, _i32, _i32, _p, _i32, _i32, _p, _sz, _p, _p]),
  "tspb_nn_init_jobs": (ctypes.c_int, [_p, _i32, _i32, _p, _p, _p]),
  "tspb_nn_init_jobs_smem": (ctypes.c_int, [_p, _i32, _i32, _i32, _i32, _p]),
  "tspb_random_init": (ctypes.c_int, [_p, _i32, _i32, _p, _p, _p]),
  "tspb_distance_matrix": (ctypes.c_int, [_p, _i32, _i32, _i32, _p, _i64, _p]),
  "tspb_three_opt": (ctypes.c_int, [_p, _i32, _i32, _p, _i64, _p, _i64, _i32, _p, _sz, _p, _p, _p]),
  "tspb_three_opt_workspace_bytes": (ctypes.c_int, [_i32, _i32, ctypes.POINTER(ctypes.c_size_t)]),
  "tspb_or_opt": (ctypes.c_int, [_p, _i32, _i32, _p, _i64, _p, _p, _p, _p, _i32, _i32, _i64, _i32, _p, _p, _p]),
  "tspb_or_opt_max_n": (ctypes.c_int, []),
  "tspb_random_init_jobs": (ctypes.c_int, [_p, _i32, _i32, _i32, _p]),
  "tspb_tape_draw_host": (ctypes.c_int, [_p, _i32, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p, _p]),
  "tspb_tape_draw": (ctypes.c_int, [_p, _p, _i32, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p, _p, _p]),
  "tspb_batch_init": (ctypes.c_int, [_p, _i32, _i32, _p]),
  "tspb_batch_offspring": (ctypes.c_int, [_p, _p, _i32, _i32, _i32, _p]),
  "tspb_batch_survival": (ctypes.c_int, [_p, _p]),
  "tspb_batch_two_opt": (ctypes.c_int, [_p, _p, _i32, _i32, _i32, _i32, _i32, _i64, _i32, _i32, _p, _p]),
  "tspb_batch_two_opt_occupancy": (ctypes.c_int, [_i32, _i32, _i32, _i32]),
  "tspb_batch_track": (ctypes.c_int, [_p, _i32, _p]),
}

TSPB_BATCH_RUN = 0
TSPB_BATCH_STOPPED = 1
TSPB_BATCH_PAUSED = 2
TSPB_BATCH_RESUME = 3
TSPB_BATCH_DONE = 4
TSPB_BATCH_HIT_OPTIMAL = 5
TSPB_BATCH_NEAR_OPTIMAL = 6
TSPB_BATCH_PHASE_POSTINIT = 0
TSPB_BATCH_PHASE_RESUME = 1
TSPB_BATCH_PHASE_RUN = 2
TSPB_BATCH_PHASE_OFFSPRING = 3
# Coordinate-based TSPLIB edge types of tspb_distance_matrix.
EDGE_TYPE_CODES = {"EUC_2D": 0, "EUC_3D": 1, "MAN_2D": 2, "MAN_3D": 3, "MAX_2D": 4, "MAX_3D": 5, "CEIL_2D": 6,
                   "ATT": 7, "GEO": 8, "XRAY1": 9}
TSPB_XOVER_PMX = 0
TSPB_XOVER_OX = 1
TSPB_MUT_INVERSION = 0
TSPB_MUT_SWAP = 1
TSPB_BATCH_COORDS = 1
TSPB_BATCH_GROUPED = 2
TSPB_BATCH_INCREMENTAL = 4
TSPB_BATCH_PAIR = 8


class Pcg64(ctypes.Structure):
  """`tspb_pcg64` of include/tspb.h: a NumPy PCG64 bit_generator.state."""

  _fields_ = [("state_hi", ctypes.c_uint64), ("state_lo", ctypes.c_uint64), ("inc_hi", ctypes.c_uint64),
              ("inc_lo", ctypes.c_uint64), ("has_uint32", _i32), ("uinteger", ctypes.c_uint32)]

  _M = (1 << 64) - 1

  @classmethod
  def from_state(cls, state: dict) -> "Pcg64 | None":
    if state.get("bit_generator") != "PCG64":
      return None
    s, inc = int(state["state"]["state"]), int(state["state"]["inc"])
    return cls(s >> 64, s & cls._M, inc >> 64, inc & cls._M, int(state["has_uint32"]), int(state["uinteger"]))

  def to_state(self) -> dict:
    return {"bit_generator": "PCG64",
            "state": {"state": (int(self.state_hi) << 64) | int(self.state_lo),
                      "inc": (int(self.inc_hi) << 64) | int(self.inc_lo)},
            "has_uint32": int(self.has_uint32), "uinteger": int(self.uinteger)}


class NNJob(ctypes.Structure):
  """`tspb_nn_job` of include/tspb.h."""

  _fields_ = [("n", _i32), ("k", _i32), ("cand", _p), ("seeds", _p), ("out", _p), ("rows", _i32), ("pad", _i32)]


class BatchInstance(ctypes.Structure):
  """`tspb_batch_instance` of include/tspb.h."""

  _fields_ = [("n", _i32), ("k", _i32), ("pop_offset", _i64), ("node_offset", _i64), ("dist", _p),
              ("dist_stride", _i64), ("coords", _p), ("cand_packed", _p), ("patience", _i64), ("optimal", _f64),
              ("rev_off", _p), ("rev_idx", _p)]


class BatchState(ctypes.Structure):
  """`tspb_batch` of include/tspb.h (device pointers of one batch of GA runs)."""

  _fields_ = [("num_instances", _i32), ("P", _i32), ("kt", _i32), ("elite", _i32), ("G", _i32), ("rows_max", _i32),
              ("mutation_rate", _f64), ("inst", _p), ("pop", _p * 2), ("fit", _p * 2), ("off", _p), ("off_fit", _p),
              ("order", _p), ("tape_tourn", _p), ("tape_cut_a", _p), ("tape_cut_b", _p), ("tape_u", _p),
              ("tape_inv_a", _p), ("tape_inv_b", _p), ("ctl", _p), ("best_cost", _p), ("best_tour", _p),
              ("history", _p), ("ties", _p), ("host_elites", _p), ("ls_status", _p), ("ls_stats", _p),
              ("clean", _p * 2), ("off_clean", _p), ("crossover", _i32), ("mutation", _i32)]

_lock = threading.Lock()
_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
  """Load libtspb.so and bind every signature (no GPU needed to load)."""
  global _lib
  with _lock:
    if _lib is not None:
      return _lib
    if not os.path.exists(path):
      raise GPUUnavailableError(f"libtspb.so is not built at {path}; run `python -m tsp_gpu_clean_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
      fn = getattr(lib, name)
      fn.restype = res
      fn.argtypes = args
    _lib = lib
    return lib


def status_text(code: int) -> str:
  return load_library().tspb_status_string(int(code)).decode()


def check(func: str, code: int) -> None:
  """Raise for a non-zero host-side status of a libtspb call."""
  if code == TSPB_OK:
    return
  if code == TSPB_ERR_NOT_PERMUTATION:
    raise NotPermutationError(f"{func}: {status_text(code)}")
  if code == TSPB_ERR_ARG:
    raise ValueError(f"{func}: {status_text(code)}")
  if code == TSPB_ERR_DEVICE_MEMORY:
    raise VRAMInsufficientError(f"{func}: {status_text(code)}")
  raise KernelError(func, code, status_text(code))


def call(name: str, *args) -> None:
  lib = load_library()
  check(name, getattr(lib, name)(*args))
