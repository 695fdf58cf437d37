"""Measured ceilings of the L2-resident 2-opt scan (L2 gather rate, INT32 issue rate).

The candidate 2-opt reads its distance matrix from L2 (4 MB at n = 1000) and its tour
state from shared memory; HBM sees a few MB per launch. Its two ceilings are the rate at
which L2 serves random 4-byte gathers and the rate at which the SMs issue integer
instructions. `measure_peaks()` times the library's two microbenchmark kernels
(`tspb_microbench_l2_gather`, `tspb_microbench_int32`) with CUDA events and returns both
rates; `python -m tsp_gpu_clean_b200.roofline` writes them to `roofline_peaks.json` beside
this file (the figures of the last measured B200).
"""

from __future__ import annotations

import json
import os

PEAKS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "roofline_peaks.json")

L2_TABLE_ENTRIES = 1 << 20  # 4 MiB of int32, the size of the 1000-city matrix
L2_ITERS = 2048
INT32_ITERS = 1024
THREADS = 256
SECTOR_BYTES = 32


def _best_ms(launch, repeats: int) -> float:
  import torch

  launch()  # warm-up (module load, clocks up)
  torch.cuda.synchronize()
  best = float("inf")
  for _ in range(repeats):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    launch()
    e1.record()
    e1.synchronize()
    best = min(best, e0.elapsed_time(e1))
  return best


def measure_peaks(repeats: int = 5) -> dict:
  """Both ceilings of the current device, from the fastest of `repeats` timed launches."""
  import torch

  from . import native
  from .device import ptr, stream_handle

  lib = native.load_library()
  props = torch.cuda.get_device_properties(torch.cuda.current_device())
  sms = int(props.multi_processor_count)
  blocks = sms * 8  # 2048 threads per SM
  table = torch.randint(0, 1 << 20, (L2_TABLE_ENTRIES,), dtype=torch.int32, device="cuda")
  sink = torch.zeros(1, dtype=torch.int32, device="cuda")

  def l2():
    native.check("tspb_microbench_l2_gather", lib.tspb_microbench_l2_gather(
      ptr(table), L2_TABLE_ENTRIES, L2_ITERS, blocks, ptr(sink), stream_handle()))

  def alu():
    native.check("tspb_microbench_int32", lib.tspb_microbench_int32(INT32_ITERS, blocks, 7, ptr(sink), stream_handle()))

  l2_ms = _best_ms(l2, repeats)
  alu_ms = _best_ms(alu, repeats)
  gathers = blocks * THREADS * L2_ITERS * 8
  ops = blocks * THREADS * INT32_ITERS * 128
  g_per_s = gathers / (l2_ms / 1e3)
  ops_per_s = ops / (alu_ms / 1e3)
  return {
    "device": props.name,
    "sms": sms,
    "l2_gathers_per_s": g_per_s,
    "l2_sector_gbs": g_per_s * SECTOR_BYTES / 1e9,  # lts__t_bytes units: one 32-byte sector per gather
    "l2_useful_gbs": g_per_s * 4 / 1e9,
    "int32_tops": ops_per_s / 1e12,  # lane operations
    "int32_warp_inst_per_s": ops_per_s / 32,
    "l2_ms": l2_ms,
    "int32_ms": alu_ms,
    "l2_table_bytes": L2_TABLE_ENTRIES * 4,
    "method": "random 4-byte ld.global.cg gathers from a 4 MiB table (8 chains per thread, 2048 threads per SM); "
              "add.s32/xor.b32 chains in PTX (8 per thread, 2048 threads per SM); best of "
              f"{repeats} CUDA-event-timed launches",
  }


def stored_peaks() -> dict | None:
  if os.path.exists(PEAKS_PATH):
    with open(PEAKS_PATH) as fh:
      return json.load(fh)
  return None


if __name__ == "__main__":
  import torch

  from .build import build_library

  build_library()
  torch.cuda.init()
  res = measure_peaks()
  with open(PEAKS_PATH, "w") as fh:
    json.dump(res, fh, indent=1)
  print(json.dumps(res))
