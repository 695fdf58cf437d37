"""Build recipe for oracle/_ref/: the reference's own 3-opt CUDA kernels, compiled from
its sources where they lie, with this directory's launcher (`ref_three_opt_launch.cu`).

TEST INFRASTRUCTURE ONLY. Run where the reference checkout is present:

    python oracle/build_ref.py /path/to/tsp_gpu_clean

The output, `oracle/_ref/libref3opt.so` (sm_100a), is kept out of the repository's
history and travels with the working tree to a GPU machine, where
`tests/golden/make_three_opt_kernel_golden.py` runs it to record golden outputs. The
reference's kernels compile from three files: `three_opt_batch.cu`,
`three_opt_multi_move.cu`, `three_opt_common.cuh` (its 3-opt experiment's `kernels/`)
and `pairwise_device.cuh` (`src/distances/kernels/`).
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
KERNELS = "benchmark_scripts/experiments-and-examples/experiment-comparing-3opt-and-2opt/kernels"
DIST_KERNELS = "src/distances/kernels"


def build(reference_root: str) -> str:
  kdir = os.path.join(reference_root, KERNELS)
  ddir = os.path.join(reference_root, DIST_KERNELS)
  for need in (os.path.join(kdir, "three_opt_batch.cu"), os.path.join(kdir, "three_opt_multi_move.cu"),
               os.path.join(ddir, "pairwise_device.cuh")):
    if not os.path.exists(need):
      raise FileNotFoundError(need)
  os.makedirs(OUT, exist_ok=True)
  lib = os.path.join(OUT, "libref3opt.so")
  cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-shared", "-Xcompiler", "-fPIC",
         "-I", kdir, "-I", ddir, os.path.join(HERE, "ref_three_opt_launch.cu"), "-o", lib]
  subprocess.run(cmd, check=True)
  return lib


if __name__ == "__main__":
  if len(sys.argv) < 2:
    sys.exit("usage: build_ref.py <reference checkout root>")
  print(build(sys.argv[1]))
