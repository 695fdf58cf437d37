"""Build recipe for libtspb.so (sm_100a), compiled in-tree next to this file.

`python -m tsp_gpu_clean_b200.build` or `build_library()` runs nvcc on every
`csrc/*.cu` with `-gencode arch=compute_100a,code=sm_100a -lineinfo -O3` and links
one shared library. The build is skipped when the library is newer than every
source and header.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libtspb.so")
OBJ = os.path.join(PKG, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
#: extra nvcc arguments (for example -D tuning constants of the kernels), space-separated
EXTRA = os.environ.get("TSPB_NVCC_EXTRA", "").split()


def _nvcc() -> str:
  for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
    if cand and os.path.exists(cand):
      return cand
  raise RuntimeError("nvcc not found; set NVCC or put the CUDA toolkit on PATH")


def sources() -> list[str]:
  return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
  if not os.path.exists(LIB):
    return True
  t = os.path.getmtime(LIB)
  deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
  return any(os.path.getmtime(p) > t for p in deps)


def build_library(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
  """Compile every CUDA source and link `libtspb.so`; returns its path."""
  if not force and not _stale():
    return LIB
  nvcc = _nvcc()
  os.makedirs(OBJ, exist_ok=True)
  objs = []
  procs = []
  for src in sources():
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    objs.append(obj)
    cmd = [nvcc, *ARCH, *FLAGS, *EXTRA, "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
    if verbose:
      cmd.insert(1, "-Xptxas=-v")
      print(" ".join(cmd))
    procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
  failed = []
  for src, p in procs:
    out, _ = p.communicate()
    if verbose or p.returncode != 0:
      sys.stdout.write(out)
    if p.returncode != 0:
      failed.append(src)
  if failed:
    raise RuntimeError(f"nvcc failed for {failed}")
  tmp = LIB + ".tmp"
  link = [nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
  r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
  if r.returncode != 0:
    sys.stdout.write(r.stdout)
    raise RuntimeError("nvcc link failed")
  os.replace(tmp, LIB)
  return LIB


if __name__ == "__main__":
  print(build_library(force="--force" in sys.argv, verbose="-v" in sys.argv))
