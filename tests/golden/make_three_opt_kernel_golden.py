"""Record outputs of the reference's 3-opt CUDA kernels (candidate scan, multi_move).

Runs on a machine with a CUDA GPU, after `python oracle/build_ref.py <reference root>`
has compiled the reference's kernels into `oracle/_ref/libref3opt.so`:

    python tests/golden/make_three_opt_kernel_golden.py [out.npz]

Writes `three_opt_kernel.npz` (next to this script by default): for every case the
distance matrix's coordinates, the k-NN table, the input tours and the tours after
`iters` launches of the reference's `three_opt_batch_kernel` or
`three_opt_multi_move_batch_kernel`, launched as `LocalSearchGPUThreeOpt._improve_grid`
launches them. Inputs are seeded synthetic instances; nothing of the reference is copied.
"""

from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import distances as odist  # noqa: E402
from oracle.three_opt_kernel import virtual_threads  # noqa: E402
from tsp_gpu_clean_b200 import instances  # noqa: E402

# (tag, n, instance, k (0: exhaustive), inner_k (0: k), threads_per_block, mode, iters, tours, start)
CASES = [
  ("cb12", 12, "uniform", 5, 0, 256, "batch", 20, 6, "random"),
  ("cb50", 50, "uniform", 8, 0, 256, "batch", 60, 6, "random"),
  ("cb50i", 50, "clustered", 8, 3, 256, "batch", 60, 6, "random"),
  ("cb120", 120, "clustered", 20, 0, 256, "batch", 3, 4, "random"),
  ("cb120t32", 120, "uniform", 10, 0, 32, "batch", 40, 4, "nn"),
  ("cb200t128", 200, "uniform", 10, 4, 128, "batch", 30, 3, "nn"),
  ("cblat", 64, "lattice", 8, 0, 256, "batch", 40, 6, "random"),
  ("cm50", 50, "uniform", 8, 0, 256, "multi_move", 20, 6, "random"),
  ("cm120", 120, "clustered", 10, 0, 64, "multi_move", 3, 4, "random"),
  ("cm200", 200, "uniform", 10, 5, 256, "multi_move", 20, 3, "nn"),
  ("cmlat", 64, "lattice", 8, 0, 16, "multi_move", 30, 6, "random"),
  ("em12", 12, "uniform", 0, 0, 256, "multi_move", 10, 6, "random"),
  ("em40", 40, "clustered", 0, 0, 256, "multi_move", 10, 4, "random"),
  ("em40t8", 40, "uniform", 0, 0, 8, "multi_move", 10, 4, "random"),
  ("emlat", 36, "lattice", 0, 0, 32, "multi_move", 10, 4, "random"),
]


def instance(kind: str, n: int, seed: int) -> np.ndarray:
  if kind == "uniform":
    return instances.uniform_instance(n, seed)
  if kind == "clustered":
    return instances.clustered_instance(n, max(2, n // 20), 30.0, seed)
  side = int(np.ceil(np.sqrt(n)))
  return np.array([[10.0 * x, 10.0 * y] for x in range(side) for y in range(side)][:n])


def nn_tours(D: np.ndarray, count: int, seed: int) -> np.ndarray:
  """Greedy nearest-neighbour tours from seeded start cities, rotated to start at 0."""
  rng = np.random.default_rng(seed)
  n = len(D)
  out = []
  for _ in range(count):
    s = int(rng.integers(0, n))
    seen = np.zeros(n, bool)
    t = [s]
    seen[s] = True
    for _ in range(n - 1):
      d = np.where(seen, np.iinfo(np.int64).max, D[t[-1]].astype(np.int64))
      nxt = int(np.argmin(d))
      t.append(nxt)
      seen[nxt] = True
    t = np.array(t)
    out.append(np.roll(t, -int(np.where(t == 0)[0][0])))
  return np.stack(out).astype(np.int32)


def main(out_path: str) -> None:
  import torch

  lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libref3opt.so"))
  lib.ref3_passes.restype = ctypes.c_int
  lib.ref3_passes.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
  res: dict[str, np.ndarray] = {}
  for c, (tag, n, kind, k, inner, tpb, mode, iters, count, start) in enumerate(CASES):
    coords = instance(kind, n, 500 + c)
    D = odist.euc2d_matrix(coords).astype(np.int32)
    cand = odist.candidate_list(k, coords=coords).astype(np.int32) if k > 0 else np.zeros((n, 0), np.int32)
    tours = instances.random_tours(n, count, 600 + c) if start == "random" else nn_tours(D, count, 600 + c)
    B = virtual_threads(tpb, n)
    d_pop = torch.from_numpy(tours.copy()).cuda()
    d_D = torch.from_numpy(D).cuda()
    d_c = torch.from_numpy(np.ascontiguousarray(cand)).cuda() if k > 0 else None
    d_pos = torch.empty((count, n), dtype=torch.int32, device="cuda")
    inner_eff = min(k, inner) if inner > 0 else k
    rc = lib.ref3_passes(1 if mode == "multi_move" else 0, d_pop.data_ptr(), d_D.data_ptr(), n, count, B,
                         d_c.data_ptr() if d_c is not None else None, k, inner_eff, d_pos.data_ptr(), iters)
    if rc != 0:
      raise RuntimeError(f"{tag}: launcher returned {rc}")
    res[f"{tag}_coords"] = coords
    res[f"{tag}_cand"] = cand
    res[f"{tag}_in"] = tours
    res[f"{tag}_out"] = d_pop.cpu().numpy()
    res[f"{tag}_meta"] = np.array([n, k, inner, tpb, 1 if mode == "multi_move" else 0, iters, B])
    print(f"{tag}: n={n} k={k} inner={inner} B={B} {mode} x{iters}")
  res["tags"] = np.array([c[0] for c in CASES])
  np.savez_compressed(out_path, **res)
  print(out_path)


if __name__ == "__main__":
  main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "three_opt_kernel.npz"))
