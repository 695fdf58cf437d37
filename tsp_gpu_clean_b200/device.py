"""Device plumbing: the GPU probe, streams, pointers and the per-context operand cache.

PyTorch is used only for device memory, streams and host<->device copies; every
computation on the path runs in libtspb.so kernels.
"""

from __future__ import annotations

import contextlib
import ctypes
import threading
import weakref
from typing import Any

import numpy as np

from .errors import GPUUnavailableError, VRAMInsufficientError
from .native import load_library

try:  # torch is the allocator and stream provider; absent torch means no GPU path
  import torch
except Exception:  # pragma: no cover - exercised only without torch
  torch = None  # type: ignore[assignment]


def require_gpu():
  """Return the torch module after checking the CUDA device and libtspb.so.

  Mirrors `require_gpu` of the reference (`src/protocols/backend.py:235-244`): a
  machine without a usable device raises instead of degrading to a CPU path.
  """
  load_library()
  if torch is None or not torch.cuda.is_available():
    raise GPUUnavailableError("no CUDA device is available; the B200 strategies do not fall back to the CPU")
  return torch


def is_device_array(x: Any) -> bool:
  return torch is not None and isinstance(x, torch.Tensor) and x.is_cuda


_RAW_STREAM = getattr(torch._C, "_cuda_getCurrentRawStream", None) if torch is not None else None
_CUR_DEVICE = getattr(torch._C, "_cuda_getDevice", None) if torch is not None else None


def stream_handle(stream=None) -> ctypes.c_void_p:
  """The cudaStream_t of `stream`, else of the current stream. The current stream's handle
  is read from torch's raw accessor when it has one: `torch.cuda.current_stream()` builds a
  Stream object and resolves the device each call, which cost a few microseconds in every
  replay of the GA engines' graphs."""
  if stream is not None:
    return ctypes.c_void_p(stream.cuda_stream)
  if _RAW_STREAM is not None and _CUR_DEVICE is not None and torch.cuda.is_initialized():
    return ctypes.c_void_p(_RAW_STREAM(_CUR_DEVICE()))
  return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t) -> ctypes.c_void_p | None:
  if t is None:
    return None
  return ctypes.c_void_p(t.data_ptr())


#: Arrays up to this size are staged through pinned memory (see device_tensor).
_PINNED_COPY_MAX = 64 << 20


def device_tensor(a: np.ndarray, dtype) -> "torch.Tensor":
  """H2D copy of a host array to the current device, stream-ordered.

  The array is first copied into pinned memory (torch's caching host allocator keeps that
  block until the copy has run), so the call does not wait for the device; a blocking copy
  from pageable memory would synchronise the stream every time."""
  t = torch.from_numpy(np.ascontiguousarray(a))
  if t.dtype != dtype:
    t = t.to(dtype)
  if t.numel() == 0:
    return torch.empty(t.shape, dtype=dtype, device="cuda")
  if t.numel() * t.element_size() > _PINNED_COPY_MAX:
    return t.to(device="cuda")  # large one-off arrays: not worth a cached pinned block
  return t.pin_memory().to(device="cuda", non_blocking=True)


_SM_COUNT: int | None = None


def auto_threads(num_tours: int) -> int:
  """CTA size of a one-CTA-per-tour 2-opt launch: wide CTAs when the batch leaves SMs idle,
  128-thread CTAs (eight resident per SM) when there are several tours per SM."""
  global _SM_COUNT
  if _SM_COUNT is None:
    _SM_COUNT = int(torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count)
  if num_tours <= _SM_COUNT:
    return 512
  if num_tours <= 4 * _SM_COUNT:
    return 256
  return 128


# bytes that this thread has already checked for the allocations that follow (checked_budget)
_CHECKED = threading.local()


def _checked() -> int:
  return getattr(_CHECKED, "bytes", 0)


@contextlib.contextmanager
def checked_budget(required_bytes: int, what: str):
  """Check once for the total of many allocations (a batch's distance matrices); the
  check_free calls inside the block, on the same thread, draw on that total instead of
  querying each time."""
  check_free(required_bytes, what)
  prev = _checked()
  _CHECKED.bytes = prev + int(required_bytes)
  try:
    yield
  finally:
    _CHECKED.bytes = prev


def check_free(required_bytes: int, what: str) -> None:
  """Raise VRAMInsufficientError before an allocation that cannot succeed. Memory that
  torch's caching allocator already holds unused is counted first (host-side counters);
  the driver is asked for free memory only when that does not cover the request."""
  if _checked() >= required_bytes:
    _CHECKED.bytes = _checked() - required_bytes
    return
  # the nested form skips the flattening that torch.cuda.memory_reserved/allocated do on
  # every call (tens of microseconds each, paid per instance of a large batch)
  stats = torch.cuda.memory_stats_as_nested_dict()
  try:
    cached = int(stats["reserved_bytes"]["all"]["current"]) - int(stats["allocated_bytes"]["all"]["current"])
  except KeyError:  # no allocation yet on this device
    cached = 0
  if required_bytes <= cached:
    return
  free, _ = torch.cuda.mem_get_info()
  if required_bytes > free + cached:
    raise VRAMInsufficientError(f"Insufficient VRAM for {what}", required_bytes=required_bytes,
                                available_bytes=free + cached)


class PinnedStager:
  """Reusable page-locked host buffers for H2D inputs and D2H results."""

  def __init__(self):
    self._bufs: dict[str, "torch.Tensor"] = {}

  def _buf(self, slot: str, nbytes: int):
    b = self._bufs.get(slot)
    if b is None or b.numel() < nbytes:
      b = torch.empty(max(nbytes, 1), dtype=torch.uint8, pin_memory=True)
      self._bufs[slot] = b
    return b

  def upload(self, a: np.ndarray, dtype) -> "torch.Tensor":
    a = np.ascontiguousarray(a)
    b = self._buf("in", a.nbytes)
    host = b[: a.nbytes].view(dtype).reshape(a.shape)
    host.numpy()[...] = a
    return host.to("cuda", non_blocking=True)

  def download(self, t: "torch.Tensor") -> np.ndarray:
    nbytes = t.numel() * t.element_size()
    b = self._buf("out", nbytes)
    host = b[:nbytes].view(t.dtype).reshape(t.shape)
    host.copy_(t, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    return host.numpy().copy()


class Workspace:
  """Monotonically growing device scratch buffer (grows, never shrinks)."""

  def __init__(self):
    self.buf = None

  def get(self, nbytes: int):
    if nbytes <= 0:
      return None
    if self.buf is None or self.buf.numel() < nbytes:
      check_free(nbytes, "2-opt workspace")
      self.buf = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    return self.buf


#: Largest |distance| for which the kernels' int32 gain arithmetic is exact.
MAX_DISTANCE = (1 << 30) - 1


class CandidateTables:
  """Device k-NN table, its distances, its reverse index (CSR) and the packed words.

  The packing kernel flags entries that do not fit 16 bits on the device; the flag is read
  on the first use of `packed` (None when an entry overflowed), or for many tables at once
  with `check_packed`, so building the tables does not wait for the device."""

  def __init__(self, cand, cand_dist, rev_off, rev_idx, packed=None, overflow=None):
    self.cand = cand
    self.cand_dist = cand_dist
    self.rev_off = rev_off
    self.rev_idx = rev_idx
    self._packed = packed
    self._overflow = overflow if packed is not None else None

  @property
  def packed(self):
    if self._overflow is not None:
      check_packed([self])
    return self._packed

  @property
  def packed_words(self):
    """The packed table before its overflow flag is read (callers then use check_packed)."""
    return self._packed

  @property
  def k(self) -> int:
    return int(self.cand.shape[1])


def check_packed(tables) -> None:
  """Read the pack-overflow flags of many CandidateTables with one device sync."""
  pending = [t for t in tables if t._overflow is not None]
  if not pending:
    return
  flags = torch.cat([t._overflow for t in pending]).cpu().numpy()
  for t, f in zip(pending, flags):
    if int(f) != 0:
      t._packed = None
    t._overflow = None

  @property
  def k(self) -> int:
    return int(self.cand.shape[1])


class DeviceOperands:
  """Device copies of one context's distances, coordinates and candidate tables.

  Uploaded once and reused by every strategy bound to the same context, the way
  the reference's `ProblemContext` owns its GPU caches (`problem_context.py:336-527`).
  """

  def __init__(self, context):
    # weak: the operands live in a WeakKeyDictionary keyed by the context, so a strong
    # reference here would keep every context (and its device matrices) alive for good
    self._context_ref = weakref.ref(context)
    self.h2d_bytes = 0
    self._dist = None
    self._coords = None
    self._symmetric = None
    # contexts of one Problem object (repetitions of a run) share its device data
    self._shared = _problem_cache(context)
    self._cand: dict[int, tuple] = self._shared.setdefault("cand", {}) if self._shared is not None else {}

  @property
  def context(self):
    ctx = self._context_ref()
    if ctx is None:
      raise RuntimeError("the problem context of these device operands no longer exists")
    return ctx

  def host_coords(self) -> np.ndarray:
    """The context's (n, 2) float64 coordinates, checked for the device's EUC_2D rebuild."""
    c = self.context.get_cpu_coordinates()
    if c is None:
      raise ValueError("problem has no coordinates for on-the-fly distances")
    c = np.ascontiguousarray(c, dtype=np.float64)
    if c.ndim != 2 or c.shape[1] != 2:
      raise ValueError("on-the-fly distances need (n, 2) EUC_2D coordinates")
    span = float(np.abs(c).max()) if c.size else 0.0
    if span * 2.0 * 1.5 >= MAX_DISTANCE:
      raise ValueError("coordinates too large for exact int32 gains")
    return c

  def has_coords(self) -> bool:
    return self._coords is not None or (self._shared is not None and "coords" in self._shared)

  def has_dist(self) -> bool:
    return self._dist is not None or (self._shared is not None and "dist" in self._shared)

  def set_coords(self, t) -> None:
    """Adopt device coordinates uploaded by the caller (a view of a batch upload)."""
    self._coords = t
    self.h2d_bytes += t.numel() * 8
    if self._shared is not None:
      self._shared["coords"] = t

  def coords(self):
    if self._coords is None and self._shared is not None:
      self._coords = self._shared.get("coords")
    if self._coords is None:
      self.set_coords(device_tensor(self.host_coords(), torch.float64))
    return self._coords

  def dist(self):
    if self._dist is None and self._shared is not None:
      self._dist = self._shared.get("dist")
    if self._dist is None:
      self._dist = self._build_dist()
      if self._shared is not None:
        self._shared["dist"] = self._dist
    return self._dist

  def _build_dist(self):
    if self._dist is None and self._euc2d_on_device():
      # The matrix of an EUC_2D coordinate problem is built in HBM from the coordinates with
      # the reference's rounding (compute_distance_matrix, matrix.py:214-273): only the
      # coordinates cross PCIe.
      n = int(self.context.dimension)
      check_free(n * n * 4, f"dense distance matrix (n={n})")
      d = torch.empty((n, n), dtype=torch.int32, device="cuda")
      if n:
        from .native import call

        call("tspb_euc2d_matrix", ptr(self.coords()), n, ptr(d), n, stream_handle())
      self._dist = d
    if self._dist is None and self._tsplib_on_device():
      # Every other coordinate type (ATT, GEO, CEIL_2D, MAN/MAX, 3-D, XRAY1) is built in HBM
      # by tspb_distance_matrix; its largest entry is checked against the int32 gain bound.
      from .native import EDGE_TYPE_CODES, call

      prob = self.context.problem
      c = np.ascontiguousarray(prob.coordinates, dtype=np.float64)
      n, dim = int(c.shape[0]), int(c.shape[1])
      check_free(n * n * 4, f"dense distance matrix (n={n})")
      d = torch.empty((n, n), dtype=torch.int32, device="cuda")
      if n:
        dc = device_tensor(c, torch.float64)
        self.h2d_bytes += c.nbytes
        call("tspb_distance_matrix", ptr(dc), n, dim, EDGE_TYPE_CODES[prob.edge_type], ptr(d), n, stream_handle())
        lo, hi = int(d.min().item()), int(d.max().item())
        if hi > MAX_DISTANCE or lo < 0:
          raise ValueError("distances outside [0, 2^30) are not supported by the int32 gain kernels")
      self._dist = d
    if self._dist is None:
      D = self.context.get_cpu_distances()
      D = np.ascontiguousarray(D, dtype=np.int32)
      if D.size and (int(D.max()) > MAX_DISTANCE or int(D.min()) < 0):
        raise ValueError("distances outside [0, 2^30) are not supported by the int32 gain kernels")
      check_free(D.nbytes, f"dense distance matrix (n={D.shape[0]})")
      self._dist = device_tensor(D, torch.int32)
      self.h2d_bytes += D.nbytes
    return self._dist

  @property
  def symmetric(self) -> bool:
    """d(a, b) == d(b, a) for every pair (the 2-opt's TSPB_MODE_SYMMETRIC). EUC_2D from
    coordinates is symmetric by its formula (dx and -dx square alike); any other matrix is
    compared with its transpose on the device once."""
    if self._symmetric is None and self._shared is not None:
      self._symmetric = self._shared.get("symmetric")
    if self._symmetric is None:
      if self._euc2d_on_device():
        sym = True
      else:
        d = self.dist()
        sym = bool(d.shape[0] == d.shape[1] and torch.equal(d, d.t()))
      self._symmetric = sym
      if self._shared is not None:
        self._shared["symmetric"] = sym
    return self._symmetric

  def _tsplib_on_device(self) -> bool:
    from .native import EDGE_TYPE_CODES

    prob = self.context.problem
    c = getattr(prob, "coordinates", None)
    if getattr(prob, "distances", None) is not None or c is None:
      return False
    shape = np.shape(c)
    return getattr(prob, "edge_type", "EUC_2D") in EDGE_TYPE_CODES and len(shape) == 2 and shape[1] in (2, 3)

  def _euc2d_on_device(self) -> bool:
    prob = self.context.problem
    if getattr(prob, "distances", None) is not None or getattr(prob, "coordinates", None) is None:
      return False
    return getattr(prob, "edge_type", "EUC_2D") == "EUC_2D"

  def use_coords(self, n: int, max_matrix_dimension: int | None) -> bool:
    threshold = max_matrix_dimension
    if threshold is None:
      threshold = int(getattr(self.context, "max_matrix_dimension", 10_000))
    prob = self.context.problem
    return (
      n > threshold
      and getattr(prob, "edge_type", "EUC_2D") == "EUC_2D"
      and getattr(prob, "coordinates", None) is not None
    )

  def distance_args(self, n: int, max_matrix_dimension: int | None = None):
    """`(dist_tensor_or_None, stride, coords_tensor_or_None)` for one launch."""
    if self.use_coords(n, max_matrix_dimension):
      return None, 0, self.coords()
    d = self.dist()
    return d, int(d.shape[1]), None

  def candidates(self, k: int, table: np.ndarray, n: int, max_matrix_dimension: int | None = None):
    """Device `CandidateTables` for a host k-NN table (cached per k and table identity)."""
    key = int(k)
    hit = self._cand.get(key)
    if hit is not None and hit[0] is table:
      return hit[1]
    from .native import call

    tab = np.ascontiguousarray(table, dtype=np.int32)
    d_cand = device_tensor(tab, torch.int32)
    self.h2d_bytes += tab.nbytes
    rows, kk = tab.shape
    d_cd = torch.empty((rows, kk), dtype=torch.int32, device="cuda")
    rev_off = torch.empty(rows + 1, dtype=torch.int32, device="cuda")
    rev_idx = torch.empty(max(rows * kk, 1), dtype=torch.int32, device="cuda")
    scratch = torch.empty(max(rows, 1), dtype=torch.int32, device="cuda")
    dist, stride, coords = self.distance_args(n, max_matrix_dimension)
    if rows and kk:
      call("tspb_candidate_distances", ptr(d_cand), rows, kk, ptr(dist), stride, ptr(coords), ptr(d_cd), stream_handle())
      call("tspb_candidate_reverse_index", ptr(d_cand), rows, kk, ptr(rev_off), ptr(rev_idx), ptr(scratch), stream_handle())
    packed = overflow = None
    if rows and kk and rows <= 0xFFFF:
      packed = torch.empty((rows, kk), dtype=torch.int32, device="cuda")
      overflow = torch.empty(1, dtype=torch.int32, device="cuda")  # zeroed by tspb_candidate_pack
      call("tspb_candidate_pack", ptr(d_cand), ptr(d_cd), rows, kk, ptr(packed), ptr(overflow), stream_handle())
    tables = CandidateTables(d_cand, d_cd, rev_off, rev_idx, packed, overflow)
    self._cand[key] = (table, tables)
    return tables


def upload_coordinates(ops_list) -> None:
  """One H2D copy for the coordinates of every operand set in `ops_list` that has none on
  the device yet; each adopts a view of the upload (offsets of 16 bytes per city, so every
  view stays aligned for the kernels' double2 loads). Operand sets that share a problem's
  data are uploaded once."""
  todo, seen = [], set()
  for o in ops_list:
    key = id(o._shared) if o._shared is not None else id(o)
    if o.has_coords() or key in seen:
      continue
    seen.add(key)
    todo.append(o)
  if not todo:
    return
  hosts = [o.host_coords() for o in todo]
  total = sum(len(h) for h in hosts)
  buf = torch.empty((max(total, 1), 2), dtype=torch.float64, pin_memory=True)
  arr = buf.numpy()
  off = 0
  for h in hosts:
    arr[off:off + len(h)] = h
    off += len(h)
  dev = buf.to("cuda", non_blocking=True)  # the caching host allocator holds buf until the copy has run
  off = 0
  for o, h in zip(todo, hosts):
    o.set_coords(dev[off:off + len(h)])
    off += len(h)


def _host_knn_rows(context, rows: np.ndarray, k_eff: int, dist=None) -> np.ndarray:
  """Rows of the reference's k-NN table computed by its own procedure (`matrix.py:177-211`:
  self masked with the largest int64, argpartition, then lexsort by (distance, id)).
  NumPy partitions every row of a block independently, so a row's result does not depend
  on the other rows of the block it is computed with. The rows' distances come from the
  device matrix `dist` when given (the same values), else from the host formula."""
  from .problem import distance_block

  prob = context.problem
  if getattr(prob, "distances", None) is not None:
    block = np.asarray(prob.distances[rows], dtype=np.int64)
  elif dist is not None:
    block = dist[torch.from_numpy(rows).to(dist.device)].cpu().numpy().astype(np.int64)
  else:
    c = np.asarray(prob.coordinates, dtype=np.float64)
    block = distance_block(c[rows], c, getattr(prob, "edge_type", "EUC_2D")).astype(np.int64)
  r = np.arange(len(rows))
  block[r, rows] = np.iinfo(np.int64).max
  cols = np.argpartition(block, k_eff, axis=1)[:, :k_eff]
  cd = block[r[:, None], cols]
  order = np.lexsort((cols, cd), axis=1)
  return cols[r[:, None], order].astype(np.int32)


def candidate_list(context, k: int) -> np.ndarray:
  """The context's k-NN table `get_cpu_candidate_list(k)` (`problem_context.py:420-454`),
  built on the device: `tspb_knn_ties` gives every row ordered by (distance, id) and flags
  the rows with a tie at the k-th boundary, the only rows where the reference's
  argpartition may pick other tied nodes; those rows are taken from the reference's own
  procedure on the host. The table is stored in the context's candidate cache, so the
  host API and every strategy bound to the context see the same table."""
  cache = getattr(context, "_cpu_candidate_lists", None)
  if cache is not None and k in cache:
    return cache[k]
  n = int(context.dimension)
  prob = context.problem
  usable = (cache is not None and n > 1 and 0 < k and min(k, n - 1) + 1 <= 64
            and (getattr(prob, "distances", None) is not None or getattr(prob, "coordinates", None) is not None))
  if not usable:
    return context.get_cpu_candidate_list(k)
  from .native import call

  k_eff = min(k, n - 1)
  ops = operands_for(context)
  dist, stride, coords = ops.distance_args(n, None)
  out = torch.empty((n, k_eff), dtype=torch.int32, device="cuda")
  ties = torch.zeros(n, dtype=torch.int32, device="cuda")
  if k_eff == n - 1:  # every other node: no (k+1)-th entry, no boundary
    call("tspb_knn", ptr(dist), stride, ptr(coords), n, k_eff, ptr(out), stream_handle())
  else:
    call("tspb_knn_ties", ptr(dist), stride, ptr(coords), n, k_eff, ptr(out), ptr(ties), stream_handle())
  table = out.cpu().numpy()
  tied = np.nonzero(ties.cpu().numpy())[0]
  if tied.size:
    # the device matrix holds the reference's values bit for bit except for GEO (device cos/acos)
    rows_from = dist if dist is not None and getattr(prob, "edge_type", "EUC_2D") != "GEO" else None
    table[tied] = _host_knn_rows(context, tied, k_eff, rows_from)
  cache[k] = table
  return table


_operands: "weakref.WeakKeyDictionary[Any, DeviceOperands]" = weakref.WeakKeyDictionary()
_problems: "weakref.WeakKeyDictionary[Any, dict]" = weakref.WeakKeyDictionary()


def _problem_cache(context) -> dict | None:
  """Device data shared by the contexts of one Problem object, or None when the problem
  cannot be weakly referenced."""
  prob = getattr(context, "problem", None)
  if prob is None:
    return None
  try:
    return _problems.setdefault(prob, {})
  except TypeError:
    return None


def operands_for(context) -> DeviceOperands:
  ops = _operands.get(context)
  if ops is None:
    ops = DeviceOperands(context)
    _operands[context] = ops
  return ops
