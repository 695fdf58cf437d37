"""Exceptions of the B200 strategies, mirroring the reference's names and meaning.

`GPUUnavailableError` and `VRAMInsufficientError` follow
`src/data_models/exceptions.py:221, 232` of the reference: GPU strategies raise
them instead of falling back to a CPU path (`two_opt.py:746-754`).
"""

from __future__ import annotations


class TSPB200Error(RuntimeError):
  """Base class for errors raised by the B200 kernels or their host wrappers."""


class GPUUnavailableError(TSPB200Error):
  """No CUDA device is reachable, or libtspb.so is not built/loadable."""


class VRAMInsufficientError(TSPB200Error):
  """An allocation would not fit in free device memory."""

  def __init__(self, message: str, required_bytes: int = 0, available_bytes: int = 0):
    super().__init__(f"{message} (required {required_bytes} B, available {available_bytes} B)")
    self.required_bytes = required_bytes
    self.available_bytes = available_bytes


class KernelError(TSPB200Error):
  """A libtspb entry point returned a non-zero status."""

  def __init__(self, func: str, status: int, text: str):
    super().__init__(f"{func}: status {status} ({text})")
    self.func = func
    self.status = status


class NotPermutationError(ValueError):
  """An input route is not a permutation of 0..n-1 (reported by the kernel)."""
