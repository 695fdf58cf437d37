"""Where tests find the reference implementation, when it is present at all.

- `TSPB_REFERENCE`: the root of a reference checkout (its packages under `src/`, its
  fixture files under `tests/fixtures/`);
- otherwise the offline install of the reference's packages under `baseline/_ref` of
  this repository (`pip install --no-deps --target baseline/_ref <checkout>`), which
  holds the packages but no fixture files.

Tests that need the reference skip when neither is there.
"""

from __future__ import annotations

import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INSTALLED = os.path.join(ROOT, "baseline", "_ref")


def checkout_root() -> str | None:
  """The reference checkout named by TSPB_REFERENCE, or None."""
  root = os.environ.get("TSPB_REFERENCE")
  return root if root and os.path.isdir(os.path.join(root, "src")) else None


def import_root() -> str | None:
  """Directory holding the reference's packages (`algorithms`, `protocols`, ...), or None."""
  root = checkout_root()
  if root is not None:
    return os.path.join(root, "src")
  if os.path.isdir(os.path.join(INSTALLED, "algorithms")) and os.path.isdir(os.path.join(INSTALLED, "protocols")):
    return INSTALLED
  return None
