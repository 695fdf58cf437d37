"""TSPLIB reader for symmetric TSP instances and tours (format of Reinelt's TSPLIB95).

The reference reads TSPLIB files through its `routing-data` dependency
(`src/loaders/tsplib_loader.py`, `tsplib_ingestor.py`), which is not installable offline;
this module is a reader of its own for what the hot path needs:

- the specification part (`NAME`, `TYPE`, `DIMENSION`, `EDGE_WEIGHT_TYPE`,
  `EDGE_WEIGHT_FORMAT`, ...; `KEY: value` with free spacing around the colon);
- `NODE_COORD_SECTION` (2 or 3 coordinates per node) for the coordinate types
  EUC_2D/3D, MAN_2D/3D, MAX_2D/3D, CEIL_2D, ATT, GEO and XRAY1;
- `EDGE_WEIGHT_SECTION` for `EXPLICIT` instances in every symmetric layout: FULL_MATRIX,
  UPPER_ROW, LOWER_ROW, UPPER_DIAG_ROW, LOWER_DIAG_ROW, UPPER_COL, LOWER_COL,
  UPPER_DIAG_COL, LOWER_DIAG_COL;
- `DISPLAY_DATA_SECTION` (kept as coordinates of an EXPLICIT instance);
- `TOUR_SECTION` of `.tour` / `.opt.tour` files (node ids until -1).

Node ids are 1-based in the file and 0-based in the arrays returned. The result is a
`problem.Problem`, so `ProblemContext` builds its distances (on the device for every
coordinate type) and k-NN tables from it like any other problem.
"""

from __future__ import annotations

from pathlib import Path
from typing import Iterable

import numpy as np

from .problem import COORDINATE_EDGE_TYPES, Problem

EXPLICIT_FORMATS = ("FULL_MATRIX", "UPPER_ROW", "LOWER_ROW", "UPPER_DIAG_ROW", "LOWER_DIAG_ROW", "UPPER_COL",
                    "LOWER_COL", "UPPER_DIAG_COL", "LOWER_DIAG_COL")
_SECTIONS = ("NODE_COORD_SECTION", "EDGE_WEIGHT_SECTION", "DISPLAY_DATA_SECTION", "TOUR_SECTION", "DEPOT_SECTION",
             "DEMAND_SECTION", "FIXED_EDGES_SECTION")


class TsplibFormatError(ValueError):
  pass


def _cells(n: int, fmt: str) -> Iterable[tuple[int, int]]:
  """(i, j) of every stored entry of a symmetric layout, in file order."""
  if fmt == "FULL_MATRIX":
    return ((i, j) for i in range(n) for j in range(n))
  if fmt in ("UPPER_ROW", "LOWER_COL"):
    return ((i, j) for i in range(n) for j in range(i + 1, n))
  if fmt in ("LOWER_ROW", "UPPER_COL"):
    return ((i, j) for i in range(n) for j in range(i))
  if fmt in ("UPPER_DIAG_ROW", "LOWER_DIAG_COL"):
    return ((i, j) for i in range(n) for j in range(i, n))
  if fmt in ("LOWER_DIAG_ROW", "UPPER_DIAG_COL"):
    return ((i, j) for i in range(n) for j in range(i + 1))
  raise TsplibFormatError(f"unsupported EDGE_WEIGHT_FORMAT {fmt!r}")


def explicit_matrix(values: np.ndarray, n: int, fmt: str) -> np.ndarray:
  """Symmetric int32 matrix from the numbers of an EDGE_WEIGHT_SECTION. A column-wise
  layout lists the transpose of the matching row-wise one, which for a symmetric matrix
  is the same sequence of values (UPPER_COL as LOWER_ROW, LOWER_DIAG_COL as UPPER_DIAG_ROW)."""
  cells = list(_cells(n, fmt))
  if len(values) < len(cells):
    raise TsplibFormatError(f"EDGE_WEIGHT_SECTION has {len(values)} numbers, {fmt} of n={n} needs {len(cells)}")
  d = np.zeros((n, n), dtype=np.int64)
  if cells:
    ij = np.asarray(cells, dtype=np.int64)
    v = np.asarray(values[: len(cells)], dtype=np.float64)
    if not np.all(v == np.round(v)):
      raise TsplibFormatError("EDGE_WEIGHT_SECTION holds non-integer weights")
    d[ij[:, 0], ij[:, 1]] = v.astype(np.int64)
    if fmt != "FULL_MATRIX":
      d[ij[:, 1], ij[:, 0]] = v.astype(np.int64)
  if np.abs(d).max(initial=0) >= 2**31:
    raise TsplibFormatError("weights do not fit int32")
  return d.astype(np.int32)


def parse(text: str, name: str | None = None) -> dict:
  """Specification entries (upper-case keys) and the raw numbers of each data section."""
  spec: dict[str, str] = {}
  sections: dict[str, list[str]] = {}
  current: list[str] | None = None
  for raw in text.splitlines():
    line = raw.strip()
    if not line:
      continue
    head = line.split(":", 1)[0].strip().upper() if ":" in line else line.split()[0].upper()
    if head == "EOF":
      break
    if head in _SECTIONS:
      current = sections.setdefault(head, [])
      rest = line.split(":", 1)[1] if ":" in line else line[len(line.split()[0]):]
      current.extend(rest.split())
      continue
    if ":" in line and head.replace("_", "").isalpha():
      spec[head] = line.split(":", 1)[1].strip()
      current = None
      continue
    if current is None:
      raise TsplibFormatError(f"data line outside a section: {raw!r}")
    current.extend(line.split())
  if name is not None:
    spec.setdefault("NAME", name)
  return {"spec": spec, "sections": sections}


def _node_rows(tokens: list[str], n: int, cols: int, what: str) -> np.ndarray:
  if len(tokens) < n * (cols + 1):
    raise TsplibFormatError(f"{what} has {len(tokens)} numbers, n={n} needs {n * (cols + 1)}")
  arr = np.asarray(tokens[: n * (cols + 1)], dtype=np.float64).reshape(n, cols + 1)
  ids = arr[:, 0].astype(np.int64)
  if sorted(ids.tolist()) != list(range(1, n + 1)):
    raise TsplibFormatError(f"{what}: node ids must be 1..{n}")
  out = np.empty((n, cols), dtype=np.float64)
  out[ids - 1] = arr[:, 1:]
  return out


def problem_from_text(text: str, name: str | None = None) -> Problem:
  """`Problem` of a symmetric TSP instance in TSPLIB format."""
  parsed = parse(text, name)
  spec, sec = parsed["spec"], parsed["sections"]
  ptype = spec.get("TYPE", "TSP").split()[0].upper()
  if ptype not in ("TSP",):
    raise TsplibFormatError(f"TYPE {ptype!r}: only symmetric TSP instances are read")
  if "DIMENSION" not in spec:
    raise TsplibFormatError("missing DIMENSION")
  n = int(spec["DIMENSION"])
  etype = spec.get("EDGE_WEIGHT_TYPE", "EUC_2D").split()[0].upper()
  pname = spec.get("NAME", "tsplib").split()[0] if spec.get("NAME") else "tsplib"
  if etype == "EXPLICIT":
    fmt = spec.get("EDGE_WEIGHT_FORMAT", "FULL_MATRIX").split()[0].upper()
    if "EDGE_WEIGHT_SECTION" not in sec:
      raise TsplibFormatError("EXPLICIT instance without EDGE_WEIGHT_SECTION")
    d = explicit_matrix(np.asarray(sec["EDGE_WEIGHT_SECTION"], dtype=np.float64), n, fmt)
    display = sec.get("DISPLAY_DATA_SECTION")
    coords = _node_rows(display, n, 2, "DISPLAY_DATA_SECTION") if display else None
    return Problem(name=pname, dimension=n, problem_type="TSP", edge_type="EXPLICIT", coordinates=coords, distances=d)
  if etype not in COORDINATE_EDGE_TYPES:
    raise TsplibFormatError(f"unsupported EDGE_WEIGHT_TYPE {etype!r}")
  if "NODE_COORD_SECTION" not in sec:
    raise TsplibFormatError(f"{etype} instance without NODE_COORD_SECTION")
  tokens = sec["NODE_COORD_SECTION"]
  cols = 3 if (etype.endswith("_3D") or etype == "XRAY1" or spec.get("NODE_COORD_TYPE", "").upper() == "THREED_COORDS"
               or len(tokens) == 4 * n) else 2
  coords = _node_rows(tokens, n, cols, "NODE_COORD_SECTION")
  return Problem.from_coordinates(coords, name=pname, edge_type=etype)


def read_problem(path: str | Path) -> Problem:
  p = Path(path)
  return problem_from_text(p.read_text(), name=p.stem)


def tour_from_text(text: str) -> np.ndarray:
  """0-based node order of a TOUR_SECTION (ids until -1 or the end of the section)."""
  sec = parse(text)["sections"].get("TOUR_SECTION")
  if sec is None:
    raise TsplibFormatError("missing TOUR_SECTION")
  ids = []
  for tok in sec:
    v = int(tok)
    if v == -1:
      break
    ids.append(v - 1)
  tour = np.asarray(ids, dtype=np.int32)
  if sorted(tour.tolist()) != list(range(len(tour))):
    raise TsplibFormatError("TOUR_SECTION is not a permutation of 1..n")
  return tour


def read_tour(path: str | Path) -> np.ndarray:
  return tour_from_text(Path(path).read_text())
