"""TSPLIB reader and the edge-type-aware host context (CPU)."""

from __future__ import annotations

import os
from pathlib import Path

import numpy as np
import pytest

from oracle import distances as odist
from tsp_gpu_clean_b200 import tsplib
from tsp_gpu_clean_b200.problem import ProblemContext

from reference_env import checkout_root  # noqa: E402

REFERENCE = checkout_root() or ""  # the fixture files live only in a checkout (TSPB_REFERENCE)


def _layout_values(d: np.ndarray, fmt: str) -> list[int]:
  """The numbers of an EDGE_WEIGHT_SECTION, written from the layout definitions
  (row-wise layouts walk rows, column-wise ones walk columns)."""
  n = d.shape[0]
  if fmt == "FULL_MATRIX":
    return [d[i, j] for i in range(n) for j in range(n)]
  rowwise = fmt.endswith("_ROW")
  upper = fmt.startswith("UPPER")
  diag = "_DIAG_" in fmt
  out = []
  for a in range(n):
    for b in range(n):
      i, j = (a, b) if rowwise else (b, a)
      keep = (j > i or (diag and j == i)) if upper else (j < i or (diag and j == i))
      if keep:
        out.append(d[i, j])
  return out


def _explicit_text(d: np.ndarray, fmt: str) -> str:
  vals = _layout_values(d, fmt)
  body = "\n".join(" ".join(str(v) for v in vals[s : s + 7]) for s in range(0, len(vals), 7))
  return (f"NAME: m{d.shape[0]}\nTYPE: TSP\nDIMENSION: {d.shape[0]}\nEDGE_WEIGHT_TYPE: EXPLICIT\n"
          f"EDGE_WEIGHT_FORMAT: {fmt} \nEDGE_WEIGHT_SECTION\n{body}\nEOF\n")


def _coord_text(c: np.ndarray, edge_type: str) -> str:
  rows = "\n".join(f"{i + 1} " + " ".join(repr(float(v)) for v in c[i]) for i in range(len(c)))
  return (f"NAME : c{len(c)}\nTYPE : TSP\nCOMMENT : synthetic: seeded\nDIMENSION : {len(c)}\n"
          f"EDGE_WEIGHT_TYPE : {edge_type}\nNODE_COORD_SECTION\n{rows}\nEOF\n")


@pytest.mark.parametrize("fmt", tsplib.EXPLICIT_FORMATS)
def test_explicit_layouts_round_trip(fmt):
  rng = np.random.default_rng(len(fmt))
  for n in (1, 2, 9):
    a = rng.integers(0, 1000, (n, n))
    d = np.triu(a, 1)
    d = (d + d.T).astype(np.int32)
    p = tsplib.problem_from_text(_explicit_text(d, fmt))
    assert p.edge_type == "EXPLICIT" and p.dimension == n
    assert np.array_equal(p.distances, d)


@pytest.mark.parametrize("edge_type", ["EUC_2D", "ATT", "GEO", "CEIL_2D", "EUC_3D", "MAN_2D", "XRAY1"])
def test_coordinate_types_give_the_oracle_matrix_and_knn(edge_type):
  from tests.golden.make_golden import dist_coords

  c = dist_coords(edge_type, 60, 31)
  p = tsplib.problem_from_text(_coord_text(c, edge_type))
  assert p.edge_type == edge_type and p.coordinates.shape == c.shape
  ctx = ProblemContext(p, seed=0)
  assert np.array_equal(ctx.get_cpu_distances(), odist.distance_matrix(c, edge_type))
  assert np.array_equal(ctx.get_cpu_candidate_list(7), odist.candidate_list(7, coords=c, edge_type=edge_type))


def test_tours_and_errors():
  tour = tsplib.tour_from_text("NAME: t\nTYPE: TOUR\nDIMENSION: 4\nTOUR_SECTION\n3\n1\n4 2\n-1\nEOF\n")
  assert tour.tolist() == [2, 0, 3, 1]
  with pytest.raises(tsplib.TsplibFormatError):
    tsplib.tour_from_text("TOUR_SECTION\n1 1 2\n-1\n")
  with pytest.raises(tsplib.TsplibFormatError):
    tsplib.problem_from_text("NAME: x\nTYPE: TSP\nEDGE_WEIGHT_TYPE: EUC_2D\nNODE_COORD_SECTION\n1 0 0\n")
  with pytest.raises(tsplib.TsplibFormatError):
    tsplib.problem_from_text("NAME: x\nTYPE: CVRP\nDIMENSION: 2\nEDGE_WEIGHT_TYPE: EUC_2D\n")
  with pytest.raises(tsplib.TsplibFormatError):
    tsplib.problem_from_text("NAME: x\nDIMENSION: 2\nEDGE_WEIGHT_TYPE: EUC_2D\nNODE_COORD_SECTION\n1 0 0\n3 1 1\n")
  with pytest.raises(tsplib.TsplibFormatError):
    tsplib.problem_from_text(_explicit_text(np.zeros((3, 3), np.int32), "UPPER_ROW").replace("UPPER_ROW", "SPIRAL"))


@pytest.mark.skipif(not REFERENCE or not os.path.isdir(os.path.join(REFERENCE, "tests", "fixtures", "tsp")),
                    reason="reference checkout not present")
def test_reference_fixture_instances_parse():
  """The TSPLIB files of the reference's own test fixtures (EUC_2D, ATT, GEO, and EXPLICIT
  in LOWER_DIAG_ROW and UPPER_ROW with display data) parse into symmetric matrices with a
  zero diagonal that equal the oracle's formulas on the parsed coordinates."""
  root = Path(REFERENCE) / "tests" / "fixtures" / "tsp"
  seen = {}
  for f in sorted(root.glob("*.tsp")):
    p = tsplib.read_problem(f)
    d = ProblemContext(p, seed=0).get_cpu_distances()
    assert d.shape == (p.dimension, p.dimension)
    assert np.array_equal(d, d.T) and not np.diag(d).any()
    if p.coordinates is not None and p.edge_type != "EXPLICIT":
      assert np.array_equal(d, odist.distance_matrix(p.coordinates, p.edge_type))
    seen[p.edge_type] = seen.get(p.edge_type, 0) + 1
  assert {"EUC_2D", "ATT", "GEO", "EXPLICIT"} <= set(seen)
