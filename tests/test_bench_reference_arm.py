"""bench.py's reference arm on the CPU: one JSON line with impl "reference", the CPU
baseline it timed and a zero-copy e2e; ranks other than 0 print nothing and exit 0."""

from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, env_extra=None):
  env = dict(os.environ)
  env.pop("RANK", None)
  env.pop("WORLD_SIZE", None)
  env.update(env_extra or {})
  p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                     capture_output=True, text=True, env=env, cwd=ROOT, timeout=240)
  assert p.returncode == 0, p.stderr[-2000:]
  return [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]


@pytest.mark.timeout(300)
@pytest.mark.parametrize("args", [["--workload", "ga100", "--cpu-gens", "3"], ["--workload", "or_opt"]])
def test_reference_arm_prints_one_contract_line(args):
  lines = _run([*args, "--steps", "1", "--warmup", "3"])
  assert len(lines) == 1
  d = lines[0]
  assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
  assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
  assert d["cpu_baseline"]["value"] == d["value"] and d["e2e"]["value"] == d["value"]
  assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
  assert d["unit"] == d["e2e"]["unit"] and d["config"]["workload"]


@pytest.mark.timeout(120)
def test_reference_arm_other_ranks_exit_quietly():
  assert _run(["--workload", "ga100", "--cpu-gens", "3", "--steps", "1", "--warmup", "3"],
              {"RANK": "1", "WORLD_SIZE": "2"}) == []
