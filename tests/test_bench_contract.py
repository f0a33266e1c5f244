"""bench.py's reference arm on the host: the reference's own compiled CPU path
(oracle/_ref) timed on the 8^3 Kuhn box, printed as one JSON line with the
GPU arm's metric, unit and workload; ranks other than 0 print nothing."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from oracle import ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "0",
                          "--steps", "2", "--warmup", "3"], capture_output=True, text=True, timeout=600, env=env,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    return [l for l in out.stdout.splitlines() if l.strip()]


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_reference_arm_json_line():
    lines = _run({"RANK": "0"})
    assert len(lines) == 1
    line = json.loads(lines[0])
    import bench
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "particle-steps/s"
    assert line["higher_is_better"] is True and line["steps"] == 2 and line["warmup"] == 3
    assert line["config"]["workload"] == bench.CONFIGS[0]["label"]
    assert line["value"] > 0 and line["newton_step_ms"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_silent():
    assert _run({"RANK": "1"}) == []
