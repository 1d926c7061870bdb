"""bench.py's reference arm on the host: the one JSON line and its keys (tiny sizes, no GPU).

The arm times the reference's own CPU implementation (the reference extension compiled from
its sources under oracle/_ref) on a bounded sample and scales it to the workload; under
torchrun only rank 0 prints.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _run(extra_env=None, *args):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run(
        [sys.executable, str(ROOT / "bench.py"), *args],
        cwd=ROOT,
        env=env,
        capture_output=True,
        text=True,
        timeout=600,
    )


def test_reference_arm_line():
    out = _run(None, "--impl", "reference", "--steps", "1", "--warmup", "0", "--mesh", "12", "--cpu-sample-mesh", "6")
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:  # the reference extension was not built here
        return
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["higher_is_better"] is False and d["unit"] == "ms" and d["value"] > 0
    assert d["value"] == d["ms_per_step"] == d["cpu_baseline"]["value"] == d["e2e"]["value"]
    assert d["config"]["workload"] and d["config"]["mesh"] == "12x12"
    cpu = d["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["cores"] >= 1 and "6x6" in cpu["sample"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_are_silent():
    out = _run({"RANK": "1", "WORLD_SIZE": "2"}, "--impl", "reference", "--steps", "1", "--warmup", "0", "--mesh", "12")
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip() == ""
