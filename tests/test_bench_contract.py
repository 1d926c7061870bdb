"""bench.py's reference arm on the host: the one JSON line and its keys (tiny sizes, no GPU).

The arm times the reference's own CPU implementation (the reference extension compiled from
its sources under oracle/_ref) on the sample mesh it can finish, reports that measured time
under that mesh's name, and loads none of this repository's native libraries; under
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
    # one reference thread: its multi-threaded decompose can hang on tiny systems (a data
    # race in its scheduler; bench.py runs it in a child process with a time limit)
    out = _run(None, "--impl", "reference", "--steps", "1", "--warmup", "0", "--mesh", "12", "--cpu-sample-mesh", "6",
               "--ref-threads", "1")
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
    # the config names the mesh that was measured, and which workload it samples
    assert d["config"]["mesh"] == "6x6" and "12x12" in d["config"]["sample_of"]
    assert d["config"]["factor_gflop"] > 0
    cpu = d["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["cores"] >= 1 and "6x6" in cpu["sample"]
    assert "not extrapolated" in cpu["sample"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_reference_arm_loads_no_repo_library():
    """The reference leg imports the generator by file and counts flops from the reference's
    own factored pattern: neither libhybsol_b200.so nor the hybsol._mod extension loads."""
    code = (
        "import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', "
        "'--mesh', '12', '--cpu-sample-mesh', '4', '--ref-threads', '1']\n"
        "try:\n    runpy.run_path('bench.py', run_name='__main__')\nexcept SystemExit:\n    pass\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('LOADED', 'libhybsol_b200' in maps, 'hybsol/_mod' in maps)\n"
    )
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "LOADED False False" in out.stdout, out.stdout[-500:]


def test_reference_leg_runs_in_a_child_process():
    """The reference's decompose runs in a child process under a time limit (its
    multi-threaded scheduler can hang); the parent gets its times, residual, solution and
    the flops counted from its factored pattern."""
    import numpy as np

    sys.path.insert(0, str(ROOT))
    import bench

    times, res, x, flops = bench.reference_sample(4, 8, 2, 0, 1)
    assert len(times) == 2 and res < 1e-12 and flops > 0 and np.isfinite(x).all()


def test_reference_arm_other_ranks_are_silent():
    out = _run({"RANK": "1", "WORLD_SIZE": "2"}, "--impl", "reference", "--steps", "1", "--warmup", "0", "--mesh", "12")
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip() == ""
