"""Test configuration: import paths, the `gpu` marker, shared helpers.

`-m "not gpu"` runs everything that needs no GPU (oracle vs golden vectors, the symbolic
phase and orderings, the host side of the extension, that the C-ABI library loads and
exports its symbols). `-m gpu` runs the parity tests proper on a B200, through the C ABI
and the `hybsol` extension; they fail (never skip) when no sm_100 device is visible.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "hybridized-solver_b200"
GOLDEN = Path(__file__).resolve().parent / "golden"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)

os.environ.setdefault("OMP_NUM_THREADS", "1")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def native():
    from hybsol.b200 import native as nat

    return nat


@pytest.fixture(scope="session")
def gpu(native):
    """The C-ABI module, after checking that a B200 is visible (fails loudly otherwise)."""
    if not native.device_available():
        pytest.fail("no sm_100 CUDA device visible: GPU tests must run on a B200")
    return native


def golden(name: str):
    return np.load(GOLDEN / name)


def reorder_rhs(sizes_old, order, b):
    """Move a vector (or (dof, k) block) from the old block layout to the new one."""
    sizes_old = np.asarray(sizes_old, dtype=np.int64)
    order = np.asarray(order, dtype=np.int64)
    n = len(sizes_old)
    new_sizes = np.empty(n, dtype=np.int64)
    new_sizes[order] = sizes_old
    off_old = np.concatenate([[0], np.cumsum(sizes_old)])
    off_new = np.concatenate([[0], np.cumsum(new_sizes)])
    out = np.empty_like(b)
    for i in range(n):
        out[off_new[order[i]] : off_new[order[i] + 1]] = b[off_old[i] : off_old[i + 1]]
    return out


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / den)
