"""Failure paths on the GPU without a GPU fault.

A bounded device-side wait is made to run out on purpose: host-side fault injection
(HYB_OPTION_WITHHOLD_ROW) keeps the pre-sum of one block row's early partial products
from ever being released in the dataflow solve, and the wait limit is shortened to a
few milliseconds (HYB_OPTION_WAIT_LIMIT_NS). The waiting CTAs give up, the solve returns
HYB_DEVICE_TIMEOUT, and the same handle then solves correctly -- the context stays usable.
Nothing here traps, faults or hangs the device: every wait ends at its limit.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import reorder_rhs

pytestmark = pytest.mark.gpu


def _system(native, n, p, seed):
    from hybsol.b200 import meshgen

    mat, b = meshgen.mesh_system(n, p, seed=seed)
    order = native.compute_ordering(mat.row_ptr, mat.cols, "first")
    pm = mat.permuted(order)
    ns = native.NativeSystem.from_matrix(pm)
    return ns, pm, reorder_rhs(mat.sizes, order, b)


def _row_with_two_lower_blocks(ns, n_blocks):
    for r in range(n_blocks - 1, -1, -1):
        if sum(1 for c in ns.row_cols(r) if c < r) >= 2:
            return r
    raise AssertionError("no block row with two lower blocks")


@pytest.mark.parametrize("prec", [0, 1])
def test_dataflow_wait_runs_out_and_handle_stays_usable(gpu, prec):
    ns, pm, bn = _system(gpu, 8, 4, seed=3)
    ns.decompose(prec)
    x_ok, info_ok = ns.solve(bn)
    assert info_ok["converged"]
    row = _row_with_two_lower_blocks(ns, pm.n_blocks)
    ns.set_option(gpu.OPTION_WAIT_LIMIT_NS, 2_000_000)  # 2 ms per wait
    ns.set_option(gpu.OPTION_WITHHOLD_ROW, row)
    with pytest.raises(gpu.HybError) as err:
        ns.solve(bn)
    assert err.value.status == gpu.DEVICE_TIMEOUT
    # injection off, default limit: the same handle and factors solve as before
    ns.set_option(gpu.OPTION_WITHHOLD_ROW, -1)
    ns.set_option(gpu.OPTION_WAIT_LIMIT_NS, 1_000_000_000)
    x, info = ns.solve(bn)
    assert np.array_equal(x, x_ok) and info["iterations"] == info_ok["iterations"]
    # and it can be factored again
    ns.decompose(prec)
    x2, _ = ns.solve(bn)
    assert np.array_equal(x2, x_ok)


def test_withhold_row_needs_two_lower_blocks(gpu):
    ns, pm, _ = _system(gpu, 4, 2, seed=1)
    ns.decompose(0)
    # block row 0 has nothing left of its diagonal
    with pytest.raises(gpu.HybError) as err:
        ns.set_option(gpu.OPTION_WITHHOLD_ROW, 0)
    assert err.value.status == 16
    with pytest.raises(gpu.HybError):
        ns.set_option(gpu.OPTION_WAIT_LIMIT_NS, 0)
