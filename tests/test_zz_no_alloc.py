"""The allocation-free FP64 solve entry point, hyb_solve_fp64_noalloc.

It is for callers that must not allocate device memory while they solve (their own pool
owns the device memory, or a cudaMalloc/cudaFree would synchronize a running loop): the
handle is created and factored beforehand, and the entry point itself only uses the
caller's device buffers and a fixed scratch array inside the library. These tests call
it through the C ABI, twice in a row on the same handle, and compare with hyb_solve (bit
for bit: both substitute with the same partial products summed in the same order) and with
the oracle. They run alone or after the rest of the suite (this file is collected last).
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import rel_err, reorder_rhs  # noqa: F401

pytestmark = pytest.mark.gpu


def _bind(native):
    lib = native.lib()
    fn = lib.hyb_solve_fp64_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    return fn


def _factored(native, n, p, nrhs, seed):
    from hybsol.b200 import meshgen

    mat, b = meshgen.mesh_system(n, p, seed=seed, nrhs=nrhs)
    order = native.compute_ordering(mat.row_ptr, mat.cols, "first")
    pm = mat.permuted(order)
    ns = native.NativeSystem.from_matrix(pm)
    ns.decompose(native.FP64)
    return ns, reorder_rhs(mat.sizes, order, b), pm


@pytest.mark.parametrize(("n", "p", "nrhs"), [(16, 4, 1), (8, 8, 3)])
def test_noalloc_solve_matches_hyb_solve_twice(gpu, n, p, nrhs):
    import torch

    from oracle import oracle as O

    solve_noalloc = _bind(gpu)
    ns, bn, pm = _factored(gpu, n, p, nrhs, seed=31)
    x_ref, _ = ns.solve(bn)
    osys = O.OracleSystem.from_csr(pm.sizes, pm.row_ptr, pm.cols, pm.vals)
    osys.decompose()
    x_oracle = osys.solve(bn)
    d_b = torch.from_numpy(np.ascontiguousarray(bn)).cuda()
    for _ in range(2):
        d_x = torch.full_like(d_b, float("nan"))
        st = solve_noalloc(ns._h, gpu._ptr(d_b), gpu._ptr(d_x), nrhs)
        assert st == 0, gpu.lib().hyb_last_cuda_error()
        x = d_x.cpu().numpy()
        assert np.array_equal(x, x_ref)
        assert rel_err(x, x_oracle) < 1e-12
    # in place (x aliasing b) gives the same result
    d_y = d_b.clone()
    assert solve_noalloc(ns._h, gpu._ptr(d_y), gpu._ptr(d_y), nrhs) == 0
    assert np.array_equal(d_y.cpu().numpy(), x_ref)


def test_noalloc_rejects_partial_overlap(gpu):
    import torch

    solve_noalloc = _bind(gpu)
    ns, bn, _ = _factored(gpu, 6, 4, 1, seed=7)
    buf = torch.zeros(2 * bn.shape[0], dtype=torch.float64, device="cuda")
    b = buf[: bn.shape[0]]
    x = buf[8 : 8 + bn.shape[0]]  # overlaps b but does not start at it
    assert solve_noalloc(ns._h, gpu._ptr(b), gpu._ptr(x), 1) == 16  # HYB_INVALID_ARGUMENT


def test_noalloc_rejects_oversized_and_unfactored(gpu):
    import torch

    solve_noalloc = _bind(gpu)
    ns, bn, _ = _factored(gpu, 8, 8, 1, seed=5)
    d_b = torch.from_numpy(bn).cuda()
    d_x = torch.empty_like(d_b)
    # scratch per stage = pivot rows x lower blocks x nrhs; 1024 right-hand sides of an
    # 8x8 p=8 mesh need more than the fixed 2^20 doubles
    big_b = torch.zeros((bn.shape[0], 1024), dtype=torch.float64, device="cuda")
    big_x = torch.empty_like(big_b)
    assert solve_noalloc(ns._h, gpu._ptr(big_b), gpu._ptr(big_x), 1024) == 24  # HYB_TOO_LARGE
    ns.set_values(np.zeros(ns.value_count))  # clears the factorization
    assert solve_noalloc(ns._h, gpu._ptr(d_b), gpu._ptr(d_x), 1) == 18  # HYB_NOT_DECOMPOSED
    ns.decompose(gpu.MIXED)
    assert solve_noalloc(ns._h, gpu._ptr(d_b), gpu._ptr(d_x), 1) == 18
