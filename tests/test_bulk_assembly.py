"""Bulk assembly: BlockSystem.add_blocks (host rows, no GPU needed) and the device path
hyb_system_add_blocks of a handle, plus the batched block products and solves the
extension's row operations use (GPU)."""

from __future__ import annotations

import numpy as np
import pytest


def _coo(mat):
    rows = np.repeat(np.arange(mat.n_blocks), np.diff(mat.row_ptr))
    return rows, np.asarray(mat.cols), np.asarray(mat.vals)


def test_add_blocks_matches_add_block():
    from hybsol import BlockSystem
    from hybsol.b200 import meshgen

    mat, _ = meshgen.mesh_system(4, meshgen.random_orders(4, 2, 5, seed=2), seed=9)
    a = BlockSystem(*[int(x) for x in mat.sizes])
    for r, c, v in mat.iter_blocks():
        a.add_block(r, c, v)
    b = BlockSystem(*[int(x) for x in mat.sizes])
    rows, cols, vals = _coo(mat)
    b.add_blocks(rows, cols, vals)
    assert np.array_equal(a.as_array(), b.as_array())
    for i in range(mat.n_blocks):
        assert a.get_row_block_indices(i) == b.get_row_block_indices(i)


def test_add_blocks_sums_repeats_in_order():
    from hybsol import BlockSystem

    s = BlockSystem(2, 1, 3)
    rng = np.random.default_rng(0)
    blocks = [(0, 0, rng.random((2, 2))), (2, 0, rng.random((3, 2))), (0, 0, rng.random((2, 2))), (1, 2, rng.random((1, 3)))]
    ref = BlockSystem(2, 1, 3)
    for r, c, v in blocks:
        ref.add_block(r, c, v)
    s.add_blocks([r for r, _, _ in blocks], [c for _, c, _ in blocks], np.concatenate([v.ravel() for _, _, v in blocks]))
    assert np.array_equal(s.as_array(), ref.as_array())
    s.add_blocks(np.array([], dtype=np.int64), np.array([], dtype=np.int64), np.array([]))  # nothing to add
    assert np.array_equal(s.as_array(), ref.as_array())


def test_add_blocks_checks_before_adding():
    from hybsol import BlockSystem

    s = BlockSystem(2, 2)
    s.add_block(0, 0, np.eye(2))
    before = s.as_array()
    with pytest.raises(ValueError, match="Row index"):
        s.add_blocks([0, 5], [0, 0], np.ones(8))
    with pytest.raises(ValueError, match="values has"):
        s.add_blocks([0, 1], [0, 1], np.ones(7))
    with pytest.raises(ValueError, match="entries"):
        s.add_blocks([0, 1], [0], np.ones(8))
    with pytest.raises(ValueError, match="integers"):
        s.add_blocks([0.5], [0], np.ones(4))
    assert np.array_equal(s.as_array(), before)
    s.add_blocks(rows=[1], cols=[1], values=np.arange(4.0))
    assert np.array_equal(s.get_block(1, 1), np.arange(4.0).reshape(2, 2))


def _pattern_system(native):
    from hybsol.b200 import meshgen

    mat, _ = meshgen.mesh_system(5, 3, seed=12)
    pm = mat.permuted(native.compute_ordering(mat.row_ptr, mat.cols, "first"))
    return pm


@pytest.mark.gpu
@pytest.mark.parametrize("device", [False, True])
def test_device_add_blocks_sums_in_input_order(gpu, device):
    """hyb_system_add_blocks: every block of the pattern given in pieces, some blocks twice,
    in shuffled order; the device sums repeats in input order (as repeated add_block calls),
    and the result factors and solves exactly as the same values loaded whole."""
    import torch

    pm = _pattern_system(gpu)
    rng = np.random.default_rng(3)
    rows_of = np.repeat(np.arange(pm.n_blocks), np.diff(pm.row_ptr))
    blocks = list(range(pm.nnz_blocks))
    picks = blocks + list(rng.choice(blocks, size=len(blocks) // 3, replace=False))
    rng.shuffle(picks)
    pieces, expect = [], np.zeros_like(pm.vals)
    for j in picks:
        v = rng.standard_normal(pm.val_ptr[j + 1] - pm.val_ptr[j])
        pieces.append(v)
        expect[pm.val_ptr[j] : pm.val_ptr[j + 1]] += v  # input order, as add_block
    rows = rows_of[picks]
    cols = pm.cols[picks]
    vals = np.concatenate(pieces)
    ns = gpu.NativeSystem(pm.sizes, pm.row_ptr, pm.cols)
    ns.add_blocks(rows, cols, torch.from_numpy(vals).cuda() if device else vals, device=device)
    for j in range(pm.nnz_blocks):
        r, c = int(rows_of[j]), int(pm.cols[j])
        got = ns.get_block(r, c, (int(pm.sizes[r]), int(pm.sizes[c])))
        assert np.array_equal(got.ravel(), expect[pm.val_ptr[j] : pm.val_ptr[j + 1]])
    ref = gpu.NativeSystem(pm.sizes, pm.row_ptr, pm.cols)
    ref.set_values(expect)
    b = rng.uniform(-1, 1, pm.dof)
    for s_ in (ns, ref):
        s_.decompose(gpu.FP64)
    assert np.array_equal(ns.solve(b)[0], ref.solve(b)[0])


@pytest.mark.gpu
def test_device_add_blocks_rejects_blocks_outside_the_pattern(gpu):
    pm = _pattern_system(gpu)
    ns = gpu.NativeSystem.from_matrix(pm)
    outside = next((r, c) for r in range(pm.n_blocks) for c in range(pm.n_blocks)
                   if c not in set(pm.cols[pm.row_ptr[r] : pm.row_ptr[r + 1]]))
    r0, c0 = 0, int(pm.cols[0])
    vals = np.ones(int(pm.sizes[r0] * pm.sizes[c0]) + int(pm.sizes[outside[0]] * pm.sizes[outside[1]]))
    before = ns.get_block(r0, c0, (int(pm.sizes[r0]), int(pm.sizes[c0])))
    with pytest.raises(KeyError):
        ns.add_blocks([r0, outside[0]], [c0, outside[1]], vals)
    assert np.array_equal(ns.get_block(r0, c0, before.shape), before)  # nothing was added


@pytest.mark.gpu
def test_batched_block_calls_match_numpy(gpu):
    import ctypes

    lib = gpu.lib()
    rng = np.random.default_rng(4)
    m, k = 7, 5
    a = rng.standard_normal((m, k))
    ns_ = [3, 9, 1, 64, 70]
    bs = [rng.standard_normal((k, n)) for n in ns_]
    cs = [rng.standard_normal((m, n)) for n in ns_]
    want = [c - a @ b for c, b in zip(cs, bs)]
    P = ctypes.c_void_p
    n_arr = np.asarray(ns_, dtype=np.uint64)
    st = lib.hyb_block_gemm_batched(len(ns_), m, k, n_arr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                    a.ctypes.data, (P * len(bs))(*[b.ctypes.data for b in bs]),
                                    (P * len(cs))(*[c.ctypes.data for c in cs]), 1, 0)
    assert st == 0
    for c, w in zip(cs, want):
        assert np.abs(c - w).max() <= 1e-13 * max(1.0, np.abs(w).max())
    d = rng.standard_normal((m, m)) + 8 * np.eye(m)
    lu = gpu.block_lu(d)
    rhs = [rng.standard_normal((m, n)) for n in ns_]
    want = [np.linalg.solve(d, r) for r in rhs]
    st = lib.hyb_block_lu_solve_batched(m, lu.ctypes.data, len(rhs), n_arr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                        (P * len(rhs))(*[r.ctypes.data for r in rhs]), 0)
    assert st == 0
    for r, w in zip(rhs, want):
        assert np.abs(r - w).max() <= 1e-12 * np.abs(w).max()
