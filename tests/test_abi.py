"""The C-ABI library and the `hybsol._mod` extension, without a GPU.

Checks that libhybsol_b200.so loads and exports every entry point include/hybsol_b200.h
declares (no compute calls), and the extension's host-side behaviour that needs no
device: construction, assembly, accessors, reordering, vector permutations and the
reference's error messages. Comparisons are against the oracle.
"""

from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as O

HEADER = ROOT / "include" / "hybsol_b200.h"

REFERENCE_METHODS = [
    "add_block", "is_valid", "as_array", "get_row_block_indices", "get_block", "get_block_size",
    "multiply_row", "eliminate_row", "has_block", "no_lower_connections", "first_column",
    "get_next_column_index", "decompose_diagonal", "solve_diagonal", "row_apply_decomposition",
    "decompose", "operations", "solve", "copy", "reorder_blocks", "compute_reordering",
    "reorder_vector", "unorder_vector",
]  # fmt: skip


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"HYB_API[^;(]*?\b(hyb_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native):
    lib = ctypes.CDLL(str(native.LIB_PATH))
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) >= set(native.EXPORTS)


def test_status_strings(native):
    lib = native.lib()
    assert lib.hyb_status_string(0) == b"success"
    assert lib.hyb_status_string(3) == b"maximum number of colors exceeded"
    assert lib.hyb_version() >= 100


def test_no_device_paths_fail_loudly(native):
    if native.device_available():
        pytest.skip("a GPU is visible: the no-device error path is not reachable")
    with pytest.raises(native.HybError, match="no sm_100"):
        native.NativeSystem([2], [0, 1], [0])
    from hybsol import BlockSystem

    s = BlockSystem(2)
    s.add_block(0, 0, np.eye(2))
    with pytest.raises(RuntimeError, match="decomposition failed with error 20"):
        s.decompose()


def test_extension_surface():
    import hybsol
    from hybsol import system
    from hybsol._mod import BlockInfo, BlockSystem

    assert hybsol.BlockSystem is BlockSystem
    for m in REFERENCE_METHODS:
        assert callable(getattr(BlockSystem, m)), m
    assert BlockSystem.__module__ == "hybsol._mod"
    for name in ("OperationInvDiag", "OperationEliminate", "TargetRow", "decompose_block_system_c", "solve_decomposed_c"):
        assert hasattr(system, name)
    b = BlockInfo(1, 2, np.arange(6.0).reshape(2, 3))
    assert (b.row, b.col, b.shape) == (1, 2, (2, 3))
    assert np.array_equal(b.value, np.arange(6.0).reshape(2, 3))


def _fill_random(rng, sizes, density=1.0):
    from hybsol import BlockSystem

    off = np.concatenate([[0], np.cumsum(sizes)])
    full = rng.random((off[-1], off[-1]))
    s = BlockSystem(*sizes)
    o = O.OracleSystem(sizes)
    for i in range(len(sizes)):
        for j in rng.permutation(len(sizes)):
            blk = full[off[i] : off[i + 1], off[j] : off[j + 1]]
            if i == j or rng.random() < density:
                s.add_block(i, int(j), blk)
                o.add_block(i, int(j), blk)
            else:
                full[off[i] : off[i + 1], off[j] : off[j + 1]] = 0
    return s, o, full, off


@pytest.mark.parametrize("n_blocks", [1, 2, 4, 10])
@pytest.mark.parametrize("max_size", [1, 2, 4, 10])
def test_as_array_and_merge(n_blocks, max_size):
    """Assembly round trip and duplicate-add summation (the reference's as_array test)."""
    rng = np.random.default_rng(67)
    sizes = rng.integers(1, max_size, n_blocks) if max_size != 1 else np.ones(n_blocks, dtype=np.int64)
    s, _, full, off = _fill_random(rng, sizes)
    assert np.array_equal(s.as_array(), full)
    second = rng.random(full.shape)
    for i in range(n_blocks):
        for j in rng.permutation(n_blocks):
            s.add_block(i, int(j), second[off[i] : off[i + 1], off[j] : off[j + 1]])
    assert np.array_equal(s.as_array(), full + second)
    for i in range(n_blocks):
        for j in range(n_blocks):
            assert s.get_block_size(i, j) == (int(sizes[i]), int(sizes[j]))
            assert np.array_equal(s.get_block(i, j), (full + second)[off[i] : off[i + 1], off[j] : off[j + 1]])


@pytest.mark.parametrize("density", [0.1, 0.5, 0.9])
def test_sparse_accessors_match_oracle(density):
    rng = np.random.default_rng(21)
    sizes = rng.integers(1, 5, 25)
    s, o, full, _ = _fill_random(rng, sizes, density)
    assert np.array_equal(s.as_array(), full)
    for i in range(25):
        assert s.get_row_block_indices(i) == o.get_row_block_indices(i)
        cols = o.get_row_block_indices(i)
        assert s.first_column(i) == cols[0]
        for c in range(25):
            assert s.has_block(i, c) == (c in cols)
        nxt = [c for c in cols if c > i]
        if nxt:
            assert s.get_next_column_index(i, i) == nxt[0]
    nl = s.no_lower_connections()
    assert nl.dtype == np.bool_ and nl.tolist() == [o.get_row_block_indices(i)[0] >= i for i in range(25)]
    cpy = s.copy()
    assert np.array_equal(cpy.as_array(), s.as_array())
    for st in ("first", "greedy", "balanced"):
        assert np.array_equal(s.compute_reordering(st), o.compute_reordering(st))


@pytest.mark.parametrize(("nb", "bs"), [(10, 4), (40, 5), (200, 10)])
def test_reorder_and_vectors(nb, bs):
    """reorder_blocks + reorder_vector/unorder_vector (the reference's ordering tests)."""
    from hybsol import BlockSystem

    rng = np.random.default_rng(2)
    sizes = rng.integers(1, bs, nb)
    s = BlockSystem(*sizes)
    o = O.OracleSystem(sizes)
    for ir in range(nb):
        s.add_block(ir, ir, np.full((sizes[ir], sizes[ir]), float(ir)))
        o.add_block(ir, ir, np.full((sizes[ir], sizes[ir]), float(ir)))
        for ic in range(ir + 1, nb):
            if rng.random() < 0.9:
                continue
            for a, b in ((ir, ic), (ic, ir)):
                v = rng.random((sizes[a], sizes[b]))
                s.add_block(a, b, v)
                o.add_block(a, b, v)
    order = rng.permuted(np.arange(nb, dtype=np.uint64))
    s.reorder_blocks(order)
    o.reorder_blocks(order)
    assert np.array_equal(s.block_sizes, o.block_sizes)
    assert np.array_equal(s.as_array(), np.array(_dense(o)))
    original = np.concatenate([np.full(s.block_sizes[i], i) for i in range(nb)]).astype(np.float64)
    expected = np.concatenate([np.full(s.block_sizes[order[i]], order[i]) for i in range(nb)]).astype(np.float64)
    assert np.array_equal(s.reorder_vector(order, original), expected)
    assert np.array_equal(s.unorder_vector(order, s.reorder_vector(order, original)), original)
    out = np.empty_like(original)
    assert s.reorder_vector(order, original, out=out) is out


def _dense(o):
    off = np.concatenate([[0], np.cumsum(o.block_sizes.astype(np.int64))])
    a = np.zeros((off[-1], off[-1]))
    for i in range(o.n_blocks):
        for c in o.get_row_block_indices(i):
            a[off[i] : off[i + 1], off[c] : off[c + 1]] = o.get_block(i, c)
    return a


def test_reference_error_messages():
    from hybsol import BlockSystem

    with pytest.raises(ValueError, match="at least one block"):
        BlockSystem()
    with pytest.raises(ValueError, match="Block size of block 1 is 0"):
        BlockSystem(2, 0)
    with pytest.raises(TypeError, match="no keyword arguments"):
        BlockSystem(2, x=1)
    s = BlockSystem(2, 3)
    with pytest.raises(ValueError, match=r"Row index must be in the range \[0, 2\), but it was 2"):
        s.add_block(2, 0, np.eye(2))
    with pytest.raises(ValueError):
        s.add_block(0, 0, np.eye(3))
    s.add_block(0, 0, np.eye(2))
    with pytest.raises(ValueError, match=r"does not contain the block \(1, 0\)"):
        s.get_block(1, 0)
    with pytest.raises(ValueError, match="Row has no entries"):
        s.first_column(1)
    with pytest.raises(ValueError, match="no entries after column"):
        s.get_next_column_index(0, 0)
    with pytest.raises(RuntimeError, match="not been decomposed"):
        s.solve(np.zeros(5))
    with pytest.raises(RuntimeError, match="not been decomposed"):
        s.operations()
    with pytest.raises(TypeError, match="Ordering strategy must be a string"):
        s.compute_reordering(1)
    with pytest.raises(ValueError, match="Unknown ordering strategy 'x'"):
        s.compute_reordering("x")
    with pytest.raises(ValueError, match="must be non-negative"):
        s.compute_reordering(max_colors=-1)
    with pytest.raises(ValueError, match="Duplicate order index 0"):
        s.reorder_blocks(np.array([0, 0], dtype=np.uint64))
    with pytest.raises(ValueError, match="Number of threads must be non-negative"):
        s.decompose(-1)
    with pytest.raises(TypeError, match="takes no arguments"):
        s.is_valid(1)
    with pytest.raises(ValueError, match="square matrix of size 2"):
        s.multiply_row(0, np.eye(3))
    with pytest.raises(ValueError, match="has no diagonal entry"):
        s.decompose_diagonal(1)
    assert s.precision is None


def test_is_valid_semantics():
    """The reference checks only the blocks left of each diagonal for a partner."""
    from hybsol import BlockSystem

    s = BlockSystem(1, 1)
    s.add_block(0, 0, [[1.0]])
    s.add_block(1, 1, [[1.0]])
    s.add_block(0, 1, [[1.0]])
    assert s.is_valid()
    s.add_block(1, 0, [[1.0]])
    assert s.is_valid()
    t = BlockSystem(1, 1)
    t.add_block(1, 1, [[1.0]])
    t.add_block(1, 0, [[1.0]])
    t.add_block(0, 0, [[1.0]])
    assert not t.is_valid()
