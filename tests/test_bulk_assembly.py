"""BlockSystem.add_blocks, the bulk form of add_block (host assembly, no GPU needed)."""

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
