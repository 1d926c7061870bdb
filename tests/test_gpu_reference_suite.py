"""The reference's own test scenarios, run against this package on a B200.

Restates the scenarios of the reference's tests/test_decompose.py, tests/test_c_system.py
and tests/test_ordering.py (same seeds, sizes and checks) against `hybsol` here, with a
tighter tolerance where the reference used pytest.approx's default, plus a comparison of
every result with the oracle.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dense_system(n_blocks, block_size, seed=15):
    from hybsol import BlockSystem

    rng = np.random.default_rng(seed)
    mat = rng.random((n_blocks * block_size, n_blocks * block_size))
    assert abs(np.linalg.det(mat)) > 1e-3
    s = BlockSystem(*np.full(n_blocks, block_size, int))
    for i in range(n_blocks):
        for j in range(n_blocks):
            s.add_block(i, j, mat[block_size * i : block_size * (i + 1), block_size * j : block_size * (j + 1)])
    lhs = rng.random(n_blocks * block_size)
    return s, mat, lhs


@pytest.mark.parametrize("n", [2, 4, 10])
def test_dense_scalar_matrix(gpu, n):
    from hybsol.system import decompose_block_system_c, solve_decomposed_c

    s, mat, lhs = _dense_system(n, 1)
    assert np.array_equal(s.as_array(), mat)
    ops, dec = decompose_block_system_c(s)
    assert rel_err(solve_decomposed_c(dec, ops, mat @ lhs), lhs) < 1e-10


@pytest.mark.parametrize("n_blocks", [2, 4, 10])
@pytest.mark.parametrize("block_size", [2, 3, 4])
def test_python_driver_vs_decompose(gpu, n_blocks, block_size):
    """Python breadth-first driver vs BlockSystem.decompose: same pattern and factors."""
    from hybsol.system import decompose_block_system_c, solve_decomposed_c

    s, mat, lhs = _dense_system(n_blocks, block_size)
    s2, _, _ = _dense_system(n_blocks, block_size)
    rhs = mat @ lhs
    ops, dec = decompose_block_system_c(s)
    s2.decompose()
    for i in range(dec.n_blocks):
        cols = dec.get_row_block_indices(i)
        assert cols == s2.get_row_block_indices(i)
        for c in cols:
            assert rel_err(dec.get_block(i, c), s2.get_block(i, c)) < 1e-12
    sol = solve_decomposed_c(dec, ops, rhs)
    sol_c = s2.solve(rhs)
    assert rel_err(sol, sol_c) < 1e-12
    assert rel_err(sol, lhs) < 1e-10
    # and against the oracle (bit-identical to the reference)
    o = O.OracleSystem([block_size] * n_blocks)
    for i in range(n_blocks):
        for j in range(n_blocks):
            o.add_block(i, j, mat[block_size * i : block_size * (i + 1), block_size * j : block_size * (j + 1)])
    o.decompose()
    assert rel_err(sol_c, o.solve(rhs)) < 1e-12
    assert s2.operations() == o.operations()


def _filled(n_blocks, max_size, seed, density=None):
    from hybsol import BlockSystem

    rng = np.random.default_rng(seed)
    sizes = rng.integers(1, max_size, n_blocks) if max_size != 1 else np.ones(n_blocks, dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(sizes)])
    full = rng.random((sizes.sum(), sizes.sum()))
    s = BlockSystem(*sizes)
    for i in range(n_blocks):
        for j in rng.permutation(n_blocks):
            if density is None or i == j or rng.random(1) < density:
                s.add_block(i, int(j), full[off[i] : off[i + 1], off[j] : off[j + 1]])
            else:
                full[off[i] : off[i + 1], off[j] : off[j + 1]] = 0
    return s, full, off, rng


@pytest.mark.parametrize("n_blocks", [1, 2, 4, 10])
@pytest.mark.parametrize("max_size", [1, 2, 4, 10])
def test_multiply_row(gpu, n_blocks, max_size):
    s, full, off, rng = _filled(n_blocks, max_size, 21)
    for i in range(n_blocks):
        inv = np.linalg.inv(s.get_block(i, i))
        s.multiply_row(i, inv)
        for j in rng.permutation(n_blocks):
            val = full[off[i] : off[i + 1], off[j] : off[j + 1]]
            assert np.allclose(s.get_block(i, int(j)), inv @ val, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("n_blocks", [1, 2, 4, 10])
@pytest.mark.parametrize("max_size", [1, 2, 4, 10])
def test_eliminate_row_dense(gpu, n_blocks, max_size):
    s, full, off, rng = _filled(n_blocks, max_size, 21)
    perm = rng.permutation(n_blocks)
    for src, tgt in zip(perm[0::2], perm[1::2]):
        mat = s.get_block(int(tgt), int(src))
        s.eliminate_row(int(src), int(tgt), mat)
        for i in range(int(src) + 1, n_blocks):
            expected = full[off[tgt] : off[tgt + 1], off[i] : off[i + 1]] - mat @ s.get_block(int(src), i)
            assert np.allclose(s.get_block(int(tgt), i), expected, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("n_blocks", [10, 25])
@pytest.mark.parametrize("max_size", [1, 4, 10])
@pytest.mark.parametrize("density", [0.1, 0.5, 0.9])
def test_eliminate_row_sparse(gpu, n_blocks, max_size, density):
    """Sparse elimination with fill, compared block for block with the oracle."""
    s, full, off, rng = _filled(n_blocks, max_size, 21, density)
    sizes = np.diff(off)
    o = O.OracleSystem(sizes)
    for i in range(n_blocks):
        for j in s.get_row_block_indices(i):
            o.add_block(i, j, s.get_block(i, j))
    perm = rng.permutation(n_blocks)
    for src, tgt in zip(perm[0::2], perm[1::2]):
        src, tgt = int(src), int(tgt)
        if not s.has_block(tgt, src):
            continue
        mat = s.get_block(tgt, src)
        s.eliminate_row(src, tgt, mat)
        o.eliminate_row(src, tgt, mat)
        assert s.get_row_block_indices(tgt) == o.get_row_block_indices(tgt)
        for c in s.get_row_block_indices(tgt):
            assert rel_err(s.get_block(tgt, c), o.get_block(tgt, c)) < 1e-12


@pytest.mark.parametrize(("n", "m"), [(2, 2), (3, 3), (10, 15)])
def test_diagonal_inverse(gpu, n, m):
    from hybsol import BlockSystem

    rng = np.random.default_rng(n * m)
    mat = rng.random((n, n))
    lhs = rng.random((n, m))
    out = np.empty_like(lhs)
    s = BlockSystem(n)
    s.add_block(0, 0, mat)
    s.decompose_diagonal(idx=0)
    s.solve_diagonal(out=out, idx=0, val=mat @ lhs)
    assert rel_err(out, lhs) < 1e-10


def test_decompose_then_accessors(gpu):
    """After decompose(): mutators raise, accessors read the device factors, copy works."""
    s, mat, lhs = _dense_system(4, 3)
    s.decompose()
    assert s.precision == "fp64"
    with pytest.raises(RuntimeError, match="already been decomposed"):
        s.add_block(0, 0, np.eye(3))
    with pytest.raises(RuntimeError, match="already been decomposed"):
        s.decompose()
    c = s.copy()
    x = s.solve(mat @ lhs)
    assert rel_err(c.solve(mat @ lhs), x) == 0.0
    out = np.empty(12)
    assert s.solve(mat @ lhs, out=out) is out
    y = mat @ lhs
    assert s.solve(y, out=y) is y and rel_err(y, lhs) < 1e-10
    X = s.solve(np.stack([mat @ lhs, 2 * (mat @ lhs)], axis=1))
    assert rel_err(X[:, 1], 2 * lhs) < 1e-10
    info = s.last_decompose_info()
    assert info["zero_pivots"] == 0 and info["filled_blocks"] == 16
    assert s.as_array().shape == (12, 12)


def test_mixed_precision_through_extension(gpu):
    s, mat, lhs = _dense_system(10, 4)
    s.decompose(precision="mixed")
    x = s.solve(mat @ lhs)
    info = s.last_solve_info()
    assert info["converged"] and info["relative_residual"] <= 1e-12
    assert rel_err(x, lhs) < 1e-9


@pytest.mark.parametrize("strat", ["first", "greedy", "balanced"])
@pytest.mark.parametrize(("nb", "bs", "sp"), [(10, 5, 0.3), (15, 5, 0.9), (200, 2, 0.8)])
def test_reorder_then_solve(gpu, strat, nb, bs, sp):
    """Coloring order -> reorder_blocks -> decompose -> solve in the original numbering."""
    from hybsol import BlockSystem

    rng = np.random.default_rng(1359)
    sizes = rng.integers(1, bs, nb)
    s = BlockSystem(*sizes)
    blocks = {}
    for ir in range(nb):
        blocks[(ir, ir)] = rng.random((sizes[ir], sizes[ir])) + 0.1 + nb * np.eye(sizes[ir])
        for ic in range(ir + 1, nb):
            if sp > rng.random(1):
                continue
            blocks[(ir, ic)] = rng.random((sizes[ir], sizes[ic]))
            blocks[(ic, ir)] = rng.random((sizes[ic], sizes[ir]))
    for (r, c), v in blocks.items():
        s.add_block(r, c, v)
    a = s.as_array()
    order = s.compute_reordering(strat)
    assert np.all(np.unique(order) == np.arange(nb))
    s.reorder_blocks(order)
    s.decompose()
    b = rng.random(a.shape[0])
    x = s.reorder_vector(order, s.solve(s.unorder_vector(order, b)))
    assert np.linalg.norm(a @ x - b) / np.linalg.norm(b) < 1e-13
