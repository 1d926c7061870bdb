"""The oracle (C restatement in oracle/hyb_oracle.c) pinned against the reference.

The golden vectors in tests/golden/ were produced by the reference itself (compiled
from its own sources, see tests/golden/make_golden.py). The restatement must reproduce
them exactly: integer orders and patterns, and the factors and solutions bit for bit
(the restatement keeps the reference's arithmetic order and its no-FMA rounding).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O

STRATS = ("first", "greedy", "balanced")


@pytest.fixture(scope="module", autouse=True)
def _built():
    O.port_library()


def _mesh_oracle(g):
    sizes = g["sizes"]
    mat_rp, mat_cols = g["row_ptr"], g["cols"]
    return sizes, mat_rp, mat_cols


@pytest.mark.parametrize("name", ["mesh16_p4.npz", "mesh6_prand.npz"])
def test_orderings_match_reference(name):
    g = golden(name)
    for st in STRATS:
        got = O.compute_ordering(g["row_ptr"], g["cols"], st)
        assert np.array_equal(got.astype(np.int64), g[f"order_{st}"]), st


def _rebuild(name):
    """Regenerate the golden system (the generator is seeded) and factor it with the oracle."""
    from hybsol.b200 import meshgen

    g = golden(name)
    p = g["p"] if "p" in g.files else 4
    nrhs = g["x_new_layout"].shape[1]
    mat, _ = meshgen.mesh_system(int(g["n"]), p, seed=int(g["seed"]), nrhs=nrhs)
    assert np.array_equal(mat.row_ptr, g["row_ptr"]) and np.array_equal(mat.cols, g["cols"])
    o = O.OracleSystem.from_csr(mat.sizes, mat.row_ptr, mat.cols, mat.vals)
    o.reorder_blocks(g["order_first"].astype(np.uint64))
    o.decompose()
    return g, o


@pytest.mark.parametrize("name", ["mesh16_p4.npz", "mesh6_prand.npz"])
def test_mesh_factors_bitwise(name):
    g, o = _rebuild(name)
    rp, cols, vals = o.export()
    assert np.array_equal(rp.astype(np.int64), g["filled_row_ptr"])
    assert np.array_equal(cols.astype(np.int64), g["filled_cols"])
    ops = np.array([(x[0], x[1] if len(x) == 2 else -1) for x in o.operations()])
    assert np.array_equal(ops, g["ops"])
    sums, sq, full = [], [], []
    n = o.n_blocks
    full_rows, tail = int(g["full_rows"]), int(g["tail_rows"])
    for i in range(n):
        for c in o.get_row_block_indices(i):
            blk = o.get_block(i, c)
            sums.append(blk.sum())
            sq.append((blk * blk).sum())
            if i < full_rows or i >= n - tail:
                full.append(blk.ravel())
    assert np.array_equal(np.array(sums), g["block_sum"])
    assert np.array_equal(np.array(sq), g["block_sumsq"])
    assert np.array_equal(np.concatenate(full), g["full_values"])


@pytest.mark.parametrize("name", ["mesh16_p4.npz", "mesh6_prand.npz"])
def test_mesh_solution_bitwise(name):
    g, o = _rebuild(name)
    x = o.solve(g["rhs_new_layout"])
    assert np.array_equal(x, g["x_new_layout"])


def test_random_pattern_orderings():
    g = golden("random_orderings.npz")
    for k in range(int(g["count"])):
        for st in STRATS:
            got = O.compute_ordering(g[f"c{k}_row_ptr"], g[f"c{k}_cols"], st)
            assert np.array_equal(got.astype(np.int64), g[f"c{k}_order_{st}"]), (k, st)
            assert sorted(got.tolist()) == list(range(len(got)))


def test_max_colors_error():
    g = golden("random_orderings.npz")
    with pytest.raises(ValueError, match="Maximum number of colors"):
        O.compute_ordering(g["c2_row_ptr"], g["c2_cols"], "first", max_colors=1)


def test_dense_block_systems_bitwise():
    g = golden("dense_blocks.npz")
    for k in range(int(g["count"])):
        mat, bs = g[f"c{k}_matrix"], int(g[f"c{k}_bs"])
        nb = mat.shape[0] // bs
        o = O.OracleSystem([bs] * nb)
        for i in range(nb):
            for j in range(nb):
                o.add_block(i, j, mat[bs * i : bs * (i + 1), bs * j : bs * (j + 1)])
        o.decompose()
        _, _, vals = o.export()
        assert np.array_equal(vals, g[f"c{k}_factors"])
        assert np.array_equal(o.solve(g[f"c{k}_rhs"]), g[f"c{k}_x"])
        ops = np.array([(x[0], x[1] if len(x) == 2 else -1) for x in o.operations()])
        assert np.array_equal(ops, g[f"c{k}_ops"])


def test_dense_kernels_against_numpy():
    rng = np.random.default_rng(3)
    for m in (1, 2, 7, 33):
        a = rng.standard_normal((m, m)) + m * np.eye(m)
        lu = O.lu_decompose(a)
        low = np.tril(lu, -1) + np.eye(m)
        up = np.triu(lu)
        assert np.allclose(low @ up, a, rtol=1e-13, atol=1e-13)
        b = rng.standard_normal((m, 3))
        assert np.allclose(O.lu_solve(lu, b), np.linalg.solve(a, b), rtol=1e-10, atol=1e-12)


@pytest.mark.skipif(not O.reference_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_equals_reference_on_random_systems():
    """Direct restatement-vs-reference runs on unsymmetric and symmetric random patterns."""
    ref = O.load_reference()
    for seed in range(6):
        rng = np.random.default_rng(100 + seed)
        nb = int(rng.integers(5, 30))
        sizes = rng.integers(1, 6, nb)
        r = ref.BlockSystem(*[int(s) for s in sizes])
        o = O.OracleSystem(sizes)
        for i in range(nb):
            for j in range(nb):
                if i == j or rng.random() < 0.25:
                    v = rng.random((sizes[i], sizes[j])) + (nb * np.eye(sizes[i]) if i == j else 0)
                    r.add_block(i, j, v)
                    o.add_block(i, j, v)
        order = r.compute_reordering("first")
        assert np.array_equal(order, o.compute_reordering("first"))
        r.reorder_blocks(order)
        o.reorder_blocks(order)
        r.decompose(0)
        o.decompose()
        for i in range(nb):
            assert r.get_row_block_indices(i) == o.get_row_block_indices(i)
            for c in r.get_row_block_indices(i):
                assert np.array_equal(r.get_block(i, c), o.get_block(i, c))
        b = rng.random(int(sizes.sum()))
        assert np.array_equal(r.solve(b), o.solve(b))
