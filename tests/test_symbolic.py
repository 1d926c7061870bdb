"""The product's host-side integer work, bit-exact with the reference (no GPU needed).

* coloring orders (hyb_compute_ordering) against the reference's golden orders;
* the symbolic phase (hyb_analyze): the filled pattern the reference's elimination
  creates and its single-thread operation order, against the golden vectors and the
  oracle on patterns the golden set does not cover (unsymmetric, ragged, dense).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O

STRATS = ("first", "greedy", "balanced")


@pytest.mark.parametrize("name", ["mesh16_p4.npz", "mesh6_prand.npz"])
def test_orderings_and_fill_match_reference(native, name):
    g = golden(name)
    for st in STRATS:
        got = native.compute_ordering(g["row_ptr"], g["cols"], st)
        assert np.array_equal(got.astype(np.int64), g[f"order_{st}"]), st
    from hybsol.b200 import meshgen

    p = g["p"] if "p" in g.files else 4
    mat, _ = meshgen.mesh_system(int(g["n"]), p, seed=int(g["seed"]))
    pm = mat.permuted(g["order_first"])
    a = native.analyze(pm.sizes, pm.row_ptr, pm.cols, pattern=True, operations=True)
    assert np.array_equal(a["filled_row_ptr"].astype(np.int64), g["filled_row_ptr"])
    assert np.array_equal(a["filled_cols"].astype(np.int64), g["filled_cols"])
    assert np.array_equal(a["ops"], g["ops"])
    assert a["filled_blocks"] == len(g["filled_cols"])


@pytest.mark.parametrize(("n", "p", "pairs"), [(8, 8, 31), (12, 8, 71), (24, 8, 287), (16, 4, 0), (6, "rand", 0)])
def test_two_pivot_pairs(native, n, p, pairs):
    """Consecutive single-pivot levels of 64-blocks pair up for the mixed form's two-pivot
    update passes: on an n x n p=8 mesh the n*n element levels form n*n/2 - 1 pairs (the
    last element has no lower or upper blocks to share); blocks of other sizes never pair."""
    from hybsol.b200 import meshgen

    pp = meshgen.random_orders(n, 2, 10, seed=3) if p == "rand" else p
    mat, _ = meshgen.mesh_system(n, pp, seed=0)
    order = native.compute_ordering(mat.row_ptr, mat.cols, "first")
    pm = mat.permuted(order)
    a = native.analyze(pm.sizes, pm.row_ptr, pm.cols)
    assert a["pair_levels"] == pairs
    assert 2 * a["pair_levels"] <= a["n_levels"]


def _banded_pattern(n, seed):
    """Random unsymmetric banded pattern of 64x64 blocks (half bandwidth 3), diagonal set."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        cs = {i} | {j for j in range(max(0, i - 3), min(n, i + 4)) if j != i and rng.random() < 0.55}
        rows.append(sorted(cs))
    row_ptr = np.cumsum([0] + [len(r) for r in rows]).astype(np.uint64)
    cols = np.array([c for r in rows for c in r], dtype=np.uint64)
    return np.full(n, 64, dtype=np.uint64), row_ptr, cols


def _restated_pairs(n, frp, fcols):
    """The pairing rule, restated on the filled pattern: levels l, l+1 (one pivot each, a
    then b, greedily from the first level) pair when b has lower and upper blocks, b lies in
    a's lower column and upper row, and a's other lower rows / upper columns are b's too."""
    filled = [set(fcols[frp[i] : frp[i + 1]].tolist()) for i in range(n)]
    lower = [{t for t in range(k + 1, n) if k in filled[t]} for k in range(n)]
    upper = [{c for c in filled[k] if c > k} for k in range(n)]
    level = [0] * n
    for k in range(n):
        deps = [j for j in range(k) if j in filled[k] or k in filled[j]]
        level[k] = 1 + max(level[j] for j in deps) if deps else 0
    piv = [[k for k in range(n) if level[k] == lv] for lv in range(max(level) + 1)]
    pairs, lv = 0, 0
    while lv + 1 < len(piv):
        if len(piv[lv]) == 1 and len(piv[lv + 1]) == 1:
            a, b = piv[lv][0], piv[lv + 1][0]
            ra, ca, rb, cb = lower[a], upper[a], lower[b], upper[b]
            if rb and cb and b in ra and b in ca and ra - {b} <= rb and ca - {b} <= cb:
                pairs += 1
                lv += 2
                continue
        lv += 1
    return pairs


@pytest.mark.parametrize("seed", range(8))
def test_pairs_match_restated_rule(native, seed):
    """The symbolic phase's pairs of levels (two-pivot passes) on random banded patterns
    agree with the pairing rule restated on the filled pattern."""
    n = 24 + seed
    sizes, row_ptr, cols = _banded_pattern(n, seed)
    a = native.analyze(sizes, row_ptr, cols, pattern=True)
    frp = a["filled_row_ptr"].astype(np.int64)
    fc = a["filled_cols"].astype(np.int64)
    assert a["pair_levels"] == _restated_pairs(n, frp, fc)


def test_mesh16_work_counts(native):
    """Exact algorithmic counts of the 16x16 p=4 system (10,558 blocks after fill, 0.531 GFLOP)."""
    g = golden("mesh16_p4.npz")
    from hybsol.b200 import meshgen

    mat, _ = meshgen.mesh_system(16, 4, seed=0)
    pm = mat.permuted(g["order_first"])
    a = native.analyze(pm.sizes, pm.row_ptr, pm.cols)
    assert a["filled_blocks"] == 10558
    assert a["nops"] == len(g["ops"])
    assert abs(a["factor_flops"] / 1e9 - 0.5311542613) < 1e-8
    # edges (one parallel stage) then the 256 elements, one per stage
    assert a["n_levels"] == 257


def test_random_orderings_match_reference(native):
    g = golden("random_orderings.npz")
    for k in range(int(g["count"])):
        for st in STRATS:
            got = native.compute_ordering(g[f"c{k}_row_ptr"], g[f"c{k}_cols"], st)
            assert np.array_equal(got.astype(np.int64), g[f"c{k}_order_{st}"]), (k, st)
        with pytest.raises(ValueError, match="Maximum number of colors"):
            native.compute_ordering(g[f"c{k}_row_ptr"], g[f"c{k}_cols"], "first", max_colors=1)


def _random_pattern(rng, nb, density, symmetric):
    rows = []
    for i in range(nb):
        cols = {i}
        for j in range(nb):
            if j != i and rng.random() < density:
                cols.add(j)
        rows.append(cols)
    if symmetric:
        for i in range(nb):
            for j in list(rows[i]):
                rows[j].add(i)
    row_ptr = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.uint64)
    cols = np.concatenate([sorted(r) for r in rows]).astype(np.uint64)
    return row_ptr, cols


@pytest.mark.parametrize("symmetric", [True, False])
@pytest.mark.parametrize("seed", range(8))
def test_fill_and_ops_match_oracle(native, seed, symmetric):
    rng = np.random.default_rng(seed)
    nb = int(rng.integers(2, 60))
    sizes = rng.integers(1, 5, nb).astype(np.uint64)
    row_ptr, cols = _random_pattern(rng, nb, float(rng.uniform(0.02, 0.4)), symmetric)
    for st in STRATS:
        assert np.array_equal(
            native.compute_ordering(row_ptr, cols, st), O.compute_ordering(row_ptr, cols, st)
        ), st
    o = O.OracleSystem(sizes)
    for i in range(nb):
        for j in cols[row_ptr[i] : row_ptr[i + 1]]:
            v = rng.random((int(sizes[i]), int(sizes[j]))) + (nb * np.eye(int(sizes[i])) if i == j else 0)
            o.add_block(i, int(j), v)
    o.decompose()
    frp, fcols, _ = o.export()
    a = native.analyze(sizes, row_ptr, cols, pattern=True, operations=True)
    assert np.array_equal(a["filled_row_ptr"], frp)
    assert np.array_equal(a["filled_cols"], fcols)
    ops = np.array([(x[0], x[1] if len(x) == 2 else -1) for x in o.operations()])
    assert np.array_equal(a["ops"], ops)


def test_single_block_and_dense(native):
    a = native.analyze([5], [0, 1], [0], pattern=True, operations=True)
    assert a["filled_blocks"] == 1 and a["n_levels"] == 1
    assert a["ops"].tolist() == [[0, -1]]
    nb = 6
    rp = np.arange(0, nb * nb + 1, nb)
    cc = np.tile(np.arange(nb), nb)
    a = native.analyze([3] * nb, rp, cc, operations=True)
    assert a["filled_blocks"] == nb * nb
    assert a["n_levels"] == nb  # a dense system is a chain


def test_bad_patterns_are_rejected(native):
    with pytest.raises(native.HybError, match="no diagonal"):
        native.analyze([2, 2], [0, 1, 2], [1, 0])
    with pytest.raises(native.HybError, match="invalid argument"):
        native.analyze([2, 2], [0, 2, 3], [1, 0, 1])  # unsorted row
    with pytest.raises(native.HybError, match="invalid argument"):
        native.analyze([2, 0], [0, 1, 2], [0, 1])  # zero block size
