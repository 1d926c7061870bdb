"""Independent systems batched into one handle (hybsol.b200.batch).

CPU: the host layout -- the stacked system ordered with the reference's coloring keeps each
system's own relative order, and vectors moved in and out through the layout give, with the
oracle solving the stacked system, each system's own solution. GPU: the device path against
one handle per system.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err, reorder_rhs
from oracle import oracle as O

SPECS = [(3, 3), (5, 4), (4, 6), (2, 5), (3, 8)]


def _systems(nrhs=1):
    from hybsol.b200 import meshgen

    mats, rhs = [], []
    for k, (side, p) in enumerate(SPECS):
        m, b = meshgen.mesh_system(side, p, seed=40 + k, nrhs=nrhs)
        mats.append(m)
        rhs.append(b)
    return mats, rhs


def test_dof_permutation_matches_block_moves(native):
    from hybsol.b200 import batch

    rng = np.random.default_rng(3)
    sizes = rng.integers(1, 7, 23)
    order = rng.permutation(23)
    b = rng.standard_normal(int(sizes.sum()))
    p = batch.dof_permutation(sizes, order)
    moved = np.empty_like(b)
    moved[p] = b
    assert np.array_equal(moved, reorder_rhs(sizes, order, b))
    assert np.array_equal(np.sort(p), np.arange(len(b)))


@pytest.mark.parametrize("strategy", ["first", "greedy", "balanced"])
def test_layout_keeps_each_system_order(native, strategy):
    from hybsol.b200 import batch

    mats, _ = _systems()
    lay = batch.BatchLayout(mats, strategy)
    for i, m in enumerate(mats):
        own = native.compute_ordering(m.row_ptr, m.cols, strategy).astype(np.int64)
        sub = lay.order[lay.block_off[i] : lay.block_off[i + 1]] - lay.block_off[i]
        assert np.array_equal(sub, own)
        # the stacked system's diagonal block range of system i is system i reordered alone
        pm = m.permuted(own)
        b0, b1 = lay.block_off[i], lay.block_off[i + 1]
        assert np.array_equal(lay.matrix.sizes[b0:b1], pm.sizes)


@pytest.mark.parametrize("nrhs", [1, 2])
def test_layout_round_trip_with_oracle(native, nrhs):
    from hybsol.b200 import batch

    mats, rhs = _systems(nrhs)
    lay = batch.BatchLayout(mats)
    big = O.OracleSystem.from_csr(lay.matrix.sizes, lay.matrix.row_ptr, lay.matrix.cols, lay.matrix.vals)
    big.decompose()
    parts = lay.from_solver(big.solve(lay.to_solver(rhs)))
    for m, b, x in zip(mats, rhs, parts):
        order = native.compute_ordering(m.row_ptr, m.cols, "first").astype(np.int64)
        pm = m.permuted(order)
        alone = O.OracleSystem.from_csr(pm.sizes, pm.row_ptr, pm.cols, pm.vals)
        alone.decompose()
        xs = alone.solve(reorder_rhs(m.sizes, order, b))
        inv = np.argsort(order)
        assert rel_err(x, reorder_rhs(pm.sizes, inv, xs)) < 1e-13
        assert rel_err(m.matvec(x), b) < 1e-12


def test_layout_rejects_mismatches(native):
    from hybsol.b200 import batch, meshgen

    mats, rhs = _systems()
    lay = batch.BatchLayout(mats)
    with pytest.raises(ValueError):
        lay.to_solver(rhs[:-1])
    with pytest.raises(ValueError):
        lay.to_solver([rhs[1]] + rhs[1:])
    other, _ = meshgen.mesh_system(3, 2, seed=1)
    with pytest.raises(ValueError):
        lay.values([other] + mats[1:])
    with pytest.raises(ValueError):
        batch.BatchLayout([])


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_batched_system_matches_single_handles(gpu, prec):
    from hybsol.b200 import batch

    mats, rhs = _systems(nrhs=2)
    bs = batch.BatchedSystem(mats)
    bs.decompose(prec)
    xs, info = bs.solve(rhs)
    assert info["converged"]
    for m, b, x in zip(mats, rhs, xs):
        order = gpu.compute_ordering(m.row_ptr, m.cols, "first").astype(np.int64)
        pm = m.permuted(order)
        ns = gpu.NativeSystem.from_matrix(pm)
        ns.decompose(gpu.FP64)
        x1, _ = ns.solve(reorder_rhs(m.sizes, order, b))
        ns.close()
        assert rel_err(x, reorder_rhs(pm.sizes, np.argsort(order), x1)) < (1e-12 if prec == 0 else 1e-11)
    # refactorization with new values through the layout
    scaled = [type(m)(m.sizes, m.row_ptr, m.cols, m.val_ptr, 2.0 * m.vals) for m in mats]
    bs.set_values(scaled)
    bs.decompose(prec)
    xs2, _ = bs.solve(rhs)
    for x, x2 in zip(xs, xs2):
        assert rel_err(2.0 * x2, x) < (1e-12 if prec == 0 else 1e-11)
    bs.close()


def test_plan_waves_properties():
    from hybsol.b200 import batch

    rng = np.random.default_rng(7)
    w = rng.integers(1, 100, 40)
    budget = 150
    waves = batch.plan_waves(w, budget)
    flat = sorted(i for v in waves for i in v)
    assert flat == list(range(40))
    assert all(sum(int(w[i]) for i in v) <= budget for v in waves)
    assert waves == batch.plan_waves(list(w), budget)  # deterministic
    assert waves == sorted(waves, key=lambda v: v[0]) and all(v == sorted(v) for v in waves)
    # a system above the budget gets a wave of its own
    big = batch.plan_waves([5, 500, 5], 100)
    assert [1] in big and sorted(i for v in big for i in v) == [0, 1, 2]
    with pytest.raises(ValueError):
        batch.plan_waves([1], 0)


def test_device_bytes_from_the_symbolic_fill(native):
    from hybsol.b200 import batch, meshgen

    m, _ = meshgen.mesh_system(4, 4, seed=1)
    order = native.compute_ordering(m.row_ptr, m.cols, "first").astype(np.int64)
    pm = m.permuted(order)
    slab = native.analyze(pm.sizes, pm.row_ptr, pm.cols)["slab_bytes_fp64"]
    b64 = batch.device_bytes(m, native.FP64)
    b32 = batch.device_bytes(m, native.MIXED)
    assert b64 == slab + 8 * len(m.vals) + 64 * m.dof
    assert b32 == slab // 2 + 8 * len(m.vals) + 64 * m.dof  # no 64-row blocks at p=4
    m8, _ = meshgen.mesh_system(2, 8, seed=1)
    assert batch.device_bytes(m8, native.MIXED) > batch.device_bytes(m8, native.FP64) // 2


@pytest.mark.gpu
def test_solve_many_in_waves(gpu):
    from hybsol.b200 import batch

    mats, rhs = _systems()
    sizes = [batch.device_bytes(m) for m in mats]
    budget = max(sizes) + min(sizes)  # forces several waves
    assert len(batch.plan_waves(sizes, budget)) > 1
    xs, infos = batch.solve_many(mats, rhs, budget)
    assert len(infos) == len(batch.plan_waves(sizes, budget))
    for m, b, x in zip(mats, rhs, xs):
        assert rel_err(m.matvec(x), b) < 1e-12


def test_batched_systems_share_stages(native):
    """The stacked system has as many elimination stages as its deepest member, not their
    sum: pivots of different systems run in the same stages (and launches)."""
    from hybsol.b200 import batch

    mats, _ = _systems()
    lay = batch.BatchLayout(mats)
    stacked = native.analyze(lay.matrix.sizes, lay.matrix.row_ptr, lay.matrix.cols)
    levels, flops = [], 0.0
    for m in mats:
        order = native.compute_ordering(m.row_ptr, m.cols, "first").astype(np.int64)
        pm = m.permuted(order)
        a = native.analyze(pm.sizes, pm.row_ptr, pm.cols)
        levels.append(a["n_levels"])
        flops += a["factor_flops"]
    assert stacked["n_levels"] == max(levels) < sum(levels)
    assert stacked["factor_flops"] == pytest.approx(flops, rel=1e-12)


@pytest.mark.gpu
def test_every_batched_system_converges_on_its_own_residual(gpu):
    """A batch of two well-conditioned systems and one ill-conditioned one (reduced shift,
    kappa_1 ~ 1e6) whose right-hand side is scaled by 1e-12, so that it is invisible in
    the norm of the whole stack: judged by the stack's norm the batch converges while that
    system is far from converged; judged per system (the batch's segments) refinement
    continues until it meets the tolerance too, and each system reports its own steps."""
    from hybsol.b200 import batch, meshgen

    easy1, b1 = meshgen.mesh_system(10, 4, seed=61)
    easy2, b2 = meshgen.mesh_system(9, 3, seed=62)
    hard, b3 = meshgen.mesh_system(8, 8, seed=0, shift=meshgen.reduced_shift(8, 8))
    mats, rhs = [easy1, easy2, hard], [b1, b2, 1e-12 * b3]

    def own_residuals(xs):
        return [float(np.linalg.norm(m.matvec(x) - b) / np.linalg.norm(b)) for m, x, b in zip(mats, xs, rhs)]

    bs = batch.BatchedSystem(mats)
    bs.decompose(gpu.MIXED)
    bs.native.set_segments([])  # judged by the whole stack
    x, ig = bs.native.solve(bs.layout.to_solver(rhs), max_iter=60)
    res_global = own_residuals(bs.layout.from_solver(x))
    assert ig["converged"] and res_global[2] > 1e-10, (ig, res_global)
    bs.native.set_segments(bs.layout.dof_off)  # judged system by system
    xs, info = bs.solve(rhs, max_iter=80)
    res = own_residuals(xs)
    assert info["converged"] and max(res) <= 1e-12 * 1.01, (info, res)
    per = info["systems"]
    assert all(s["iterations"] is not None for s in per)
    assert per[2]["iterations"] > max(per[0]["iterations"], per[1]["iterations"])
    # the device's residuals against a host recomputation: forming b - A x rounds at about
    # u ||A|| ||x|| / ||b||, a few 1e-15 here, so they agree to that
    for s, r in zip(per, res):
        assert s["relative_residual"] == pytest.approx(r, rel=1e-3, abs=2e-14)
    bs.close()


@pytest.mark.parametrize(("side", "p"), [(3, 2), (5, 4), (4, 6)])
def test_pattern_bytes_from_the_pattern_alone(native, side, p):
    """Waves of many systems are planned before their values exist: the generator's
    pattern alone gives the same pattern and the same device bytes as the full system."""
    from hybsol.b200 import batch, meshgen

    m, _ = meshgen.mesh_system(side, p, seed=7)
    sizes, row_ptr, cols = meshgen.mesh_pattern(side, p)
    assert np.array_equal(sizes, m.sizes) and np.array_equal(row_ptr, m.row_ptr) and np.array_equal(cols, m.cols)
    for prec in (native.FP64, native.MIXED):
        assert batch.pattern_bytes(sizes, row_ptr, cols, prec) == batch.device_bytes(m, prec)
