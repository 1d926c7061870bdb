"""Parity of the B200 factorization and solve with the oracle and the reference.

Plain FP64 form (the drop-in): factors block-for-block within 1e-12 relative (per block,
relative to the block's largest entry) of the oracle, which is bit-identical to the
reference; identical filled pattern and operation list; solutions within 1e-12 relative.
Mixed form: FP32 factors refined in FP64 to a relative residual <= 1e-12, solution
within 1e-11 relative of the oracle's. Larger systems, beyond the oracle's reach in a
test, are checked through size-independent properties: the FP64 residual against A and
the agreement of the plain and mixed forms.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, rel_err, reorder_rhs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_FACTOR = 1e-12
TOL_X = 1e-12
TOL_X_MIXED = 1e-11


def _native_from(gpu, mat):
    order = gpu.compute_ordering(mat.row_ptr, mat.cols, "first")
    pm = mat.permuted(order)
    return order, pm, gpu.NativeSystem.from_matrix(pm)


def _check_factors(ns, osys, pm):
    worst = 0.0
    for i in range(pm.n_blocks):
        cols = ns.row_cols(i)
        assert cols == osys.get_row_block_indices(i), i
        for c in cols:
            got = ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c])))
            ref = osys.get_block(i, c)
            worst = max(worst, rel_err(got, ref))
    assert worst < TOL_FACTOR, worst
    return worst


def _mesh(n, p, seed, nrhs=1):
    from hybsol.b200 import meshgen

    return meshgen.mesh_system(n, p, seed=seed, nrhs=nrhs)


@pytest.mark.parametrize(
    ("n", "p", "nrhs"),
    [(16, 4, 1), (8, 8, 1), (6, "rand", 4), (4, 10, 2), (1, 3, 1)],
)
def test_mesh_fp64_matches_oracle(gpu, n, p, nrhs):
    from hybsol.b200 import meshgen

    pp = meshgen.random_orders(n, 2, 10, seed=11) if p == "rand" else p
    mat, b = _mesh(n, pp, seed=3, nrhs=nrhs)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    osys = O.OracleSystem.from_csr(pm.sizes, pm.row_ptr, pm.cols, pm.vals)
    osys.decompose()
    info = ns.decompose(gpu.FP64)
    assert info["zero_pivots"] == 0 and info["non_finite"] == 0
    _check_factors(ns, osys, pm)
    assert ns.operations() == osys.operations()
    x, sinfo = ns.solve(bn)
    assert rel_err(x, osys.solve(bn)) < TOL_X
    assert sinfo["relative_residual"] < 1e-13


def test_golden_mesh16_solution(gpu):
    """The reference's own solution of the 16x16 p=4 system (golden vector)."""
    g = golden("mesh16_p4.npz")
    mat, _ = _mesh(16, 4, seed=0)
    order, pm, ns = _native_from(gpu, mat)
    assert np.array_equal(order.astype(np.int64), g["order_first"])
    ns.decompose(gpu.FP64)
    x, _ = ns.solve(g["rhs_new_layout"])
    assert rel_err(x, g["x_new_layout"]) < TOL_X
    frp = np.concatenate([[0], np.cumsum([len(ns.row_cols(i)) for i in range(pm.n_blocks)])])
    assert np.array_equal(frp, g["filled_row_ptr"])
    ops = np.array([(o[0], o[1] if len(o) == 2 else -1) for o in ns.operations()])
    assert np.array_equal(ops, g["ops"])
    sums = np.array(
        [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))).sum() for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    )
    scale = np.sqrt(g["block_sumsq"]) + 1e-300
    assert np.max(np.abs(sums - g["block_sum"]) / scale) < 1e-12


def test_golden_mesh6_uneven_four_rhs(gpu):
    g = golden("mesh6_prand.npz")
    mat, _ = _mesh(6, g["p"], seed=5, nrhs=4)
    order, pm, ns = _native_from(gpu, mat)
    ns.decompose(gpu.FP64)
    x, _ = ns.solve(g["rhs_new_layout"])
    assert rel_err(x, g["x_new_layout"]) < TOL_X


@pytest.mark.parametrize(("n", "p", "nrhs"), [(16, 4, 1), (8, 8, 4), (6, "rand", 4)])
def test_mesh_mixed_refines_to_fp64(gpu, n, p, nrhs):
    from hybsol.b200 import meshgen

    pp = meshgen.random_orders(n, 2, 10, seed=11) if p == "rand" else p
    mat, b = _mesh(n, pp, seed=4, nrhs=nrhs)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    osys = O.OracleSystem.from_csr(pm.sizes, pm.row_ptr, pm.cols, pm.vals)
    osys.decompose()
    ns.decompose(gpu.MIXED)
    x, sinfo = ns.solve(bn, tol=1e-12)
    assert sinfo["converged"] and sinfo["relative_residual"] <= 1e-12
    assert 1 <= sinfo["iterations"] <= 10
    assert rel_err(x, osys.solve(bn)) < TOL_X_MIXED


def test_many_systems_in_one_handle(gpu):
    """Independent systems stacked block-diagonally factor in shared stages."""
    from hybsol.b200 import meshgen

    mats, rhs = [], []
    for k, (side, p) in enumerate([(3, 3), (5, 4), (4, 6), (2, 5)]):
        m, b = meshgen.mesh_system(side, p, seed=20 + k, nrhs=2)
        mats.append(m)
        rhs.append(b)
    big = meshgen.block_diagonal(mats)
    b = np.concatenate(rhs)
    order, pm, ns = _native_from(gpu, big)
    bn = reorder_rhs(big.sizes, order, b)
    osys = O.OracleSystem.from_csr(pm.sizes, pm.row_ptr, pm.cols, pm.vals)
    osys.decompose()
    ns.decompose(gpu.FP64)
    _check_factors(ns, osys, pm)
    x, _ = ns.solve(bn)
    assert rel_err(x, osys.solve(bn)) < TOL_X
    ns.decompose(gpu.MIXED)
    x2, info = ns.solve(bn)
    assert info["converged"] and rel_err(x2, x) < TOL_X_MIXED


def _random_system(rng, nb, max_size, density, sym=True, dom=True):
    sizes = rng.integers(1, max_size + 1, nb)
    rows = []
    vals = {}
    for i in range(nb):
        for j in range(nb):
            if i == j or rng.random() < density:
                vals[(i, j)] = rng.random((sizes[i], sizes[j]))
                if sym:
                    vals.setdefault((j, i), rng.random((sizes[j], sizes[i])))
    for i in range(nb):
        if dom:
            vals[(i, i)] = vals[(i, i)] + 2 * nb * max_size * np.eye(sizes[i])
    from hybsol.b200.meshgen import _assemble

    keys = sorted(vals)
    rows = np.array([k[0] for k in keys])
    cols = np.array([k[1] for k in keys])
    return _assemble(sizes.astype(np.int64), rows, cols, [vals[k] for k in keys])


@pytest.mark.parametrize("seed", range(6))
def test_random_sparse_systems(gpu, seed):
    rng = np.random.default_rng(seed)
    mat = _random_system(rng, int(rng.integers(3, 40)), int(rng.integers(1, 12)), float(rng.uniform(0.05, 0.5)), sym=seed % 2 == 0)
    osys = O.OracleSystem.from_csr(mat.sizes, mat.row_ptr, mat.cols, mat.vals)
    osys.decompose()
    ns = gpu.NativeSystem.from_matrix(mat)
    ns.decompose(gpu.FP64)
    _check_factors(ns, osys, mat)
    assert ns.operations() == osys.operations()
    b = rng.uniform(-1, 1, mat.dof)
    x, _ = ns.solve(b)
    assert rel_err(x, osys.solve(b)) < TOL_X


@pytest.mark.parametrize("size", [1, 31, 64, 65, 100, 130, 200])
def test_block_sizes_across_tiles(gpu, size):
    """Blocks smaller than, equal to and larger than the 64-wide tiles, and diagonal
    blocks too large for shared memory (the global-memory LU/TRSM paths)."""
    rng = np.random.default_rng(size)
    sizes = np.array([size, max(1, size // 2), size, 3], dtype=np.int64)
    nb = len(sizes)
    vals, keys = [], []
    for i in range(nb):
        for j in range(nb):
            keys.append((i, j))
            v = rng.standard_normal((sizes[i], sizes[j])) / np.sqrt(sizes[j])
            if i == j:
                v += 4 * np.eye(sizes[i])
            vals.append(v)
    from hybsol.b200.meshgen import _assemble

    mat = _assemble(sizes, np.array([k[0] for k in keys]), np.array([k[1] for k in keys]), vals)
    osys = O.OracleSystem.from_csr(mat.sizes, mat.row_ptr, mat.cols, mat.vals)
    osys.decompose()
    ns = gpu.NativeSystem.from_matrix(mat)
    ns.decompose(gpu.FP64)
    _check_factors(ns, osys, mat)
    b = rng.uniform(-1, 1, (mat.dof, 3))
    x, _ = ns.solve(b)
    assert rel_err(x, osys.solve(b)) < TOL_X


def test_zero_pivot_is_reported_not_raised(gpu):
    from hybsol.b200.meshgen import _assemble

    mat = _assemble(
        np.array([2, 2]), np.array([0, 0, 1, 1]), np.array([0, 1, 0, 1]),
        [np.array([[0.0, 1.0], [1.0, 1.0]]), np.eye(2), np.eye(2), np.eye(2) * 3],
    )  # fmt: skip
    ns = gpu.NativeSystem.from_matrix(mat)
    info = ns.decompose(gpu.FP64)
    assert info["zero_pivots"] >= 1 and info["first_bad_pivot"] == 0


@pytest.mark.parametrize("prec", [0, 1])
def test_lookahead_schedule_matches_in_order(gpu, prec):
    """The lookahead schedule (next pivot on a second stream) gives the in-order factors."""
    mat, b = _mesh(12, 8, seed=13)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    ns.decompose(prec)
    blocks = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    ns.set_lookahead(False)
    ns.set_values(pm.vals)
    ns.decompose(prec)
    blocks2 = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    assert all(np.array_equal(x, y) for x, y in zip(blocks, blocks2))


@pytest.mark.parametrize("prec", [0, 1])
def test_alternating_walk_matches_forward(gpu, prec):
    """Walking the targets backwards on alternate levels changes only which CTA updates a
    target when, not its arithmetic: the factors are bit-identical."""
    mat, b = _mesh(12, 8, seed=14)
    order, pm, ns = _native_from(gpu, mat)
    ns.decompose(prec)
    blocks = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    ns.set_option(gpu.OPTION_ALTERNATE_WALK, 0)
    ns.set_values(pm.vals)
    ns.decompose(prec)
    blocks2 = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    assert all(np.array_equal(x, y) for x, y in zip(blocks, blocks2))


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("p", [8, "rand"])
def test_pivot_lu_once_matches_fused(gpu, prec, p):
    """Factoring each 33-64-row pivot once and solving its strips from the stored factors
    gives the fused kernel's factors bit for bit (padded pivots of uneven orders included)."""
    from hybsol.b200 import meshgen

    pp = meshgen.random_orders(8, 2, 10, seed=31) if p == "rand" else p
    mat, b = _mesh(8, pp, seed=15)
    order, pm, ns = _native_from(gpu, mat)
    ns.set_option(gpu.OPTION_ROW_PIVOTS, 0)  # the 256-thread kernels
    ns.set_option(gpu.OPTION_PIVOT_LU_ONCE, 1)
    ns.decompose(prec)
    blocks = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    ns.set_option(gpu.OPTION_PIVOT_LU_ONCE, 0)
    ns.set_values(pm.vals)
    ns.decompose(prec)
    blocks2 = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    assert all(np.array_equal(x, y) for x, y in zip(blocks, blocks2))


@pytest.mark.parametrize(("prec", "pairs"), [(0, 1), (1, 1), (1, 0)])
def test_row_pivots_match_256_thread_kernels(gpu, prec, pairs):
    """The 64-thread pivot kernel (LU by rows, row solves by columns, splits in the same
    launch) gives the factors of the 256-thread kernels bit for bit, in both forms."""
    mat, b = _mesh(12, 8, seed=21)
    order, pm, ns = _native_from(gpu, mat)
    ns.set_option(gpu.OPTION_PAIR_PASSES, pairs)
    ns.set_option(gpu.OPTION_ROW_PIVOTS, 1)
    ns.decompose(prec)
    blocks = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    ns.set_option(gpu.OPTION_ROW_PIVOTS, 0)
    ns.set_values(pm.vals)
    ns.decompose(prec)
    blocks2 = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    assert all(np.array_equal(x, y) for x, y in zip(blocks, blocks2))


def test_update_sm_reserve_is_schedule_only(gpu):
    """Leaving SMs free for the pivot chain changes which CTA updates a target, not the
    target's arithmetic: the mixed factors are bit-identical for 0, 4 and 16 free SMs."""
    mat, b = _mesh(12, 8, seed=29)
    order, pm, ns = _native_from(gpu, mat)
    ref = None
    for reserve in (0, 4, 16):
        ns.set_option(gpu.OPTION_UPDATE_SM_RESERVE, reserve)
        ns.set_values(pm.vals)
        ns.decompose(gpu.MIXED)
        blocks = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
        if ref is None:
            ref = blocks
        else:
            assert all(np.array_equal(x, y) for x, y in zip(ref, blocks)), reserve
    with pytest.raises(gpu.HybError):
        ns.set_option(gpu.OPTION_UPDATE_SM_RESERVE, 65)


@pytest.mark.parametrize("pairs", [0, 1])
def test_inverse_pivots_match_substitution(gpu, pairs):
    """Mixed form: each 64-row pivot factored once and its upper blocks taken as products
    with its inverse (the default) against the blocked substitution: the FP32 factors agree
    to rounding, both refine to 1e-12 and agree with the oracle; the inverses written for
    the inner solves are those the factorization used."""
    mat, b = _mesh(12, 8, seed=27)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    osys = O.OracleSystem.from_csr(pm.sizes, pm.row_ptr, pm.cols, pm.vals)
    osys.decompose()
    xo = osys.solve(bn)
    ns.set_option(gpu.OPTION_PAIR_PASSES, pairs)
    out = {}
    for mode in (2, 1):
        ns.set_option(gpu.OPTION_ROW_PIVOTS, mode)
        ns.set_values(pm.vals)
        ns.decompose(gpu.MIXED)
        out[mode] = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
        x, info = ns.solve(bn)
        assert info["converged"] and info["relative_residual"] <= 1e-12, (mode, info)
        assert rel_err(x, xo) < TOL_X_MIXED
    worst = max(rel_err(a, b) for a, b in zip(out[2], out[1]))
    assert 0 < worst < 1e-3, worst


@pytest.mark.parametrize("prec", [0, 1])
def test_sampled_update_profile(gpu, prec):
    """Event pairs around every n-th level's update: ceil(levels / n) timed levels, the same
    level count for every stride, and factors identical to an untimed decomposition."""
    import ctypes

    mat, b = _mesh(10, 8, seed=23)
    order, pm, ns = _native_from(gpu, mat)
    ns.set_option(gpu.OPTION_PAIR_PASSES, 1)  # the mixed form then counts pairs as one pass
    lib = gpu.lib()
    ns.decompose(prec)
    ref = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    counts = {}
    for stride in (1, 4):
        assert lib.hyb_profile_enable(ns._h, stride) == 0
        ns.set_values(pm.vals)
        ns.decompose(prec)
        prof = gpu.KernelProfile()
        assert lib.hyb_profile_read(ns._h, ctypes.byref(prof)) == 0
        counts[stride] = (prof.launches, prof.passes, prof.levels, prof.pivots_timed)
        assert prof.total_ms > 0 and prof.c_elems > 0
        blocks = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
        assert all(np.array_equal(x, y) for x, y in zip(ref, blocks))
    passes, levels = counts[1][1], counts[1][2]
    assert passes > 4 and counts[1] == (passes, passes, levels, levels)
    assert counts[4][:3] == ((passes + 3) // 4, passes, levels)
    # the FP64 form takes one pass per level; the mixed form applies most pivots in pairs
    assert passes == levels if prec == 0 else levels // 2 < passes < levels
    assert lib.hyb_profile_enable(ns._h, -1) != 0
    assert lib.hyb_profile_enable(ns._h, 0) == 0


@pytest.mark.parametrize("n", [8, 12])
def test_pair_passes_match_single_passes(gpu, n):
    """Two pivots per tensor-core pass (mixed form default) against one pass per pivot: the
    factors differ only by the FP32 rounding of summing both products before subtracting
    (well inside BF16x3 accuracy), both refine to 1e-12 and agree with the oracle; with
    pairs, the lookahead schedule and the alternating walk give bit-identical factors."""
    mat, b = _mesh(n, 8, seed=19)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    osys = O.OracleSystem.from_csr(pm.sizes, pm.row_ptr, pm.cols, pm.vals)
    osys.decompose()
    xo = osys.solve(bn)

    def factor(opts=None):
        for k, v in (opts or {}).items():
            ns.set_option(k, v)
        ns.set_values(pm.vals)
        ns.decompose(gpu.MIXED)
        fs = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
        x, info = ns.solve(bn)
        assert info["converged"] and info["relative_residual"] <= 1e-12, info
        assert rel_err(x, xo) < TOL_X_MIXED
        return fs

    paired = factor({gpu.OPTION_PAIR_PASSES: 1})
    single = factor({gpu.OPTION_PAIR_PASSES: 0})
    worst = max(rel_err(a, b) for a, b in zip(paired, single))
    assert 0 < worst < 1e-3, worst  # the pair path ran, and only rounding separates them
    ns.set_option(gpu.OPTION_PAIR_PASSES, 1)
    for opts in ({gpu.OPTION_LOOKAHEAD: 0}, {gpu.OPTION_LOOKAHEAD: 1, gpu.OPTION_ALTERNATE_WALK: 0}):
        again = factor(opts)
        assert all(np.array_equal(x, y) for x, y in zip(paired, again)), opts


@pytest.mark.parametrize("n", [5, 12])
def test_tensor_core_mixed_matches_cuda_core_mixed(gpu, n):
    """The tcgen05 split-BF16 updates and the FP32 CUDA-core updates both refine to 1e-12
    and agree on the solution; the tensor-core factors stay within BF16x3 accuracy."""
    mat, b = _mesh(n, 8, seed=17)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    ns.decompose(gpu.FP64)
    x64, _ = ns.solve(bn)
    f64 = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    ns.set_values(pm.vals)
    ns.set_option(gpu.OPTION_BLOCK_SCALING, 0)  # the factors of A itself, to compare with FP64's
    ns.decompose(gpu.MIXED)
    ftc = [ns.get_block(i, c, (int(pm.sizes[i]), int(pm.sizes[c]))) for i in range(pm.n_blocks) for c in ns.row_cols(i)]
    xtc, itc = ns.solve(bn)
    ns.set_tensor_core_mixed(False)
    ns.set_values(pm.vals)
    ns.decompose(gpu.MIXED)
    xcc, icc = ns.solve(bn)
    assert itc["converged"] and icc["converged"]
    assert rel_err(xtc, x64) < TOL_X_MIXED and rel_err(xcc, x64) < TOL_X_MIXED
    worst = max(rel_err(a, b) for a, b in zip(ftc, f64))
    assert worst < 1e-3, worst


def test_refactorization_reuses_the_handle(gpu):
    mat, b = _mesh(8, 4, seed=9)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    ns.decompose(gpu.FP64)
    x1, _ = ns.solve(bn)
    ns.set_values(pm.vals * 2.0)
    ns.decompose(gpu.FP64)
    x2, _ = ns.solve(bn)
    assert rel_err(x2, x1 / 2.0) < 1e-13
    cp = ns.copy()
    x3, _ = cp.solve(bn)
    assert np.array_equal(x3, x2)


@pytest.mark.parametrize("n", [32, 48])
def test_larger_mesh_properties(gpu, n):
    """Above the oracle's comfortable size: FP64 residual and plain/mixed agreement."""
    mat, b = _mesh(n, 8, seed=1)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    ns.decompose(gpu.FP64)
    x64, i64 = ns.solve(bn)
    assert i64["relative_residual"] < 1e-13
    r = ns.residual(bn, x64)
    assert np.linalg.norm(r) / np.linalg.norm(bn) < 1e-13
    ns.decompose(gpu.MIXED)
    xm, im = ns.solve(bn, tol=1e-12)
    assert im["converged"] and im["relative_residual"] <= 1e-12
    assert rel_err(xm, x64) < TOL_X_MIXED


def test_dense_single_block_kernels(gpu):
    rng = np.random.default_rng(5)
    for m in (1, 5, 64, 100, 300):
        a = rng.standard_normal((m, m)) + m * np.eye(m)
        lu = gpu.block_lu(a)
        ref = O.lu_decompose(a)
        assert rel_err(lu, ref) < 1e-12
        b = rng.standard_normal((m, 70))
        assert rel_err(gpu.block_lu_solve(lu, b), O.lu_solve(ref, b)) < 1e-12


@pytest.mark.parametrize(("n", "p", "nrhs"), [(12, 8, 1), (6, "rand", 3), (16, 4, 2)])
@pytest.mark.parametrize("prec", [0, 1])
def test_dataflow_solve_matches_staged(gpu, n, p, nrhs, prec):
    """The dataflow substitution (one cooperative launch per direction, pivots released by
    flags) forms the same partial products in the same order as the staged one, so the
    solutions agree bit for bit; both match the oracle."""
    from hybsol.b200 import meshgen

    pp = meshgen.random_orders(n, 2, 10, seed=5) if p == "rand" else p
    mat, b = _mesh(n, pp, seed=21, nrhs=nrhs)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    ns.decompose(prec)
    x_flow, info_f = ns.solve(bn)
    x_flow2, _ = ns.solve(bn)  # flags and tickets carry over between solves
    ns.set_dataflow_solve(False)
    x_staged, info_s = ns.solve(bn)
    assert np.array_equal(x_flow, x_staged) and np.array_equal(x_flow, x_flow2)
    assert info_f["iterations"] == info_s["iterations"]
    osys = O.OracleSystem.from_csr(pm.sizes, pm.row_ptr, pm.cols, pm.vals)
    osys.decompose()
    assert rel_err(x_flow, osys.solve(bn)) < (TOL_X if prec == 0 else TOL_X_MIXED)


@pytest.mark.parametrize("umma", [True, False])
def test_mixed_inner_solve_with_diagonal_inverses(gpu, umma):
    """The mixed form's FP32 solve applies explicit inverses of the 64x64 diagonal blocks:
    unrefined it is already close to the FP64 solution, and one refinement step reaches
    1e-12, as with substitution."""
    mat, b = _mesh(10, 8, seed=29)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    ns.decompose(gpu.FP64)
    x64, _ = ns.solve(bn)
    ns.set_tensor_core_mixed(umma)
    ns.set_values(pm.vals)
    ns.decompose(gpu.MIXED)
    x0, info0 = ns.solve(bn, max_iter=0)
    assert rel_err(x0, x64) < 1e-4
    x1, info1 = ns.solve(bn)
    assert info1["converged"] and info1["iterations"] <= 2
    assert info1["relative_residual"] <= 1e-12 and rel_err(x1, x64) < TOL_X_MIXED


@pytest.mark.parametrize("prec", [0, 1])
def test_uneven_orders_large_pivot_grids(gpu, prec):
    """64x64 mesh with per-element orders 2..10: pivots of 33-64 rows take the padded fused
    LU + row-solve kernel with more CTAs than fit at once (and 128-wide upper blocks in two
    strips); every CTA must factor the unfactored block. The FP64 residual pins it."""
    from hybsol.b200 import meshgen

    n = 64
    mat, b = _mesh(n, meshgen.random_orders(n, 2, 10, seed=0), seed=0)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    ns.decompose(prec)
    x, info = ns.solve(bn)
    assert info["relative_residual"] < (1e-13 if prec == 0 else 1e-12)


@pytest.mark.parametrize("kind", [-1, 0, 1, 2])
def test_generic_update_kernels_match_oracle(gpu, kind):
    """Uneven orders 2..10: every generic Schur-update kernel -- 32x32 and 64x64 SIMT tiles,
    the FP64 tensor pipe (DMMA, operands zero-padded) and the tuned choice per size bucket --
    gives the oracle's FP64 factors within 1e-12 per block; the mixed form (FP64 products
    into FP32 factors on the DMMA path) refines to the FP64 solution."""
    from hybsol.b200 import meshgen

    pp = meshgen.random_orders(7, 2, 10, seed=19)
    mat, b = _mesh(7, pp, seed=8, nrhs=2)
    order, pm, ns = _native_from(gpu, mat)
    bn = reorder_rhs(mat.sizes, order, b)
    ns.set_option(gpu.OPTION_UPDATE_KERNEL, kind)
    osys = O.OracleSystem.from_csr(pm.sizes, pm.row_ptr, pm.cols, pm.vals)
    osys.decompose()
    ns.decompose(gpu.FP64)
    _check_factors(ns, osys, pm)
    x, _ = ns.solve(bn)
    xo = osys.solve(bn)
    assert rel_err(x, xo) < TOL_X
    if kind == -1:
        tuned = ns.tuned_kernels(gpu.FP64)
        assert (tuned >= 0).any() and set(np.unique(tuned[tuned >= 0])) <= {0, 1, 2}
    ns.set_values(pm.vals)
    ns.decompose(gpu.MIXED)
    xm, im = ns.solve(bn)
    assert im["converged"] and rel_err(xm, xo) < TOL_X_MIXED


@pytest.mark.parametrize("shape", [0, 1, 2])
def test_fp64_update_mma_shapes_match_oracle(gpu, shape):
    """The FP64 64-block update with each FP64 MMA instruction shape (m8n8k4, m16n8k8,
    m16n8k16) gives the oracle's factors within 1e-12 per block."""
    mat, b = _mesh(8, 8, seed=27)
    order, pm, ns = _native_from(gpu, mat)
    ns.set_option(gpu.OPTION_FP64_MMA_SHAPE, shape)
    osys = O.OracleSystem.from_csr(pm.sizes, pm.row_ptr, pm.cols, pm.vals)
    osys.decompose()
    ns.decompose(gpu.FP64)
    _check_factors(ns, osys, pm)
    bn = reorder_rhs(mat.sizes, order, b)
    assert rel_err(ns.solve(bn)[0], osys.solve(bn)) < TOL_X
