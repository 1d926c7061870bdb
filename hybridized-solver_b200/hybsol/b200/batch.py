"""Many independent block systems factored and solved together on one device handle.

The systems are stacked block-diagonally. Each system is ordered on its own with the
reference's coloring (any strategy), and its ordered blocks keep a contiguous index range
of the stack, so every system gets exactly the order -- and hence the factors -- it would
get alone. Ordering the union instead would tie a system's order to the others' under the
greedy and balanced strategies, which rank colours by counts over all blocks. Elimination
stages come from dependencies, not from indices, so pivots of different systems still
share stages, and with them kernel launches, which is what makes many small systems cheap.

``BatchLayout`` is the host-side part (stacking, ordering, moving vectors in and out);
``BatchedSystem`` adds the device handle. When the systems' factors exceed one device,
``plan_waves`` packs them into waves under a byte budget (from the exact symbolic fill of
each system) and ``solve_many`` runs the waves one after another.
"""

from __future__ import annotations

import numpy as np

from . import meshgen, native


def dof_permutation(sizes, order) -> np.ndarray:
    """``p`` with ``x_new[p] = x_old`` when old block ``i`` becomes block ``order[i]``
    (the renumbering of ``BlockMatrix.permuted`` and of the reference's ``reorder_blocks``)."""
    sizes = np.asarray(sizes, dtype=np.int64)
    order = np.asarray(order, dtype=np.int64)
    new_sizes = np.empty_like(sizes)
    new_sizes[order] = sizes
    off_old = np.concatenate([[0], np.cumsum(sizes)])
    off_new = np.concatenate([[0], np.cumsum(new_sizes)])
    block_of = np.repeat(np.arange(len(sizes)), sizes)
    within = np.arange(off_old[-1]) - off_old[block_of]
    return off_new[order[block_of]] + within


class BatchLayout:
    """Stacked, reordered form of independent systems (``meshgen.BlockMatrix`` each)."""

    def __init__(self, systems, strategy: str = "first"):
        self.systems = list(systems)
        if not self.systems:
            raise ValueError("no systems to batch")
        stacked = meshgen.block_diagonal(self.systems)
        self.dof_off = np.concatenate([[0], np.cumsum([m.dof for m in self.systems])]).astype(np.int64)
        self.block_off = np.concatenate([[0], np.cumsum([m.n_blocks for m in self.systems])]).astype(np.int64)
        own = [native.compute_ordering(m.row_ptr, m.cols, strategy).astype(np.int64) for m in self.systems]
        self.order = np.concatenate([o + b0 for o, b0 in zip(own, self.block_off[:-1])])
        # each system's blocks stay in its own index range, in its own order
        for i, o in enumerate(own):
            sub = self.order[self.block_off[i] : self.block_off[i + 1]] - self.block_off[i]
            assert np.array_equal(sub, o), "a batched system lost its own ordering"
        self.matrix = stacked.permuted(self.order)
        self.perm = dof_permutation(stacked.sizes, self.order)

    @property
    def count(self) -> int:
        return len(self.systems)

    def to_solver(self, rhs) -> np.ndarray:
        """One right-hand side per system (``(dof_i,)`` or ``(dof_i, k)``, the same k for all)
        -> the stacked vector in the solver's block order."""
        if len(rhs) != self.count:
            raise ValueError(f"expected {self.count} right-hand sides, got {len(rhs)}")
        parts = [np.asarray(r, dtype=np.float64) for r in rhs]
        for i, r in enumerate(parts):
            if r.shape[0] != self.dof_off[i + 1] - self.dof_off[i]:
                raise ValueError(f"right-hand side {i} has {r.shape[0]} rows, its system {self.dof_off[i + 1] - self.dof_off[i]}")
        b = np.concatenate(parts)
        out = np.empty_like(b)
        out[self.perm] = b
        return out

    def from_solver(self, x) -> list:
        """The solver's stacked solution -> one solution per system."""
        y = np.asarray(x)[self.perm]
        return [y[self.dof_off[i] : self.dof_off[i + 1]] for i in range(self.count)]

    def values(self, systems) -> np.ndarray:
        """New values for the same patterns, in the solver's order (for a refactorization)."""
        systems = list(systems)
        if len(systems) != self.count:
            raise ValueError(f"expected {self.count} systems, got {len(systems)}")
        for a, b in zip(systems, self.systems):
            if not (
                np.array_equal(a.sizes, b.sizes) and np.array_equal(a.row_ptr, b.row_ptr) and np.array_equal(a.cols, b.cols)
            ):
                raise ValueError("a system's block pattern differs from the batch's")
        return meshgen.block_diagonal(systems).permuted(self.order).vals


class BatchedSystem:
    """Independent systems factored and solved on one device handle (see the module text)."""

    def __init__(self, systems, strategy: str = "first"):
        self.layout = BatchLayout(systems, strategy)
        self.native = native.NativeSystem.from_matrix(self.layout.matrix)
        # every system's unknowns are one contiguous range of the stack: refinement judges
        # each system by its own residual, not by the norm of the whole stack
        self.native.set_segments(self.layout.dof_off)
        self._precision = None

    def set_values(self, systems):
        self.native.set_values(self.layout.values(systems))

    def decompose(self, precision: int = native.FP64) -> dict:
        self._precision = precision
        return self.native.decompose(precision)

    def solve(self, rhs, tol: float = 1e-12, max_iter: int = 50):
        """Solve every system for its right-hand side; returns (solutions, info). ``info``
        is the stack's solve info plus ``systems``: per system, ``iterations`` (the
        refinement steps after which its own relative residual first met ``tol``, None if
        it never did) and ``relative_residual`` (its own ||b_i - A_i x_i|| / ||b_i||, the
        largest over its right-hand sides)."""
        b = self.layout.to_solver(rhs)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        x, info = self.native.solve(b, tol=tol, max_iter=max_iter)
        first, rel = self.native.segment_results(nrhs)
        never = np.iinfo(np.uint32).max
        info["systems"] = [
            {
                "iterations": None if (first[i] == never).any() else int(first[i].max()),
                "relative_residual": float(rel[i].max()),
            }
            for i in range(self.layout.count)
        ]
        return self.layout.from_solver(x), info

    def close(self):
        self.native.close()


def device_bytes(system, precision: int = native.FP64, strategy: str = "first") -> int:
    """Device memory one system needs on a handle: its factor slab (FP64, or FP32 for the
    mixed form) from the exact symbolic fill under the reference's ordering, the original
    FP64 values, and the solve vectors; an estimate of the handle's footprint, not a bound
    on the allocator's."""
    order = native.compute_ordering(system.row_ptr, system.cols, strategy).astype(np.int64)
    pm = system.permuted(order)
    a = native.analyze(pm.sizes, pm.row_ptr, pm.cols)
    slab = int(a["slab_bytes_fp64"]) // (2 if precision == native.MIXED else 1)
    inv = 16384 * int(np.count_nonzero(np.asarray(system.sizes) == 64)) if precision == native.MIXED else 0
    return slab + 8 * len(system.vals) + 64 * int(system.dof) + inv


def pattern_bytes(sizes, row_ptr, cols, precision: int = native.FP64, strategy: str = "first") -> int:
    """``device_bytes`` from the block pattern alone (no values needed)."""
    sizes = np.asarray(sizes, dtype=np.int64)
    row_ptr = np.asarray(row_ptr, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    order = native.compute_ordering(row_ptr, cols, strategy).astype(np.int64)
    n = len(sizes)
    inv = np.empty(n, dtype=np.int64)
    inv[order] = np.arange(n)
    new_sizes = sizes[inv]
    counts = np.diff(row_ptr)[inv]
    new_ptr = np.concatenate([[0], np.cumsum(counts)])
    new_cols = np.concatenate([np.sort(order[cols[row_ptr[r] : row_ptr[r + 1]]]) for r in inv])
    a = native.analyze(new_sizes, new_ptr, new_cols)
    slab = int(a["slab_bytes_fp64"]) // (2 if precision == native.MIXED else 1)
    inv_bytes = 16384 * int(np.count_nonzero(sizes == 64)) if precision == native.MIXED else 0
    rows = np.repeat(np.arange(n), np.diff(row_ptr))
    nvals = int(np.sum(sizes[rows] * sizes[cols]))
    return slab + 8 * nvals + 64 * int(sizes.sum()) + inv_bytes


def plan_waves(weights, budget: int) -> list:
    """Indices of systems per wave: largest first, each into the first wave with room
    (first-fit decreasing); a system larger than the budget gets a wave of its own.
    Waves and their indices are in ascending order, so every caller gets the same plan."""
    if budget <= 0:
        raise ValueError("budget must be positive")
    w = [int(x) for x in weights]
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    waves, room = [], []
    for i in order:
        for k in range(len(waves)):
            if w[i] <= room[k]:
                waves[k].append(i)
                room[k] -= w[i]
                break
        else:
            waves.append([i])
            room.append(budget - w[i])
    waves = [sorted(v) for v in waves]
    waves.sort(key=lambda v: v[0])
    return waves


def solve_many(systems, rhs, budget: int, precision: int = native.FP64, tol: float = 1e-12, max_iter: int = 50):
    """Factor and solve independent systems in waves of at most ``budget`` device bytes
    (``plan_waves`` on ``device_bytes``); returns (solutions in input order, per-wave infos)."""
    systems = list(systems)
    if len(rhs) != len(systems):
        raise ValueError(f"expected {len(systems)} right-hand sides, got {len(rhs)}")
    waves = plan_waves([device_bytes(m, precision) for m in systems], budget)
    out = [None] * len(systems)
    infos = []
    for wave in waves:
        bs = BatchedSystem([systems[i] for i in wave])
        try:
            bs.decompose(precision)
            xs, info = bs.solve([rhs[i] for i in wave], tol=tol, max_iter=max_iter)
        finally:
            bs.close()
        for i, x in zip(wave, xs):
            out[i] = x
        infos.append(info)
    return out, infos
