"""Synthetic hybridized quad-mesh block systems.

A mesh of ``n x n`` quadrilateral elements. Every element carries one interior
unknown block of ``p_e**2`` rows, every mesh edge one block of ``max(p)`` rows over
its (one or two) adjacent elements. The nonzero blocks are all diagonal blocks and
the element<->edge couplings of each element's four edges, in both directions --
the pattern the reference's hybridized solver factors.

Numbering (element first):

* element ``e = y*n + x``;
* horizontal edge at ``(x, y)``, ``y in [0, n]``: ``n*n + y*n + x``;
* vertical edge at ``(x, y)``, ``x in [0, n]``: ``n*n + n*(n+1) + y*(n+1) + x``.

Values, drawn from ``numpy.random.default_rng(seed)`` in this order:

1. for each element ``e`` in order and each of its edges ``h(x,y), h(x,y+1),
   v(x,y), v(x+1,y)``: the block ``B(e,g)`` then ``B(g,e)``, entries
   ``N(0,1)/sqrt(columns of that block)``;
2. the diagonal blocks in block order: ``N(0,1)/sqrt(s) + shift*(sum of the
   Frobenius norms of the row's off-diagonal blocks + 1)*I``, ``shift = 1``
   giving a diagonally dominant system;
3. the right-hand sides ``U[-1, 1]`` of shape ``(dof,)`` or ``(dof, nrhs)``.

Reduced-shift value sets scale the diagonal shift by ``alpha < 1`` (the same draws, so only
the diagonals change). The system loses diagonal dominance and its condition number grows
as ``alpha`` falls; ``tune_shift`` bisects ``alpha`` until a 1-norm condition estimate hits a
target (1e6 for the ill-conditioned set), and ``REDUCED_SHIFT`` records the values found.

The reference's coloring ("first") places all edges before all elements for this
pattern, whatever the numbering, so the factorization sees the edge rows first.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class BlockMatrix:
    """A block-sparse matrix in block-CSR form.

    ``sizes[i]`` is the size of block row/column ``i``; row ``i`` holds the blocks
    ``cols[row_ptr[i]:row_ptr[i+1]]`` (ascending), and block ``j`` stores its values
    row-major in ``vals[val_ptr[j]:val_ptr[j+1]]``.
    """

    sizes: np.ndarray
    row_ptr: np.ndarray
    cols: np.ndarray
    val_ptr: np.ndarray
    vals: np.ndarray

    @property
    def n_blocks(self) -> int:
        return len(self.sizes)

    @property
    def dof(self) -> int:
        return int(self.sizes.sum())

    @property
    def nnz_blocks(self) -> int:
        return len(self.cols)

    def block(self, j: int) -> np.ndarray:
        """Value of the ``j``-th stored block (CSR order) as a 2-D view."""
        r = int(np.searchsorted(self.row_ptr, j, side="right") - 1)
        c = int(self.cols[j])
        return self.vals[self.val_ptr[j] : self.val_ptr[j + 1]].reshape(int(self.sizes[r]), int(self.sizes[c]))

    def iter_blocks(self):
        """Yield ``(row, col, value)`` for every stored block, in CSR order."""
        sizes = self.sizes
        for r in range(self.n_blocks):
            for j in range(int(self.row_ptr[r]), int(self.row_ptr[r + 1])):
                c = int(self.cols[j])
                yield r, c, self.vals[self.val_ptr[j] : self.val_ptr[j + 1]].reshape(int(sizes[r]), int(sizes[c]))

    def to_dense(self) -> np.ndarray:
        off = np.concatenate([[0], np.cumsum(self.sizes)])
        a = np.zeros((self.dof, self.dof))
        for r, c, v in self.iter_blocks():
            a[off[r] : off[r + 1], off[c] : off[c + 1]] = v
        return a

    def permuted(self, order) -> "BlockMatrix":
        """Symmetric block permutation: old block ``i`` becomes block ``order[i]``.

        The same renumbering as ``BlockSystem.reorder_blocks(order)``.
        """
        order = np.asarray(order, dtype=np.int64)
        n = self.n_blocks
        inv = np.empty(n, dtype=np.int64)
        inv[order] = np.arange(n)
        sizes = self.sizes[inv]
        row_nnz = np.diff(self.row_ptr)[inv]
        row_ptr = np.concatenate([[0], np.cumsum(row_nnz)]).astype(np.int64)
        cols = np.empty_like(self.cols)
        src_blocks = np.empty(len(self.cols), dtype=np.int64)
        for new_r in range(n):
            old_r = inv[new_r]
            b, e = int(self.row_ptr[old_r]), int(self.row_ptr[old_r + 1])
            new_c = order[self.cols[b:e]]
            srt = np.argsort(new_c, kind="stable")
            cols[row_ptr[new_r] : row_ptr[new_r + 1]] = new_c[srt]
            src_blocks[row_ptr[new_r] : row_ptr[new_r + 1]] = b + srt
        counts = self.val_ptr[src_blocks + 1] - self.val_ptr[src_blocks]
        val_ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        starts = self.val_ptr[src_blocks]
        idx = np.repeat(starts - val_ptr[:-1], counts) + np.arange(val_ptr[-1])
        return BlockMatrix(sizes, row_ptr, cols, val_ptr, self.vals[idx])

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """``A @ x`` for ``x`` of shape ``(dof,)`` or ``(dof, k)`` (float64, on the host)."""
        off = np.concatenate([[0], np.cumsum(self.sizes)])
        y = np.zeros_like(x, dtype=np.float64)
        for r, c, v in self.iter_blocks():
            y[off[r] : off[r + 1]] += v @ x[off[c] : off[c + 1]]
        return y


def _assemble(sizes: np.ndarray, rows: np.ndarray, cols: np.ndarray, blocks: list) -> BlockMatrix:
    """Sort (row, col, value) triples into block-CSR (duplicates are not expected)."""
    order = np.lexsort((cols, rows))
    rows = rows[order]
    cols = cols[order]
    counts = sizes[rows] * sizes[cols]
    val_ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    vals = np.empty(int(val_ptr[-1]), dtype=np.float64)
    for k, src in enumerate(order):
        vals[val_ptr[k] : val_ptr[k + 1]] = blocks[src].ravel()
    row_ptr = np.zeros(len(sizes) + 1, dtype=np.int64)
    np.add.at(row_ptr, rows + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    return BlockMatrix(sizes.astype(np.int64), row_ptr, cols.astype(np.int64), val_ptr, vals)


def mesh_layout(n: int, p):
    """Block sizes and the four edges of every element for an ``n x n`` mesh.

    ``p`` is a scalar order or an array of ``n*n`` per-element orders.
    Returns ``(sizes, elem_edges)`` with ``elem_edges[e] = (h(x,y), h(x,y+1), v(x,y), v(x+1,y))``.
    """
    ne = n * n
    pe = np.broadcast_to(np.asarray(p, dtype=np.int64), (ne,)).reshape(n, n)
    h0 = ne
    v0 = ne + n * (n + 1)
    ys, xs = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    elem_edges = np.stack(
        [
            h0 + ys * n + xs,
            h0 + (ys + 1) * n + xs,
            v0 + ys * (n + 1) + xs,
            v0 + ys * (n + 1) + xs + 1,
        ],
        axis=-1,
    ).reshape(ne, 4)
    sizes = np.zeros(ne + 2 * n * (n + 1), dtype=np.int64)
    sizes[:ne] = (pe * pe).ravel()
    edge_p = np.zeros(len(sizes), dtype=np.int64)
    flat_p = pe.ravel()
    for k in range(4):
        np.maximum.at(edge_p, elem_edges[:, k], flat_p)
    sizes[ne:] = edge_p[ne:]
    return sizes, elem_edges


def mesh_system(n: int, p, seed: int = 0, nrhs: int = 1, shift: float = 1.0):
    """Build the mesh system and its right-hand side(s).

    Returns ``(matrix, rhs)``; ``rhs`` has shape ``(dof,)`` when ``nrhs == 1``,
    else ``(dof, nrhs)``.
    """
    rng = np.random.default_rng(seed)
    sizes, elem_edges = mesh_layout(n, p)
    ne = n * n
    nb = len(sizes)
    # 1. couplings, element by element, edge by edge: B(e,g) then B(g,e)
    se = sizes[:ne]
    sg = sizes[elem_edges]  # (ne, 4)
    per_elem = 2 * (se[:, None] * sg).sum(axis=1)
    draws = rng.standard_normal(int(per_elem.sum()))
    rows, cols, blocks = [], [], []
    norms = np.zeros(nb)
    pos = 0
    for e in range(ne):
        s_e = int(se[e])
        for k in range(4):
            g = int(elem_edges[e, k])
            s_g = int(sizes[g])
            cnt = s_e * s_g
            b_eg = draws[pos : pos + cnt].reshape(s_e, s_g) / np.sqrt(s_g)
            pos += cnt
            b_ge = draws[pos : pos + cnt].reshape(s_g, s_e) / np.sqrt(s_e)
            pos += cnt
            rows += [e, g]
            cols += [g, e]
            blocks += [b_eg, b_ge]
            norms[e] += np.linalg.norm(b_eg)
            norms[g] += np.linalg.norm(b_ge)
    # 2. diagonals in block order
    diag_draws = rng.standard_normal(int((sizes * sizes).sum()))
    pos = 0
    for i in range(nb):
        s = int(sizes[i])
        d = diag_draws[pos : pos + s * s].reshape(s, s) / np.sqrt(s)
        pos += s * s
        d[np.diag_indices(s)] += shift * (norms[i] + 1.0)
        rows.append(i)
        cols.append(i)
        blocks.append(d)
    mat = _assemble(sizes, np.asarray(rows, dtype=np.int64), np.asarray(cols, dtype=np.int64), blocks)
    dof = int(sizes.sum())
    rhs = rng.uniform(-1.0, 1.0, dof if nrhs == 1 else (dof, nrhs))
    return mat, rhs


def mesh_pattern(n: int, p):
    """The block pattern of ``mesh_system(n, p)`` without its values: ``(sizes, row_ptr,
    cols)`` in the same (element-first) numbering, columns ascending in every row."""
    sizes, elem_edges = mesh_layout(n, p)
    ne = n * n
    rows = np.concatenate([np.repeat(np.arange(ne), 4), elem_edges.ravel(), np.arange(len(sizes))])
    cols = np.concatenate([elem_edges.ravel(), np.repeat(np.arange(ne), 4), np.arange(len(sizes))])
    order = np.lexsort((cols, rows))
    rows, cols = rows[order], cols[order]
    row_ptr = np.zeros(len(sizes) + 1, dtype=np.int64)
    np.add.at(row_ptr, rows + 1, 1)
    return sizes.astype(np.int64), np.cumsum(row_ptr), cols.astype(np.int64)


def random_orders(n: int, pmin: int, pmax: int, seed: int = 0) -> np.ndarray:
    """Per-element orders drawn uniformly from ``{pmin, ..., pmax}``."""
    return np.random.default_rng(seed).integers(pmin, pmax + 1, n * n)


def many_mesh_specs(count: int, side_range=(8, 64), p_range=(3, 6), seed: int = 0):
    """(side, p) of ``count`` independent systems, sides and orders drawn uniformly."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        side = int(rng.integers(side_range[0], side_range[1] + 1))
        p = int(rng.integers(p_range[0], p_range[1] + 1))
        out.append((side, p))
    return out


def block_diagonal(mats: list) -> BlockMatrix:
    """Stack independent systems into one block-diagonal system (blocks renumbered)."""
    sizes = np.concatenate([m.sizes for m in mats])
    row_ptr = [np.zeros(1, dtype=np.int64)]
    cols, val_ptr, vals = [], [np.zeros(1, dtype=np.int64)], []
    b0 = 0
    nb0 = 0
    v0 = 0
    for m in mats:
        row_ptr.append(m.row_ptr[1:] + nb0)
        cols.append(m.cols + b0)
        val_ptr.append(m.val_ptr[1:] + v0)
        vals.append(m.vals)
        b0 += m.n_blocks
        nb0 += m.nnz_blocks
        v0 += len(m.vals)
    return BlockMatrix(
        sizes.astype(np.int64),
        np.concatenate(row_ptr),
        np.concatenate(cols),
        np.concatenate(val_ptr),
        np.concatenate(vals),
    )


# Shift scale alpha giving a 1-norm condition number of about 1e6 for the seed-0 mesh
# system of (elements per side, p): found by tune_shift with the exact kappa_1 (dense
# inverse) for the small meshes and with the library's Hager estimate from the FP64
# factors on a B200 for the large ones. Value: (alpha, kappa_1 at alpha, how it was found).
REDUCED_SHIFT: dict = {
    (8, 8): (0.1146255054005839, 9.640e5, "exact kappa_1 (dense inverse)"),
    (16, 4): (0.2513574752782007, 1.117e6, "exact kappa_1 (dense inverse)"),
    (32, 8): (0.2013112914936568, 1.206e6, "Hager estimate from the FP64 factors on a B200"),
    (64, 8): (0.2420077241865368, 1.090e6, "Hager estimate from the FP64 factors on a B200"),
    (128, 8): (0.25, 1.008e6, "Hager estimate from the FP64 factors on a B200"),
}


def reduced_shift(n: int, p) -> float:
    """The recorded shift scale of the ill-conditioned (kappa_1 ~ 1e6) set for this mesh."""
    try:
        return REDUCED_SHIFT[(int(n), int(p))][0]
    except (KeyError, ValueError):
        raise KeyError(
            f"no reduced shift recorded for {n}x{n} p={p}: find it with `python -m hybsol.b200.tune_shift {n} {p}`"
        ) from None


def diagonal_weights(mat: BlockMatrix, shift_per_row: np.ndarray):
    """Indices of the diagonal entries in ``mat.vals`` and the shift each one carries per
    unit of ``alpha`` (its block row's ``sum of off-diagonal Frobenius norms + 1``)."""
    idx, w = [], []
    for r in range(mat.n_blocks):
        b, e = int(mat.row_ptr[r]), int(mat.row_ptr[r + 1])
        j = b + int(np.searchsorted(mat.cols[b:e], r))
        s = int(mat.sizes[r])
        idx.append(mat.val_ptr[j] + np.arange(s) * (s + 1))
        w.append(np.full(s, shift_per_row[r]))
    return np.concatenate(idx), np.concatenate(w)


def row_shift_amounts(mat: BlockMatrix, n: int) -> np.ndarray:
    """Per block row, the diagonal shift of ``alpha = 1``: the sum of the Frobenius norms of
    the row's off-diagonal blocks, plus one (as the generator adds it)."""
    out = np.ones(mat.n_blocks)
    for r in range(mat.n_blocks):
        for j in range(int(mat.row_ptr[r]), int(mat.row_ptr[r + 1])):
            if int(mat.cols[j]) != r:
                out[r] += np.linalg.norm(mat.vals[mat.val_ptr[j] : mat.val_ptr[j + 1]])
    return out


def shifted_values(mat: BlockMatrix, alpha_from: float, alpha_to: float, weights=None) -> np.ndarray:
    """Values of ``mat`` (generated with shift ``alpha_from``) re-shifted to ``alpha_to``
    without regenerating the draws (equal to ``mesh_system(shift=alpha_to)`` up to one
    rounding of each diagonal entry). ``weights`` from ``diagonal_weights`` may be reused."""
    idx, w = weights if weights is not None else diagonal_weights(mat, row_shift_amounts(mat, 0))
    vals = mat.vals.copy()
    vals[idx] += (alpha_to - alpha_from) * w
    return vals


def tune_shift(kappa_of_alpha, target: float = 1e6, tol_decades: float = 0.1, alpha_hi: float = 1.0,
               max_steps: int = 30):
    """Bisect the shift scale so that ``kappa_of_alpha(alpha)`` is within ``tol_decades``
    (log10) of ``target``. Starts at ``alpha_hi`` (which must be better conditioned than
    the target), halves alpha until the condition number passes the target, then bisects
    the bracket in log alpha. Returns ``(alpha, kappa, [(alpha, kappa), ...])``."""
    history = []

    def kap(a):
        k = float(kappa_of_alpha(a))
        history.append((a, k))
        return k

    hi, k_hi = alpha_hi, kap(alpha_hi)
    if not k_hi < target:
        raise ValueError(f"alpha={alpha_hi} is already at kappa {k_hi:.3g} >= {target:.3g}")
    lo = hi
    for _ in range(max_steps):
        lo = lo / 2
        k_lo = kap(lo)
        if abs(np.log10(k_lo / target)) <= tol_decades:
            return lo, k_lo, history
        if k_lo >= target:
            break
        hi, k_hi = lo, k_lo
    else:
        raise RuntimeError("no alpha above the target condition number was found")
    for _ in range(max_steps):
        mid = float(np.sqrt(lo * hi))
        k_mid = kap(mid)
        if abs(np.log10(k_mid / target)) <= tol_decades:
            return mid, k_mid, history
        if k_mid >= target:
            lo = mid
        else:
            hi = mid
    raise RuntimeError(f"bisection did not reach kappa {target:.3g} within {max_steps} steps: {history[-3:]}")


def exact_kappa1(mat: BlockMatrix, vals=None) -> float:
    """1-norm condition number from the dense inverse (small systems only)."""
    m = mat if vals is None else BlockMatrix(mat.sizes, mat.row_ptr, mat.cols, mat.val_ptr, vals)
    a = m.to_dense()
    return float(np.abs(a).sum(axis=0).max() * np.abs(np.linalg.inv(a)).sum(axis=0).max())
