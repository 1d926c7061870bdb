"""Generate the golden vectors under tests/golden/ from the REFERENCE itself.

Runs j4nr0th/hybridized-solver's own extension, compiled from its sources into
oracle/_ref by ``make -C oracle ref`` (needs the reference tree mounted, which is only
the case in the build container), on seeded inputs, and stores its outputs:

* ``mesh16_p4.npz``  -- the 16x16-element, p=4 quad mesh (the reference's CPU
  configuration): coloring orders for all three strategies, the filled pattern after
  ``decompose()``, the operation list (one OpenMP thread), per-block factor checksums,
  the full factors of the first 40 block rows, and the solution of one RHS.
  (Full factors are kept for the first ``full_rows`` and last ``tail_rows`` block rows.)
* ``mesh6_prand.npz`` -- a 6x6 mesh with per-element orders in {2..10} and 4 RHS.
* ``random_orderings.npz`` -- coloring orders of random symmetric block patterns
  (the builder of the reference's ordering tests) for all strategies.
* ``dense_blocks.npz`` -- full factors and solution of dense block systems.

Usage: ``python tests/golden/make_golden.py`` (writes next to this file).
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "hybridized-solver_b200"))

os.environ.setdefault("OMP_NUM_THREADS", "1")  # the op list order is only defined for one thread

from hybsol.b200 import meshgen  # noqa: E402
from oracle.oracle import load_reference  # noqa: E402

STRATS = ("first", "greedy", "balanced")


def _load(ref, mat):
    s = ref.BlockSystem(*[int(x) for x in mat.sizes])
    for r, c, v in mat.iter_blocks():
        s.add_block(r, c, v)
    return s


def _pattern(s):
    rows = [s.get_row_block_indices(i) for i in range(s.n_blocks)]
    row_ptr = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    cols = np.array([c for r in rows for c in r], dtype=np.int64)
    return rows, row_ptr, cols


def _ops(s):
    return np.array([(o[0], o[1] if len(o) == 2 else -1) for o in s.operations()], dtype=np.int64)


def mesh_case(ref, n, p, seed, nrhs, full_rows, tail_rows=0):
    mat, b = meshgen.mesh_system(n, p, seed=seed, nrhs=nrhs)
    s = _load(ref, mat)
    out = {
        "sizes": mat.sizes,
        "row_ptr": mat.row_ptr,
        "cols": mat.cols,
        "seed": np.int64(seed),
        "n": np.int64(n),
    }
    for st in STRATS:
        out[f"order_{st}"] = s.compute_reordering(st).astype(np.int64)
    order = out["order_first"]
    s.reorder_blocks(order.astype(np.uint64))
    cols_b = b if b.ndim == 2 else b[:, None]
    bn = np.stack([s.unorder_vector(order.astype(np.uint64), np.ascontiguousarray(cols_b[:, j])) for j in range(cols_b.shape[1])], axis=1)
    s.decompose(0)
    rows, frp, fcols = _pattern(s)
    out["filled_row_ptr"] = frp
    out["filled_cols"] = fcols
    out["ops"] = _ops(s)
    sums, sq = [], []
    full = []
    for i, r in enumerate(rows):
        for c in r:
            blk = s.get_block(i, c)
            sums.append(blk.sum())
            sq.append((blk * blk).sum())
            if i < full_rows or i >= s.n_blocks - tail_rows:
                full.append(blk.ravel())
    out["block_sum"] = np.array(sums)
    out["block_sumsq"] = np.array(sq)
    out["full_rows"] = np.int64(full_rows)
    out["tail_rows"] = np.int64(tail_rows)
    out["full_values"] = np.concatenate(full)
    xs = np.stack([s.solve(np.ascontiguousarray(bn[:, j])) for j in range(bn.shape[1])], axis=1)
    out["rhs_new_layout"] = bn
    out["x_new_layout"] = xs
    return out


def random_orderings(ref):
    out = {}
    k = 0
    for seed, nb, bs, sp in ((1359, 10, 5, 0.3), (1359, 15, 5, 0.9), (1359, 200, 2, 0.8), (7, 60, 4, 0.5), (11, 120, 3, 0.95)):
        rng = np.random.default_rng(seed)
        sizes = rng.integers(1, bs, nb)
        s = ref.BlockSystem(*[int(x) for x in sizes])
        for ir in range(nb):
            s.add_block(ir, ir, rng.random((sizes[ir], sizes[ir])) + 0.1)
            for ic in range(ir + 1, nb):
                if sp > rng.random(1):
                    continue
                s.add_block(ir, ic, rng.random((sizes[ir], sizes[ic])))
                s.add_block(ic, ir, rng.random((sizes[ic], sizes[ir])))
        _, rp, cc = _pattern(s)
        out[f"c{k}_sizes"] = sizes.astype(np.int64)
        out[f"c{k}_row_ptr"] = rp
        out[f"c{k}_cols"] = cc
        for st in STRATS:
            out[f"c{k}_order_{st}"] = s.compute_reordering(st).astype(np.int64)
        # a capped color count that the pattern cannot meet
        maxdeg = int(np.max(np.diff(rp)))
        out[f"c{k}_maxdeg"] = np.int64(maxdeg)
        k += 1
    out["count"] = np.int64(k)
    return out


def dense_blocks(ref):
    out = {}
    k = 0
    for nb, bs in ((2, 2), (4, 3), (10, 4), (5, 7)):
        rng = np.random.default_rng(15)
        mat = rng.random((nb * bs, nb * bs))
        s = ref.BlockSystem(*([bs] * nb))
        for i in range(nb):
            for j in range(nb):
                s.add_block(i, j, mat[bs * i : bs * (i + 1), bs * j : bs * (j + 1)])
        lhs = rng.random(nb * bs)
        rhs = mat @ lhs
        s.decompose(0)
        out[f"c{k}_matrix"] = mat
        out[f"c{k}_bs"] = np.int64(bs)
        out[f"c{k}_rhs"] = rhs
        out[f"c{k}_factors"] = np.concatenate(
            [s.get_block(i, j).ravel() for i in range(nb) for j in s.get_row_block_indices(i)]
        )
        out[f"c{k}_x"] = s.solve(rhs)
        out[f"c{k}_ops"] = _ops(s)
        k += 1
    out["count"] = np.int64(k)
    return out


def main():
    ref = load_reference()
    np.savez_compressed(HERE / "mesh16_p4.npz", **mesh_case(ref, 16, 4, seed=0, nrhs=1, full_rows=40))
    p6 = meshgen.random_orders(6, 2, 10, seed=5)
    np.savez_compressed(HERE / "mesh6_prand.npz", p=p6, **mesh_case(ref, 6, p6, seed=5, nrhs=4, full_rows=30, tail_rows=3))
    np.savez_compressed(HERE / "random_orderings.npz", **random_orderings(ref))
    np.savez_compressed(HERE / "dense_blocks.npz", **dense_blocks(ref))
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
