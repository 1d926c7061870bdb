"""Python access to the two CPU checkers.

TEST INFRASTRUCTURE ONLY. ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs
of ``bench.py`` may import this module, and only to check against it or to time
the reference's CPU path. The product (``hybridized-solver_b200/``) never does.

* :class:`OracleSystem` wraps ``_build/libhyb_oracle.so``, the C restatement of the
  reference's block LU (``hyb_oracle.c``, which cites the reference line by line).
* :func:`load_reference` imports the reference extension itself, compiled from
  j4nr0th/hybridized-solver's own ``src/*.c`` into ``_ref/hybsol_ref/`` by
  ``make -C oracle ref`` (only possible where the reference sources are mounted;
  the compiled module travels with the repository like any other built file).
"""

from __future__ import annotations

import ctypes
import importlib.machinery
import importlib.util
import os
import sysconfig
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "_build" / "libhyb_oracle.so"
REF_MOD = HERE / "_ref" / "hybsol_ref" / ("_mod" + sysconfig.get_config_var("EXT_SUFFIX"))

STRATEGIES = {"first": 0, "greedy": 1, "balanced": 2}

_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)
_lib = None


def _p(arr, typ):
    return arr.ctypes.data_as(typ)


def port_library() -> ctypes.CDLL:
    """Load (once) the C restatement; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not PORT_LIB.exists():
        raise FileNotFoundError(f"{PORT_LIB} is missing: run `make -C oracle port`")
    lib = ctypes.CDLL(str(PORT_LIB))
    vp = ctypes.c_void_p
    u64 = ctypes.c_uint64
    sig = {
        "orc_create": (vp, [u64, _u64p]),
        "orc_destroy": (None, [vp]),
        "orc_copy": (vp, [vp]),
        "orc_n_blocks": (u64, [vp]),
        "orc_block_size": (u64, [vp, u64]),
        "orc_row_count": (u64, [vp, u64]),
        "orc_row_cols": (None, [vp, u64, _u64p]),
        "orc_add_block": (ctypes.c_int, [vp, u64, u64, _f64p]),
        "orc_get_block": (ctypes.c_int, [vp, u64, u64, _f64p]),
        "orc_total_blocks": (u64, [vp]),
        "orc_export": (None, [vp, _u64p, _u64p, _f64p]),
        "orc_export_value_count": (u64, [vp]),
        "orc_lu_decompose": (None, [u64, _f64p]),
        "orc_lu_solve": (None, [u64, _f64p, u64, _f64p, _f64p]),
        "orc_matmul": (None, [u64, u64, u64, _f64p, _f64p, _f64p]),
        "orc_eliminate_row": (ctypes.c_int, [vp, u64, u64, _f64p]),
        "orc_decompose_diagonal": (None, [vp, u64]),
        "orc_apply_diagonal_inverse": (None, [vp, u64]),
        "orc_decompose": (ctypes.c_int, [vp]),
        "orc_nops": (u64, [vp]),
        "orc_get_ops": (None, [vp, _i64p]),
        "orc_solve": (ctypes.c_int, [vp, _f64p]),
        "orc_compute_ordering": (ctypes.c_int, [u64, _u64p, _u64p, ctypes.c_int, u64, _u64p]),
        "orc_reorder_blocks": (ctypes.c_int, [vp, _u64p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class OracleSystem:
    """A block system held by the C restatement (mirrors the reference's storage)."""

    def __init__(self, block_sizes, _handle=None):
        lib = port_library()
        self._lib = lib
        if _handle is not None:
            self._h = _handle
        else:
            sizes = np.ascontiguousarray(block_sizes, dtype=np.uint64)
            self._h = lib.orc_create(len(sizes), _p(sizes, _u64p))
            if not self._h:
                raise ValueError("invalid block sizes")
        n = lib.orc_n_blocks(self._h)
        self.block_sizes = np.array([lib.orc_block_size(self._h, i) for i in range(n)], dtype=np.uint64)
        self.n_blocks = int(n)

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.orc_destroy(self._h)
            self._h = None

    @classmethod
    def from_csr(cls, block_sizes, row_ptr, cols, values) -> "OracleSystem":
        """Build from a block-CSR pattern with row-major block values concatenated in order."""
        s = cls(block_sizes)
        sizes = np.asarray(block_sizes, dtype=np.int64)
        vals = np.ascontiguousarray(values, dtype=np.float64)
        pos = 0
        for r in range(len(sizes)):
            for j in range(int(row_ptr[r]), int(row_ptr[r + 1])):
                c = int(cols[j])
                cnt = int(sizes[r] * sizes[c])
                s.add_block(r, c, vals[pos : pos + cnt].reshape(sizes[r], sizes[c]))
                pos += cnt
        return s

    def copy(self) -> "OracleSystem":
        return OracleSystem(None, _handle=self._lib.orc_copy(self._h))

    def add_block(self, row, col, val):
        v = np.ascontiguousarray(val, dtype=np.float64)
        rc = self._lib.orc_add_block(self._h, row, col, _p(v, _f64p))
        if rc:
            raise ValueError(f"add_block failed with {rc}")

    def get_block(self, row, col):
        out = np.empty((int(self.block_sizes[row]), int(self.block_sizes[col])))
        rc = self._lib.orc_get_block(self._h, row, col, _p(out, _f64p))
        if rc:
            raise ValueError(f"no block ({row}, {col})")
        return out

    def get_row_block_indices(self, row):
        cnt = self._lib.orc_row_count(self._h, row)
        out = np.empty(cnt, dtype=np.uint64)
        self._lib.orc_row_cols(self._h, row, _p(out, _u64p))
        return tuple(int(c) for c in out)

    def export(self):
        """Return (row_ptr, cols, values) of the stored blocks, rows in order."""
        nb = self._lib.orc_total_blocks(self._h)
        nv = self._lib.orc_export_value_count(self._h)
        row_ptr = np.empty(self.n_blocks + 1, dtype=np.uint64)
        cols = np.empty(nb, dtype=np.uint64)
        vals = np.empty(nv, dtype=np.float64)
        self._lib.orc_export(self._h, _p(row_ptr, _u64p), _p(cols, _u64p), _p(vals, _f64p))
        return row_ptr, cols, vals

    def eliminate_row(self, row_src, row_tgt, val):
        v = np.ascontiguousarray(val, dtype=np.float64)
        rc = self._lib.orc_eliminate_row(self._h, row_tgt, row_src, _p(v, _f64p))
        if rc:
            raise ValueError(f"eliminate_row failed with {rc}")

    def decompose(self):
        rc = self._lib.orc_decompose(self._h)
        if rc:
            raise RuntimeError(f"Block system decomposition failed with error {rc}.")

    def operations(self):
        n = self._lib.orc_nops(self._h)
        ops = np.empty(2 * n, dtype=np.int64)
        self._lib.orc_get_ops(self._h, _p(ops, _i64p))
        return tuple((int(r),) if c < 0 else (int(r), int(c)) for r, c in ops.reshape(-1, 2))

    def solve(self, val):
        v = np.array(val, dtype=np.float64, copy=True)
        if v.ndim == 1:
            rc = self._lib.orc_solve(self._h, _p(v, _f64p))
            if rc:
                raise RuntimeError("system not decomposed")
            return v
        out = np.empty_like(v)
        for j in range(v.shape[1]):
            col = np.ascontiguousarray(v[:, j])
            self._lib.orc_solve(self._h, _p(col, _f64p))
            out[:, j] = col
        return out

    def compute_reordering(self, strategy="first", max_colors=0):
        row_ptr, cols, _ = self.export()
        return compute_ordering(row_ptr, cols, strategy, max_colors)

    def reorder_blocks(self, order):
        o = np.ascontiguousarray(order, dtype=np.uint64)
        rc = self._lib.orc_reorder_blocks(self._h, _p(o, _u64p))
        if rc:
            raise ValueError(f"reorder failed with {rc}")
        self.block_sizes = np.array(
            [self._lib.orc_block_size(self._h, i) for i in range(self.n_blocks)], dtype=np.uint64
        )


def compute_ordering(row_ptr, cols, strategy="first", max_colors=0):
    """Integer coloring order of a block-CSR pattern, as the reference computes it."""
    lib = port_library()
    rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
    cc = np.ascontiguousarray(cols, dtype=np.uint64)
    n = len(rp) - 1
    if max_colors == 0:
        max_colors = int(np.max(np.diff(rp))) if n else 0
    out = np.empty(n, dtype=np.uint64)
    rc = lib.orc_compute_ordering(n, _p(rp, _u64p), _p(cc, _u64p), STRATEGIES[strategy], max_colors, _p(out, _u64p))
    if rc == 3:
        raise ValueError(f"Maximum number of colors ({max_colors}) exceeded.")
    if rc:
        raise RuntimeError(f"ordering failed with {rc}")
    return out


def lu_decompose(a):
    lib = port_library()
    m = np.array(a, dtype=np.float64, copy=True, order="C")
    lib.orc_lu_decompose(m.shape[0], _p(m, _f64p))
    return m


def lu_solve(lu, b):
    lib = port_library()
    lu = np.ascontiguousarray(lu, dtype=np.float64)
    b2 = np.ascontiguousarray(b, dtype=np.float64)
    ncols = 1 if b2.ndim == 1 else b2.shape[1]
    out = np.empty_like(b2)
    lib.orc_lu_solve(lu.shape[0], _p(lu, _f64p), ncols, _p(b2, _f64p), _p(out, _f64p))
    return out


def reference_available() -> bool:
    return REF_MOD.exists()


def load_reference():
    """Import the reference extension compiled from its own sources (oracle/_ref)."""
    if not REF_MOD.exists():
        raise FileNotFoundError(f"{REF_MOD} is missing: run `make -C oracle ref` where the reference is mounted")
    name = "hybsol_ref._mod"
    loader = importlib.machinery.ExtensionFileLoader(name, str(REF_MOD))
    spec = importlib.util.spec_from_file_location(name, str(REF_MOD), loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def factor_flops(sizes, rows) -> float:
    """Algorithmic flops of the block LU from a factored pattern: for every pivot k of m
    rows, 2/3 m^3 (diagonal LU) + 2 m^2 U (row solve over the U columns of its upper
    blocks) + 2 L m U (Schur updates, L the rows of its lower column). ``rows[k]`` are the
    columns of block row k after the decomposition (the fill included), e.g. the reference's
    ``get_row_block_indices`` (src/block_system.c:312-349) of a decomposed system."""
    sizes = np.asarray(sizes, dtype=np.float64)
    n = len(sizes)
    up = np.zeros(n)
    lc = np.zeros(n)
    for k in range(n):
        cols = np.asarray(rows[k], dtype=np.int64)
        upper = cols[cols > k]
        lower = cols[cols < k]
        up[k] = sizes[upper].sum()
        # block (k, j) with j < k puts row k into the lower column of pivot j
        np.add.at(lc, lower, sizes[k])
    m = sizes
    return float(np.sum(2.0 / 3.0 * m**3 + 2.0 * m * m * up + 2.0 * lc * m * up))
