"""ctypes access to the C ABI of ``libhybsol_b200.so`` (``include/hybsol_b200.h``).

This is the same boundary the ``hybsol._mod`` extension binds, exposed to Python for
callers that hold device buffers (e.g. torch tensors) or want the raw entry points.
Loading fails loudly when the library has not been built: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent.parent / "libhybsol_b200.so"

FP64 = 0
MIXED = 1
MEMORY_HOST = 0
MEMORY_DEVICE = 1
ORDERING = {"first": 0, "greedy": 1, "balanced": 2}

SUCCESS = 0
NOT_CONVERGED = 23
TOO_LARGE = 24
DEVICE_TIMEOUT = 25

# hyb_option values (include/hybsol_b200.h)
OPTION_LOOKAHEAD = 0
OPTION_TENSOR_CORE_MIXED = 1
OPTION_DATAFLOW_SOLVE = 2
OPTION_WAIT_LIMIT_NS = 3
OPTION_WITHHOLD_ROW = 4
OPTION_REFINEMENT = 5  # 0 auto (refinement, then FGMRES when it stalls), 1 refinement only, 2 FGMRES
OPTION_FP64_REFINEMENT = 6
OPTION_KRYLOV_RESTART = 7
OPTION_GROWTH_LIMIT = 8
OPTION_BLOCK_SCALING = 9
OPTION_ALTERNATE_WALK = 10
OPTION_UPDATE_KERNEL = 11  # -1 tuned, 0 32x32 SIMT, 1 64x64 SIMT, 2 DMMA
OPTION_PIVOT_LU_ONCE = 12
OPTION_FP64_MMA_SHAPE = 13
OPTION_PAIR_PASSES = 14  # mixed form: two consecutive pivots per tensor-core pass
OPTION_ROW_PIVOTS = 15  # 64-row pivots: -1 per precision, 0 256-thread kernels, 1 blocked, 2 inverse + products
OPTION_UPDATE_SM_RESERVE = 16  # mixed form: SMs the two-pivot update leaves free for the pivot work

_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)


class DecomposeInfo(ctypes.Structure):
    _fields_ = [
        ("n_levels", ctypes.c_uint64),
        ("filled_blocks", ctypes.c_uint64),
        ("factor_values", ctypes.c_uint64),
        ("factor_flops", ctypes.c_double),
        ("zero_pivots", ctypes.c_uint64),
        ("non_finite", ctypes.c_uint64),
        ("first_bad_pivot", ctypes.c_int64),
        ("growth_fp64", ctypes.c_uint64),
        ("growth_kept", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class SolveInfo(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_uint32),
        ("relative_residual", ctypes.c_double),
        ("krylov_iterations", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {
            "iterations": self.iterations,
            "relative_residual": self.relative_residual,
            "krylov_iterations": self.krylov_iterations,
        }


class Condition(ctypes.Structure):
    _fields_ = [
        ("kappa1", ctypes.c_double),
        ("norm1", ctypes.c_double),
        ("inv_norm1", ctypes.c_double),
        ("solves", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Analysis(ctypes.Structure):
    _fields_ = [
        ("filled_blocks", ctypes.c_uint64),
        ("factor_values", ctypes.c_uint64),
        ("n_levels", ctypes.c_uint64),
        ("nops", ctypes.c_uint64),
        ("slab_bytes_fp64", ctypes.c_uint64),
        ("factor_flops", ctypes.c_double),
        ("pair_levels", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class KernelProfile(ctypes.Structure):
    _fields_ = [
        ("launches", ctypes.c_uint64),
        ("total_ms", ctypes.c_double),
        ("flops", ctypes.c_double),
        ("c_elems", ctypes.c_double),
        ("ab_elems", ctypes.c_double),
        ("levels", ctypes.c_uint64),
        ("passes", ctypes.c_uint64),
        ("pivots_timed", ctypes.c_uint64),
        ("pivot_ms", ctypes.c_double),
        ("pivot_units", ctypes.c_uint64),
        ("pivot_levels", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class HybError(RuntimeError):
    """A C-ABI call returned a non-success status."""

    def __init__(self, status: int, what: str):
        self.status = status
        detail = lib().hyb_last_cuda_error().decode() if status in (2, 16, 17, 19, 24, 25) else ""
        msg = f"{what} failed: {lib().hyb_status_string(status).decode()} ({status})"
        super().__init__(msg + (f": {detail}" if detail else ""))


_lib = None

EXPORTS = {
    "hyb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "hyb_last_cuda_error": (ctypes.c_char_p, []),
    "hyb_version": (ctypes.c_int, []),
    "hyb_device_available": (ctypes.c_int, []),
    "hyb_compute_ordering": (ctypes.c_int, [ctypes.c_uint64, _u64p, _u64p, ctypes.c_int, ctypes.c_uint64, _u64p]),
    "hyb_analyze": (
        ctypes.c_int,
        [ctypes.c_uint64, _u64p, _u64p, _u64p, ctypes.POINTER(Analysis), _u64p, _u64p, _i64p],
    ),
    "hyb_system_create": (ctypes.c_int, [ctypes.c_uint64, _u64p, _u64p, _u64p, ctypes.POINTER(ctypes.c_void_p)]),
    "hyb_system_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "hyb_system_copy": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "hyb_system_set_values": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "hyb_system_value_count": (ctypes.c_uint64, [ctypes.c_void_p]),
    "hyb_system_dof": (ctypes.c_uint64, [ctypes.c_void_p]),
    "hyb_system_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "hyb_system_set_option": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64]),
    "hyb_decompose": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(DecomposeInfo)]),
    "hyb_solve": (
        ctypes.c_int,
        [
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_uint64,
            ctypes.c_int,
            ctypes.c_double,
            ctypes.c_uint32,
            ctypes.POINTER(SolveInfo),
        ],
    ),
    "hyb_residual": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int],
    ),
    "hyb_solve_transpose": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int],
    ),
    "hyb_condition_estimate": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Condition)]),
    "hyb_system_set_segments": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _u64p]),
    "hyb_tuned_kernels": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int32)]),
    "hyb_system_add_blocks": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_uint64, _u64p, _u64p, ctypes.c_void_p, ctypes.c_int],
    ),
    "hyb_block_gemm_batched": (
        ctypes.c_int,
        [
            ctypes.c_uint64,
            ctypes.c_uint64,
            ctypes.c_uint64,
            _u64p,
            ctypes.c_void_p,
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.c_int,
            ctypes.c_int,
        ],
    ),
    "hyb_block_lu_solve_batched": (
        ctypes.c_int,
        [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, _u64p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int],
    ),
    "hyb_segment_results": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), _f64p]),
    "hyb_row_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _u64p]),
    "hyb_row_cols": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _u64p]),
    "hyb_get_block": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, _f64p]),
    "hyb_operations": (ctypes.c_int, [ctypes.c_void_p, _u64p, _i64p]),
    "hyb_last_launch_count": (ctypes.c_uint64, [ctypes.c_void_p]),
    "hyb_profile_enable": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "hyb_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(KernelProfile)]),
    "hyb_block_lu": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int]),
    "hyb_block_lu_solve": (
        ctypes.c_int,
        [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int],
    ),
    "hyb_block_gemm": (
        ctypes.c_int,
        [
            ctypes.c_uint64,
            ctypes.c_uint64,
            ctypes.c_uint64,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_int,
            ctypes.c_int,
        ],
    ),
}


def lib() -> ctypes.CDLL:
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C hybridized-solver_b200`")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in EXPORTS.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def _check(status: int, what: str, ok=(SUCCESS,)) -> int:
    if status not in ok:
        raise HybError(status, what)
    return status


def _ptr(a):
    """Raw address of a numpy array or a torch tensor (anything with data_ptr())."""
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)


def device_available() -> bool:
    return bool(lib().hyb_device_available())


def compute_ordering(row_ptr, cols, strategy: str = "first", max_colors: int = 0) -> np.ndarray:
    rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
    cc = np.ascontiguousarray(cols, dtype=np.uint64)
    n = len(rp) - 1
    out = np.empty(n, dtype=np.uint64)
    st = lib().hyb_compute_ordering(
        n, rp.ctypes.data_as(_u64p), cc.ctypes.data_as(_u64p), ORDERING[strategy], max_colors, out.ctypes.data_as(_u64p)
    )
    if st == 3:
        raise ValueError(f"Maximum number of colors ({max_colors}) exceeded.")
    _check(st, "hyb_compute_ordering")
    return out


def analyze(sizes, row_ptr, cols, pattern: bool = False, operations: bool = False):
    """Host-only symbolic phase. Returns the statistics dict, plus ``filled_row_ptr`` /
    ``filled_cols`` when ``pattern`` and ``ops`` (pairs, -1 for INVDIA) when ``operations``."""
    s = np.ascontiguousarray(sizes, dtype=np.uint64)
    rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
    cc = np.ascontiguousarray(cols, dtype=np.uint64)
    info = Analysis()
    args = (len(s), s.ctypes.data_as(_u64p), rp.ctypes.data_as(_u64p), cc.ctypes.data_as(_u64p), ctypes.byref(info))
    _check(lib().hyb_analyze(*args, None, None, None), "hyb_analyze")
    out = info.as_dict()
    if pattern or operations:
        frp = np.empty(len(s) + 1, dtype=np.uint64) if pattern else None
        fc = np.empty(max(1, info.filled_blocks), dtype=np.uint64) if pattern else None
        ops = np.empty(2 * max(1, info.nops), dtype=np.int64) if operations else None
        _check(
            lib().hyb_analyze(
                *args,
                frp.ctypes.data_as(_u64p) if pattern else None,
                fc.ctypes.data_as(_u64p) if pattern else None,
                ops.ctypes.data_as(_i64p) if operations else None,
            ),
            "hyb_analyze",
        )
        if pattern:
            out["filled_row_ptr"] = frp
            out["filled_cols"] = fc[: info.filled_blocks]
        if operations:
            out["ops"] = ops[: 2 * info.nops].reshape(-1, 2)
    return out


class NativeSystem:
    """One block system on the device, driven through the C ABI."""

    def __init__(self, sizes, row_ptr, cols, _handle=None):
        if _handle is not None:
            self._h = _handle
        else:
            s = np.ascontiguousarray(sizes, dtype=np.uint64)
            rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
            cc = np.ascontiguousarray(cols, dtype=np.uint64)
            h = ctypes.c_void_p()
            _check(
                lib().hyb_system_create(
                    len(s), s.ctypes.data_as(_u64p), rp.ctypes.data_as(_u64p), cc.ctypes.data_as(_u64p), ctypes.byref(h)
                ),
                "hyb_system_create",
            )
            self._h = h
        self.dof = int(lib().hyb_system_dof(self._h))
        self.value_count = int(lib().hyb_system_value_count(self._h))

    @classmethod
    def from_matrix(cls, mat) -> "NativeSystem":
        """From a :class:`hybsol.b200.meshgen.BlockMatrix`, values loaded."""
        s = cls(mat.sizes, mat.row_ptr, mat.cols)
        s.set_values(mat.vals)
        return s

    def close(self):
        if getattr(self, "_h", None):
            lib().hyb_system_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def copy(self) -> "NativeSystem":
        h = ctypes.c_void_p()
        _check(lib().hyb_system_copy(self._h, ctypes.byref(h)), "hyb_system_copy")
        return NativeSystem(None, None, None, _handle=h)

    def set_lookahead(self, enable: bool):
        _check(lib().hyb_system_set_option(self._h, 0, 1 if enable else 0), "hyb_system_set_option")

    def set_tensor_core_mixed(self, enable: bool):
        _check(lib().hyb_system_set_option(self._h, 1, 1 if enable else 0), "hyb_system_set_option")

    def set_dataflow_solve(self, enable: bool):
        """Dataflow substitution (one cooperative launch per direction) or one launch per stage."""
        _check(lib().hyb_system_set_option(self._h, 2, 1 if enable else 0), "hyb_system_set_option")

    def set_option(self, option: int, value: int):
        """Any ``hyb_option`` of the handle (``OPTION_*`` above)."""
        _check(lib().hyb_system_set_option(self._h, option, int(value)), "hyb_system_set_option")

    @property
    def stream(self) -> int:
        return int(lib().hyb_system_stream(self._h) or 0)

    def set_values(self, values, device: bool = False):
        if not device:
            values = np.ascontiguousarray(values, dtype=np.float64)
            assert values.size == self.value_count
        _check(
            lib().hyb_system_set_values(self._h, _ptr(values), MEMORY_DEVICE if device else MEMORY_HOST),
            "hyb_system_set_values",
        )

    def decompose(self, precision: int = FP64) -> dict:
        info = DecomposeInfo()
        _check(lib().hyb_decompose(self._h, precision, ctypes.byref(info)), "hyb_decompose")
        return info.as_dict()

    def solve(self, b, tol: float = 1e-12, max_iter: int = 50, out=None, residual: bool = True):
        """Solve for host ``b`` of shape (dof,) or (dof, k); returns (x, info)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        x = np.empty_like(b) if out is None else out
        info = SolveInfo()
        st = lib().hyb_solve(
            self._h, _ptr(b), _ptr(x), nrhs, MEMORY_HOST, tol if residual else 0.0, max_iter, ctypes.byref(info)
        )
        _check(st, "hyb_solve", ok=(SUCCESS, NOT_CONVERGED))
        d = info.as_dict()
        d["converged"] = st == SUCCESS
        return x, d

    def solve_device(self, b, x, nrhs: int, tol: float = 1e-12, max_iter: int = 50, residual: bool = False) -> dict:
        """Solve with device pointers (torch tensors) ``b`` and ``x``."""
        info = SolveInfo()
        st = lib().hyb_solve(
            self._h, _ptr(b), _ptr(x), nrhs, MEMORY_DEVICE, tol if residual else 0.0, max_iter, ctypes.byref(info)
        )
        _check(st, "hyb_solve", ok=(SUCCESS, NOT_CONVERGED))
        d = info.as_dict()
        d["converged"] = st == SUCCESS
        return d

    def solve_transpose(self, b) -> np.ndarray:
        """Solve A^T x = b (host arrays) with the FP64 factors."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty_like(b)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        _check(lib().hyb_solve_transpose(self._h, _ptr(b), _ptr(x), nrhs, MEMORY_HOST), "hyb_solve_transpose")
        return x

    def condition_estimate(self) -> dict:
        """1-norm condition estimate from the FP64 factors (kappa1, norm1, inv_norm1, solves)."""
        c = Condition()
        _check(lib().hyb_condition_estimate(self._h, ctypes.byref(c)), "hyb_condition_estimate")
        return c.as_dict()

    def add_blocks(self, rows, cols, values, device: bool = False):
        """Bulk assembly on the device: block i at (rows[i], cols[i]) gets its row-major
        values from ``values`` (blocks concatenated in input order) added; repeats sum in
        input order. ``values`` is a host array, or a device tensor with ``device=True``."""
        r = np.ascontiguousarray(rows, dtype=np.uint64)
        c = np.ascontiguousarray(cols, dtype=np.uint64)
        if not device:
            values = np.ascontiguousarray(values, dtype=np.float64)
        st = lib().hyb_system_add_blocks(
            self._h, len(r), r.ctypes.data_as(_u64p), c.ctypes.data_as(_u64p), _ptr(values),
            MEMORY_DEVICE if device else MEMORY_HOST,
        )
        if st == 1:
            raise KeyError("a block is not in the system's pattern")
        _check(st, "hyb_system_add_blocks")

    def tuned_kernels(self, precision: int) -> np.ndarray:
        """Tuned generic update kernel per size bucket (7 x 7: pivot class, target class), -1 untuned."""
        out = np.empty(49, dtype=np.int32)
        _check(lib().hyb_tuned_kernels(self._h, precision, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
               "hyb_tuned_kernels")
        return out.reshape(7, 7)

    def set_segments(self, offsets):
        """Independent systems stacked in this handle: segment s holds the unknowns
        [offsets[s], offsets[s+1]). Refinement then converges every segment on its own."""
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        self._nseg = max(0, len(off) - 1)
        _check(
            lib().hyb_system_set_segments(self._h, self._nseg, off.ctypes.data_as(_u64p) if self._nseg else None),
            "hyb_system_set_segments",
        )

    def segment_results(self, nrhs: int = 1):
        """(first converged step per segment and column, UINT32_MAX if never; final relative
        residuals), each of shape (nseg, nrhs), after a refined solve."""
        it = np.empty((self._nseg, nrhs), dtype=np.uint32)
        rr = np.empty((self._nseg, nrhs), dtype=np.float64)
        _check(
            lib().hyb_segment_results(
                self._h, it.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), rr.ctypes.data_as(_f64p)
            ),
            "hyb_segment_results",
        )
        return it, rr

    def residual(self, b, x) -> np.ndarray:
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        r = np.empty_like(b)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        _check(lib().hyb_residual(self._h, _ptr(b), _ptr(x), _ptr(r), nrhs, MEMORY_HOST), "hyb_residual")
        return r

    def row_cols(self, row: int) -> tuple:
        cnt = ctypes.c_uint64()
        _check(lib().hyb_row_count(self._h, row, ctypes.byref(cnt)), "hyb_row_count")
        out = np.empty(cnt.value, dtype=np.uint64)
        _check(lib().hyb_row_cols(self._h, row, out.ctypes.data_as(_u64p)), "hyb_row_cols")
        return tuple(int(c) for c in out)

    def get_block(self, row: int, col: int, shape) -> np.ndarray:
        out = np.empty(shape, dtype=np.float64)
        _check(lib().hyb_get_block(self._h, row, col, out.ctypes.data_as(_f64p)), "hyb_get_block")
        return out

    def operations(self) -> tuple:
        n = ctypes.c_uint64()
        _check(lib().hyb_operations(self._h, ctypes.byref(n), None), "hyb_operations")
        ops = np.empty(2 * n.value, dtype=np.int64)
        _check(lib().hyb_operations(self._h, ctypes.byref(n), ops.ctypes.data_as(_i64p)), "hyb_operations")
        return tuple((int(r),) if c < 0 else (int(r), int(c)) for r, c in ops.reshape(-1, 2))

    def last_launch_count(self) -> int:
        return int(lib().hyb_last_launch_count(self._h))


def block_lu(a: np.ndarray) -> np.ndarray:
    m = np.array(a, dtype=np.float64, order="C", copy=True)
    _check(lib().hyb_block_lu(m.shape[0], _ptr(m), MEMORY_HOST), "hyb_block_lu")
    return m


def block_lu_solve(lu: np.ndarray, b: np.ndarray) -> np.ndarray:
    lu = np.ascontiguousarray(lu, dtype=np.float64)
    b2 = np.ascontiguousarray(b, dtype=np.float64)
    out = np.empty_like(b2)
    ncols = 1 if b2.ndim == 1 else b2.shape[1]
    _check(
        lib().hyb_block_lu_solve(lu.shape[0], _ptr(lu), ncols, _ptr(b2), _ptr(out), MEMORY_HOST), "hyb_block_lu_solve"
    )
    return out
