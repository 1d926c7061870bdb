"""Python-level drivers over the fine-grained ``BlockSystem`` methods.

The same helpers the reference ships in ``python/hybsol/system.py``: operation records,
a breadth-first decomposition driven from Python (``decompose_block_system_c``) and the
matching solve (``solve_decomposed_c``). They are a cross-check of ``BlockSystem.decompose``
and ``BlockSystem.solve``, not a fast path: every step is one call into ``hybsol._mod``,
whose block products and factorisations run on the GPU.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence

import numpy as np
import numpy.typing as npt

from hybsol._mod import BlockSystem

__all__ = [
    "BlockSystem",
    "OperationInvDiag",
    "OperationEliminate",
    "TargetRow",
    "decompose_block_system_c",
    "solve_decomposed_c",
]


@dataclass(frozen=True)
class OperationInvDiag:
    """Apply the inverse of a factored diagonal block (``python/hybsol/system.py:12-27``).

    Parameters
    ----------
    block_index : int
        Row whose diagonal block is applied.
    """

    block_index: int

    def __init__(self, block_index: int) -> None:
        object.__setattr__(self, "block_index", int(block_index))


@dataclass(frozen=True)
class OperationEliminate:
    """Eliminate a target row with a source row (``python/hybsol/system.py:30-55``).

    Parameters
    ----------
    target_block_index : int
        Row being eliminated.
    source_block_index : int
        Row used for the elimination; its block in the target row is the multiplier.
    """

    target_block_index: int
    source_block_index: int

    def __init__(self, target_block_index: int, source_block_index: int) -> None:
        object.__setattr__(self, "target_block_index", int(target_block_index))
        object.__setattr__(self, "source_block_index", int(source_block_index))


_Operation = OperationInvDiag | OperationEliminate


@dataclass(frozen=True)
class TargetRow:
    """A row still to be eliminated and the first column it needs (``system.py:61-66``)."""

    index: int
    first_entry: int


def _finish_row(system: BlockSystem, row: int, operations: list) -> None:
    system.decompose_diagonal(row)
    system.row_apply_decomposition(row)
    operations.append(OperationInvDiag(row))


def decompose_block_system_c(system: BlockSystem) -> tuple[tuple[_Operation, ...], BlockSystem]:
    """LU-decompose a block system in rounds, in place (``python/hybsol/system.py:69-154``).

    Rows without blocks left of the diagonal are factored first. Each round then takes
    every waiting row whose next needed source row is already factored (scanning the
    waiting list from its end), eliminates that one source, and either finishes the row
    or puts it back with its next needed column.

    Returns
    -------
    tuple of operations
        The operations that map the system to its upper factor (the inverse of the lower
        factor, applied in order).
    BlockSystem
        The same system, now holding the factors.
    """
    if not system.is_valid():
        raise ValueError("Block system is not valid.")
    operations: list[_Operation] = []
    finished: set[int] = set()
    waiting: list[TargetRow] = []
    for row, free in enumerate(system.no_lower_connections()):
        if free:
            _finish_row(system, row, operations)
            finished.add(row)
        else:
            waiting.append(TargetRow(row, system.first_column(row)))

    while waiting:
        available = set(finished)
        round_ops: list[OperationEliminate] = []
        deferred: list[TargetRow] = []
        for target in reversed(waiting):
            if target.first_entry in available:
                round_ops.append(OperationEliminate(target.index, target.first_entry))
            else:
                deferred.append(target)
        if not round_ops:
            raise RuntimeError("No row can be eliminated: the system's dependencies are cyclic.")
        waiting = deferred
        for op in round_ops:
            operations.append(op)
            tgt, src = op.target_block_index, op.source_block_index
            system.eliminate_row(src, tgt, system.get_block(tgt, src))
            nxt = system.get_next_column_index(tgt, src)
            if nxt == tgt:
                _finish_row(system, tgt, operations)
                finished.add(tgt)
            else:
                waiting.append(TargetRow(tgt, nxt))
    return tuple(operations), system


def solve_decomposed_c(
    decomposed: BlockSystem, operations: Sequence[_Operation], forcing: npt.ArrayLike
) -> npt.NDArray[np.float64]:
    """Solve with a system decomposed by :func:`decompose_block_system_c`
    (``python/hybsol/system.py:157-199``): replay the operations, then back-substitute
    with the upper blocks (identity diagonal) from the last row up."""
    y = np.array(forcing, dtype=np.float64, copy=True)
    bounds = np.concatenate([[0], np.cumsum(decomposed.block_sizes.astype(np.int64))])
    parts = [y[bounds[i] : bounds[i + 1]] for i in range(decomposed.n_blocks)]
    for op in operations:
        if isinstance(op, OperationInvDiag):
            i = op.block_index
            decomposed.solve_diagonal(i, parts[i], parts[i])
        elif isinstance(op, OperationEliminate):
            t, s = op.target_block_index, op.source_block_index
            parts[t] -= decomposed.get_block(t, s) @ parts[s]
        else:
            raise TypeError(f"Invalid operation type {type(op)}")
    for row in range(decomposed.n_blocks - 2, -1, -1):
        for col in reversed(decomposed.get_row_block_indices(row)):
            if col == row:
                break
            parts[row] -= decomposed.get_block(row, col) @ parts[col]
    return np.concatenate(parts)
