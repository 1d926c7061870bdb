"""The multi-system path across ranks, on CPU with two `gloo` ranks.

Independent systems are split across ranks by LPT on their exact factorization flops; no
data-path collective is needed, only a gather of per-system results. Each rank here runs
the host symbolic phase of its systems (the part that needs no GPU) and the ranks check
that every system was processed exactly once and that the per-rank loads are balanced.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import PKG, ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    import sys

    for p in (str(ROOT), str(PKG)):
        if p not in sys.path:
            sys.path.insert(0, p)
    from datetime import timedelta

    import torch

    from hybsol.b200 import meshgen, native, shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    specs = meshgen.many_mesh_specs(12, side_range=(2, 7), p_range=(2, 4), seed=3)
    flops = []
    for side, p in specs:
        m, _ = meshgen.mesh_system(side, p, seed=0)
        order = native.compute_ordering(m.row_ptr, m.cols)
        pm = m.permuted(order)
        flops.append(native.analyze(pm.sizes, pm.row_ptr, pm.cols)["factor_flops"])
    assignment = shard.assign_lpt(flops, world)
    mine = assignment[rank]
    results = torch.zeros(len(specs), dtype=torch.float64)
    for i in mine:
        side, p = specs[i]
        m, _ = meshgen.mesh_system(side, p, seed=i)
        order = native.compute_ordering(m.row_ptr, m.cols)
        pm = m.permuted(order)
        a = native.analyze(pm.sizes, pm.row_ptr, pm.cols)
        results[i] = a["filled_blocks"] + 1.0  # marks "processed by some rank"
    dist.all_reduce(results, op=dist.ReduceOp.SUM)
    counts = torch.zeros(len(specs), dtype=torch.float64)
    counts[mine] = 1.0
    dist.all_reduce(counts, op=dist.ReduceOp.SUM)
    if rank == 0:
        np.savez(out_path, results=results.numpy(), counts=counts.numpy(), flops=np.array(flops))
    dist.barrier()
    dist.destroy_process_group()


def test_lpt_assignment_properties():
    from hybsol.b200 import shard

    w = [9, 7, 6, 5, 5, 4, 3, 2, 1, 1]
    a = shard.assign_lpt(w, 3)
    assert sorted(i for r in a for i in r) == list(range(len(w)))
    ld = shard.loads(w, a)
    assert max(ld) <= 4 / 3 * (sum(w) / 3) + max(w)
    assert shard.assign_lpt(w, 1) == [list(range(len(w)))]
    assert shard.assign_lpt([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard.assign_lpt(w, 0)


def test_two_ranks_cover_every_system_once(tmp_path):
    out = tmp_path / "res.npz"
    mp.spawn(_worker, args=(2, _free_port(), str(out)), nprocs=2, join=True)
    r = np.load(out)
    assert np.all(r["counts"] == 1.0)
    assert np.all(r["results"] > 1.0)
