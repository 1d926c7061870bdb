#!/usr/bin/env python
"""Benchmark: decompose + solve of a hybridized quad-mesh block system on B200.

Metric (the reference's headline): decompose+solve time in ms, FP32+refinement
("mixed") against plain FP64, to a relative FP64 residual of 1e-12, on one GPU.

Workload: the quad-mesh block system of the reference's hybridized solver, N x N
elements (default 128 x 128), order p (default 8): 64x64 element blocks, 8x8 edge blocks,
element<->edge couplings, seeded values, one right-hand side, ordered by the reference's
first-fit coloring (edges first). The 256 x 256 mesh of the original target needs 1.1 TB
of FP64 factors and cannot be held by one GPU; 128 x 128 (137.5 GB FP64) is the largest
that fits, so it is the default.

A step = load the values (device-resident for `value`, pinned host for `e2e`), factor,
and solve one right-hand side (the mixed form iterates refinement to 1e-12). The symbolic
phase (fill pattern and schedule) runs once per pattern before timing and is reported as
`analysis_ms`.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--mesh 128] [--p 8]
  python bench.py --impl reference ...   # the reference's own CPU path, rank 0 only

Under torchrun with N > 1 every rank factors its own copy (replicas: one system does
not shard), timing is max over ranks, and value is the per-step time (weak scaling).
"""

from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "hybridized-solver_b200"))

METRIC = "decompose+solve ms: FP32+refine vs plain FP64 on one B200 at 1e-12 residual"
TOL = 1e-12
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
CPU_SAMPLE_MESH = 20  # reference CPU sample: 20x20 elements at the same p
# DRAM bytes (read + write) per 64x64 FP32 target block of a tensor-core update stage,
# measured with ncu (dram__bytes_read.sum + dram__bytes_write.sum, one pass) on a 96x96
# p=8 stage, whose targets exceed L2: 245.3 MB for ~9,000 target blocks.
TC_DRAM_BYTES_PER_TARGET_BLOCK = 245.3e6 / 9000
# the two-pivot pass (k_update64_tc2) at 96x96 p=8: priority + rest launches of one pair,
# dram__bytes_read.sum + dram__bytes_write.sum (12.6 + 152.5 + 82.6 MB) over ~9,400 target blocks
TC2_DRAM_BYTES_PER_TARGET_BLOCK = 247.7e6 / 9400


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mesh", type=int, default=128)
    ap.add_argument(
        "--p",
        default="8",
        help="element order: an integer, or 'rand' for a per-element order drawn uniformly from 2..10 (seed 0)",
    )
    ap.add_argument("--nrhs", type=int, default=1, help="right-hand sides per solve (configs with 4 RHS)")
    ap.add_argument("--cpu-sample-mesh", type=int, default=CPU_SAMPLE_MESH)
    ap.add_argument(
        "--ref-threads",
        type=int,
        default=0,
        help="threads of the reference's decompose (default: every host core the process may use)",
    )
    ap.add_argument("--ref-child", nargs=6, metavar=("N", "P", "STEPS", "WARMUP", "THREADS", "OUT"), help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-profile", action="store_true", help="do not time the dominant kernel with events")
    ap.add_argument(
        "--profile-stride",
        type=int,
        default=32,
        help="time the Schur update of every n-th level with events (each event pair costs a few us of its stage)",
    )
    ap.add_argument(
        "--single",
        action="store_true",
        help="one decompose + solve per form and nothing else (the command ncu captures run)",
    )
    ap.add_argument("--form", choices=["both", "fp64", "mixed"], default="both", help="forms --single runs")
    ap.add_argument(
        "--shift",
        choices=["dominant", "reduced"],
        default="dominant",
        help="value set: the diagonally dominant one (shift scale 1), or the reduced shift recorded for this mesh "
        "(1-norm condition number ~1e6; the FP64 form then refines with its own factors to reach the tolerance)",
    )
    ap.add_argument("--alpha", type=float, default=None, help="shift scale of --shift reduced (default: the recorded one)")
    ap.add_argument(
        "--many",
        type=int,
        default=0,
        help="instead of the headline: this many independent systems (sides 8..64, orders 3..6, 4 RHS, seed 0), "
        "the mixed form batched on shared handles in waves against FP64 run one system at a time",
    )
    args = ap.parse_args()
    if args.shift == "reduced":
        from hybsol.b200 import meshgen

        args.alpha = args.alpha if args.alpha is not None else meshgen.reduced_shift(args.mesh, args.p)
    else:
        args.alpha = 1.0
    return args


def run_single(args):
    """One FP64 and one mixed decompose + solve of the workload, for profilers."""
    import numpy as np

    from hybsol.b200 import native

    pm, bn = build_workload(args.mesh, args.p, shift=args.alpha)
    ns = native.NativeSystem.from_matrix(pm)
    ns.set_option(native.OPTION_FP64_REFINEMENT, int(args.shift == "reduced"))
    forms = {"both": (native.FP64, native.MIXED), "fp64": (native.FP64,), "mixed": (native.MIXED,)}[args.form]
    for prec in forms:
        ns.set_values(pm.vals)
        ns.decompose(prec)
        x, info = ns.solve(bn)
        assert np.isfinite(x).all() and info["relative_residual"] < 1e-10, info
    ns.close()
    return 0


def shift_description(alpha):
    if alpha == 1.0:
        return "dominant: diagonal shift = sum of the row's off-diagonal block norms + 1"
    from hybsol.b200 import meshgen

    rec = [v for v in meshgen.REDUCED_SHIFT.values() if v[0] == alpha]
    kappa = f", kappa_1 ~ {rec[0][1]:.2g} ({rec[0][2]})" if rec else ""
    return f"reduced: diagonal shift scaled by alpha={alpha:.6g}{kappa}"


def workload_config(n, p, extra=None):
    if str(p) == "rand":
        blocks = "per-element p uniform in 2..10 (element blocks 4x4 to 100x100, edge blocks the larger neighbour's p)"
    else:
        p = int(p)
        blocks = f"p={p} (element blocks {p * p}x{p * p}, edge blocks {p}x{p})"
    nrhs = int((extra or {}).pop("nrhs", 1))
    cfg = {
        "workload": f"hybridized quad mesh {n}x{n} elements, {blocks}, {nrhs} RHS, seed 0, reference first-fit "
        "coloring order",
        "mesh": f"{n}x{n}",
        "p": p,
        "nrhs": nrhs,
        "tolerance": TOL,
        "l2": "inputs larger than L2 (factor slab >> 126 MB)",
    }
    if extra and "alpha" in extra:
        cfg["values"] = shift_description(extra.pop("alpha"))
    if extra:
        cfg.update(extra)
    return cfg


# ---------------------------------------------------------------------------------
# workload


def element_orders(n, p):
    """The mesh generator's order argument: one order for every element, or per-element
    orders uniform in 2..10 (seed 0) for p == 'rand'."""
    from hybsol.b200 import meshgen

    if str(p) == "rand":
        return meshgen.random_orders(n, 2, 10, seed=0)
    return int(p)


def build_workload(n, p, with_order=False, shift=1.0, nrhs=1):
    import numpy as np

    from hybsol.b200 import batch, meshgen, native

    mat, b = meshgen.mesh_system(n, element_orders(n, p), seed=0, shift=shift, nrhs=nrhs)
    order = native.compute_ordering(mat.row_ptr, mat.cols, "first")
    pm = mat.permuted(order)
    perm = batch.dof_permutation(mat.sizes, order)  # x_new[perm] = x_old
    bn = np.empty_like(b)
    bn[perm] = b
    if with_order:
        return pm, bn, perm
    return pm, bn


# ---------------------------------------------------------------------------------
# clocks


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while the timed region runs."""

    FIELDS = (
        "index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
            self.proc = subprocess.Popen(cmd, stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        with open(self.file.name) as f:
            rows = [r for r in csv.reader(io.StringIO(f.read())) if len(r) >= 10]
        os.unlink(self.file.name)
        mine = [r for r in rows if self.uuid and self.uuid in r[1]] or rows
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in mine:
            try:
                sm.append(float(r[2]))
                smax.append(float(r[3]))
                power.append(float(r[4]))
            except ValueError:
                continue
            for name, v in zip(names, r[6:10]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s, pw in zip(sm, power) if pw > 0.3 * max(power)] or sm
        return {
            "sm_mhz": statistics.median(loaded),
            "sm_max_mhz": max(smax),
            "reasons": sorted(reasons),
            "samples": len(sm),
            "power_w_max": max(power),
        }


# ---------------------------------------------------------------------------------
# reference CPU path


def load_meshgen():
    """The synthetic mesh generator (pure NumPy), imported from its file alone: the
    reference legs must not import the ``hybsol`` package, whose import loads this
    repository's native library."""
    import importlib.util

    path = ROOT / "hybridized-solver_b200" / "hybsol" / "b200" / "meshgen.py"
    spec = importlib.util.spec_from_file_location("_bench_meshgen", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# The reference's multi-threaded decompose can hang: its phase-2 scheduler (src/blocks.c
# of the reference, the claim loop of block_system_decompose) spins on plain, unsynchronised
# reads of the target states, the open-target count and the search start, which the
# compiler may hoist out of the loops; on small systems, where most threads spin, a run
# occasionally never returns. Each sample therefore runs in a child process with a time
# limit, and is retried once.
REF_CHILD_TIMEOUT_S = 900


def reference_sample(n, p, steps, warmup, threads):
    """reference_sample_inline in a child process (see above); raises RuntimeError when
    both tries ran out of time."""
    import numpy as np

    for attempt in range(2):
        with tempfile.TemporaryDirectory() as tmp:
            out = os.path.join(tmp, "ref.npz")
            cmd = [sys.executable, str(Path(__file__).resolve()), "--ref-child", str(n), str(p), str(steps),
                   str(warmup), str(threads), out]
            env = dict(os.environ, OMP_NUM_THREADS=str(threads))
            try:
                subprocess.run(cmd, check=True, timeout=REF_CHILD_TIMEOUT_S, env=env, stdout=subprocess.DEVNULL)
            except subprocess.TimeoutExpired:
                continue
            d = np.load(out)
            return list(d["times"]), float(d["res"]), d["x"], float(d["flops"])
    raise RuntimeError(f"the reference's decompose did not return within {REF_CHILD_TIMEOUT_S} s, twice")


def reference_child(args):
    import numpy as np

    n, p, steps, warmup, threads, out = args.ref_child
    times, res, x, flops = reference_sample_inline(int(n), p, int(steps), int(warmup), int(threads))
    np.savez(out, times=np.asarray(times), res=res, x=x, flops=flops)
    return 0


def reference_sample_inline(n, p, steps, warmup, threads):
    """Decompose + solve of the reference extension (compiled from its own sources in
    oracle/_ref) on the n x n mesh, through its public BlockSystem API: assembly, the
    reference's coloring, reorder_blocks, decompose(n_threads) and solve. Returns the
    per-step times (s), the relative residual, the solution in the mesh's numbering and
    the algorithmic flops counted from the reference's own factored pattern."""
    import numpy as np

    from oracle import oracle as O

    mg = load_meshgen()
    ref = O.load_reference()
    orders = mg.random_orders(n, 2, 10, seed=0) if str(p) == "rand" else int(p)
    mat, b = mg.mesh_system(n, orders, seed=0)
    times = []
    for it in range(warmup + steps):
        s = ref.BlockSystem(*[int(x) for x in mat.sizes])
        for r, c, v in mat.iter_blocks():
            s.add_block(r, c, v)
        order = s.compute_reordering("first")
        s.reorder_blocks(order)
        bn = s.unorder_vector(order, b)
        t0 = time.perf_counter()
        s.decompose(threads)
        x = s.solve(bn)
        dt = time.perf_counter() - t0
        if it >= warmup:
            times.append(dt)
    xo = s.reorder_vector(order, x)
    res = float(np.linalg.norm(mat.matvec(xo) - b) / np.linalg.norm(b))
    flops = O.factor_flops(np.asarray(s.block_sizes), [s.get_row_block_indices(i) for i in range(mat.n_blocks)])
    return times, res, xo, flops


def sample_workload_name(n, p):
    return workload_config(n, p)["workload"]


def cpu_baseline(full_flops, p, sample_mesh, threads=0):
    """The reference on the box's host cores, on the sample mesh; `value` extrapolates
    the measured time to the benchmarked workload by algorithmic GFLOP (marked as such)."""
    from oracle import oracle as O

    cores = threads or O.cpu_count()
    times, res, x, sample_flops = reference_sample(sample_mesh, p, 1, 0, cores)
    best = min(times)
    scale = full_flops / sample_flops
    return {
        "value": best * 1e3 * scale,
        "unit": "ms",
        "cores": cores,
        "kind": "reference",
        "extrapolated": True,
        "sample": (
            f"reference extension (oracle/_ref, built from the reference's src/*.c) decompose(n_threads={cores}) + "
            f"solve on the {sample_mesh}x{sample_mesh} p={p} mesh ({sample_flops / 1e9:.1f} GFLOP): measured "
            f"{best * 1e3:.1f} ms ({sample_flops / best / 1e9:.1f} GFLOP/s, residual {res:.1e}); `value` is that "
            f"time EXTRAPOLATED by GFLOP to the {full_flops / 1e9:.0f}-GFLOP workload, not measured"
        ),
        "sample_ms": best * 1e3,
        "sample_gflops": sample_flops / best / 1e9,
        "sample_workload": sample_workload_name(sample_mesh, p),
    }, x


def run_reference(args):
    """The reference's own CPU path, measured on the sample mesh it can finish within the
    run (default 20x20 at the benchmark's p): `value` is the measured time per step of that
    mesh, and `config` names it. The same mesh is timed on the GPU by our arm
    (`same_mesh_pair` in its line), which is the like-for-like comparison."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O

    if not O.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference extension not built (oracle/_ref missing)"}))
        return 0
    cores = args.ref_threads or O.cpu_count()
    n = args.cpu_sample_mesh
    try:
        times, res, _, flops = reference_sample(n, args.p, args.steps, args.warmup, cores)
    except RuntimeError as e:
        print(json.dumps({"impl": "reference", "unavailable": f"{e} (a data race in its OpenMP scheduler)"}))
        return 0
    ms = statistics.mean(times) * 1e3
    cpu = {
        "value": ms,
        "unit": "ms",
        "cores": cores,
        "kind": "reference",
        "sample": f"the whole {n}x{n} p={args.p} mesh per step ({flops / 1e9:.1f} GFLOP, "
        f"{flops / (ms * 1e-3) / 1e9:.1f} GFLOP/s, residual {res:.1e}); measured, not extrapolated",
    }
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": ms,
        "unit": "ms",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(
            n,
            args.p,
            {
                "factor_gflop": flops / 1e9,
                "sample_of": workload_config(args.mesh, args.p)["workload"],
                "note": f"the reference's CPU path cannot finish the {args.mesh}x{args.mesh} mesh within a run; "
                "this line measures the largest mesh it finishes per step, and our arm times the same mesh on the GPU",
            },
        ),
        "cpu_baseline": cpu,
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------------
# our arm


def load_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return json.loads(path.read_text()), "measured"
    return dict(FALLBACK_PEAKS), "fallback"


def gemm_peak(dtype):
    """cuBLAS GEMM throughput (TFLOP/s) measured here, the denominator for FP64/FP32 kernels."""
    import torch

    n = 8192
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(5):
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2 * n**3 / (best * 1e-3) / 1e12


def same_mesh_pair(args, x_ref, ref_ms):
    """Our FP64 and mixed forms on the mesh the reference's CPU path was measured on (the
    cpu_baseline sample), with the same step protocol as the headline (device-resident
    inputs, CUDA events, warm-up) and end to end through the C ABI from pinned host
    buffers; the FP64 solution is compared element-wise with the reference's."""
    import ctypes

    import numpy as np
    import torch

    from hybsol.b200 import native

    lib = native.lib()
    n = args.cpu_sample_mesh
    pm, bn, perm = build_workload(n, args.p, with_order=True)
    ns = native.NativeSystem(pm.sizes, pm.row_ptr, pm.cols)
    stream = torch.cuda.ExternalStream(ns.stream)
    d_vals = torch.from_numpy(pm.vals).to("cuda")
    d_b = torch.from_numpy(bn).to("cuda")
    d_x = torch.empty_like(d_b)
    out = {"workload": sample_workload_name(n, args.p), "reference_ms": ref_ms, "reference_kind": "oracle/_ref"}
    steps, warmup = max(3, args.steps), max(3, args.warmup)
    for name, prec in (("fp64", native.FP64), ("mixed", native.MIXED)):

        def step():
            native._check(lib.hyb_system_set_values(ns._h, native._ptr(d_vals), native.MEMORY_DEVICE), "set_values")
            ns.decompose(prec)
            return ns.solve_device(d_b, d_x, 1, tol=TOL, max_iter=30, residual=(prec == native.MIXED))

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for e0, e1 in ev:
            e0.record(stream)
            info = step()
            e1.record(stream)
        torch.cuda.synchronize()
        out[f"{name}_ms"] = statistics.mean(a.elapsed_time(b) for a, b in ev)
        if prec == native.FP64:
            x = d_x.cpu().numpy()[perm]  # back to the mesh's numbering
            out["fp64_rel_err_vs_reference"] = float(np.abs(x - x_ref).max() / np.abs(x_ref).max())
        else:
            out["mixed_iterations"] = info["iterations"]
            out["mixed_relative_residual"] = info["relative_residual"]
    h_vals = torch.from_numpy(pm.vals).pin_memory()
    h_b = torch.from_numpy(bn).pin_memory()
    h_x = torch.empty_like(h_b).pin_memory()
    sinfo = native.SolveInfo()
    for name, prec in (("fp64", native.FP64), ("mixed", native.MIXED)):

        def e2e():
            native._check(lib.hyb_system_set_values(ns._h, native._ptr(h_vals), native.MEMORY_HOST), "set_values")
            ns.decompose(prec)
            native._check(
                lib.hyb_solve(ns._h, native._ptr(h_b), native._ptr(h_x), 1, native.MEMORY_HOST, TOL, 30,
                              ctypes.byref(sinfo)),
                "hyb_solve",
            )

        e2e()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            e2e()
        out[f"e2e_{name}_ms"] = (time.perf_counter() - t0) * 1e3 / steps
    out["e2e_speedup_mixed_vs_reference"] = ref_ms / out["e2e_mixed_ms"]
    out["e2e_speedup_fp64_vs_reference"] = ref_ms / out["e2e_fp64_ms"]
    out["steps"], out["warmup"] = steps, warmup
    ns.close()
    return out


def run_many(args):
    """Many independent systems: the mixed form on batched handles (each system ordered
    alone, stacked, its pivots sharing stages with the others', refined until every system
    meets 1e-12 against its own right-hand sides), in waves that fit the device, against the
    plain FP64 form run on the same systems one at a time. Each handle is factored once
    untimed (symbolic phase, graph capture) before its timed decompose + solve; times are
    CUDA events on the handle's stream."""
    import numpy as np
    import torch

    from hybsol.b200 import batch, meshgen, native

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    specs = meshgen.many_mesh_specs(args.many, (8, 64), (3, 6), seed=0)

    def system(k):  # regenerated on demand: only one wave's systems are held at a time
        side, p = specs[k]
        return meshgen.mesh_system(side, p, seed=1000 + k, nrhs=4)

    def timed(ns, fn):
        st = torch.cuda.ExternalStream(ns.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        out = fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    # mixed: batched handles in waves planned from the patterns
    t0 = time.perf_counter()
    free, _ = torch.cuda.mem_get_info()
    budget = int(0.45 * free)
    weights = [batch.pattern_bytes(*meshgen.mesh_pattern(side, p), native.MIXED) for side, p in specs]
    waves = batch.plan_waves(weights, budget)
    plan_s = time.perf_counter() - t0
    mixed_ms, worst_mixed, iters, flops, dof_total = 0.0, 0.0, [], 0.0, 0
    x_mixed = [None] * len(specs)
    for wave in waves:
        pairs = [system(k) for k in wave]
        mats, rhs = [m for m, _ in pairs], [b for _, b in pairs]
        del pairs
        dof_total += sum(m.dof for m in mats)
        bs = batch.BatchedSystem(mats)
        flops += native.analyze(bs.layout.matrix.sizes, bs.layout.matrix.row_ptr, bs.layout.matrix.cols)["factor_flops"]
        bs.decompose(native.MIXED)
        bs.solve(rhs)  # warm-up: graphs captured, buffers sized
        bs.set_values(mats)

        def step():
            bs.decompose(native.MIXED)
            return bs.solve(rhs, max_iter=60)

        ms, (xs, info) = timed(bs.native, step)
        mixed_ms += ms
        for k, x, si in zip(wave, xs, info["systems"]):
            x_mixed[k] = x
            worst_mixed = max(worst_mixed, si["relative_residual"])
            iters.append(si["iterations"] if si["iterations"] is not None else -1)
        bs.close()
        del bs, mats, rhs
        torch.cuda.empty_cache()
    gen_s = time.perf_counter() - t0
    # FP64, one system at a time
    fp64_ms, worst_fp64, err = 0.0, 0.0, 0.0
    for i in range(len(specs)):
        m, b = system(i)
        order = native.compute_ordering(m.row_ptr, m.cols, "first").astype(np.int64)
        pm = m.permuted(order)
        perm = batch.dof_permutation(m.sizes, order)
        bn = np.empty_like(b)
        bn[perm] = b
        ns = native.NativeSystem.from_matrix(pm)
        ns.decompose(native.FP64)
        ns.solve(bn)
        ns.set_values(pm.vals)

        def step64():
            ns.decompose(native.FP64)
            return ns.solve(bn)

        ms, (x, info) = timed(ns, step64)
        fp64_ms += ms
        worst_fp64 = max(worst_fp64, info["relative_residual"])
        x = x[perm]
        err = max(err, float(np.abs(x_mixed[i] - x).max() / np.abs(x).max()))
        ns.close()
    line = {
        "metric": "decompose+solve ms of many independent systems: FP32+refine batched vs plain FP64 one at a time",
        "value": mixed_ms,
        "unit": "ms",
        "n_gpus": 1,
        "higher_is_better": False,
        "dtype": "f32 factors + f64 refinement",
        "data": "synthetic",
        "config": {
            "workload": f"{args.many} independent quad-mesh systems, side uniform in 8..64, order uniform in 3..6 "
            "(seed 0), 4 RHS each, reference first-fit coloring order per system",
            "systems": args.many,
            "dof_total": int(dof_total),
            "factor_gflop": flops / 1e9,
            "waves": len(waves),
            "wave_budget_bytes": budget,
        },
        "fp64_one_at_a_time_ms": fp64_ms,
        "speedup_vs_fp64_one_at_a_time": fp64_ms / mixed_ms,
        "accuracy": {
            "worst_system_relative_residual_mixed": worst_mixed,
            "worst_system_relative_residual_fp64": worst_fp64,
            "worst_system_rel_err_mixed_vs_fp64": err,
            "refinement_steps_per_system": {"min": int(min(iters)), "max": int(max(iters))},
        },
        "wave_plan_s": plan_s,
        "mixed_leg_wall_s": gen_s,
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    import ctypes

    import numpy as np
    import torch
    import torch.distributed as dist

    from hybsol.b200 import native

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if not native.device_available():
        raise RuntimeError("bench.py needs an sm_100 GPU")
    lib = native.lib()
    peaks, peak_src = load_peaks()
    fp64_peak = gemm_peak(torch.float64)
    fp32_peak = gemm_peak(torch.float32)

    t0 = time.perf_counter()
    pm, bn = build_workload(args.mesh, args.p, shift=args.alpha, nrhs=args.nrhs)
    nr = args.nrhs
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    ns = native.NativeSystem(pm.sizes, pm.row_ptr, pm.cols)
    analysis_ms = (time.perf_counter() - t0) * 1e3
    reduced = args.shift == "reduced"
    # the reduced set needs refinement in the FP64 form too (its plain solve misses 1e-12)
    ns.set_option(native.OPTION_FP64_REFINEMENT, int(reduced))
    ana = native.analyze(pm.sizes, pm.row_ptr, pm.cols)
    flops = ana["factor_flops"]
    stream = torch.cuda.ExternalStream(ns.stream)

    d_vals = torch.from_numpy(pm.vals).to("cuda")
    d_b = torch.from_numpy(bn).to("cuda")
    d_x = torch.empty_like(d_b)
    if not args.no_profile:
        lib.hyb_profile_enable(ns._h, max(1, args.profile_stride))

    def device_step(prec):
        """One step with inputs resident in HBM; returns (launches, solve info)."""
        launches = 0
        native._check(lib.hyb_system_set_values(ns._h, native._ptr(d_vals), native.MEMORY_DEVICE), "set_values")
        ns.decompose(prec)
        launches += ns.last_launch_count()
        info = ns.solve_device(d_b, d_x, nr, tol=TOL, max_iter=60, residual=(prec == native.MIXED or reduced))
        launches += ns.last_launch_count()
        return launches, info

    def timed_form(prec):
        for _ in range(args.warmup):
            device_step(prec)
        barrier()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        launches, info = 0, None
        for k in range(args.steps):
            starts[k].record(stream)
            lk, info = device_step(prec)
            ends[k].record(stream)
            launches += lk
        barrier()
        ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
        prof = native.KernelProfile()
        have_prof = lib.hyb_profile_read(ns._h, ctypes.byref(prof)) == 0 and prof.launches > 0
        return statistics.mean(ms), launches, info, (prof if have_prof else None)

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    with ClockSampler(uuid) as clocks:
        fp64_ms, fp64_launches, fp64_info, fp64_prof = timed_form(native.FP64)
        x64 = d_x.cpu().numpy()
        r64 = ns.residual(bn, x64)
        fp64_relres = float(np.linalg.norm(r64) / np.linalg.norm(bn))
        mixed_ms, mixed_launches, mixed_info, mixed_prof = timed_form(native.MIXED)
        xm = d_x.cpu().numpy()
    clk = clocks.summary()
    fp64_ms = max_over_ranks(fp64_ms)
    mixed_ms = max_over_ranks(mixed_ms)
    err_vs_fp64 = float(np.abs(xm - x64).max() / np.abs(x64).max())

    # end to end through the C ABI: pinned host values and RHS in, solution out
    h_vals = torch.from_numpy(pm.vals).pin_memory()
    h_b = torch.from_numpy(bn).pin_memory()
    h_x = torch.empty_like(h_b).pin_memory()
    sinfo = native.SolveInfo()

    def e2e_step():
        native._check(lib.hyb_system_set_values(ns._h, native._ptr(h_vals), native.MEMORY_HOST), "set_values")
        ns.decompose(native.MIXED)
        st = lib.hyb_solve(
            ns._h, native._ptr(h_b), native._ptr(h_x), nr, native.MEMORY_HOST, TOL, 60, ctypes.byref(sinfo)
        )
        native._check(st, "hyb_solve")

    e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    barrier()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps)

    def roofline(prof, bound, peak, unit, elem_bytes, peak_note, step_ms, kernel, traffic_per_block=None):
        """One update pass -- one level, or in the mixed form a pair of levels applied in one
        two-pivot pass -- (both lookahead launches, timed with events on the handle's stream,
        every profile-stride-th pass of the timed steps) against its bound; algorithmic work
        per pass from the pattern: 2 m k n flops per target block and source pivot, and the
        FP32/FP64 bytes of reading and writing every target once plus reading the
        lower-column and upper-row operands once. The share of the step scales the sampled
        mean to every pass with an update."""
        if prof is None:
            return None
        avg_ms = prof.total_ms / prof.launches
        flops_per = prof.flops / prof.launches
        bytes_per = elem_bytes * (2 * prof.c_elems + prof.ab_elems) / prof.launches
        tflops = flops_per / (avg_ms * 1e-3) / 1e12
        gbs = bytes_per / (avg_ms * 1e-3) / 1e9
        achieved, per_launch = (tflops, flops_per) if bound == "tensor" else (gbs, bytes_per)
        traffic = None
        if traffic_per_block is not None:
            traffic = traffic_per_block * prof.c_elems / prof.launches / 4096.0
        return {
            "bound": bound,
            "achieved": achieved,
            "peak": peak,
            "unit": unit,
            "frac": achieved / peak,
            "traffic": traffic,
            "kernel": kernel,
            "avg_launch_ms": avg_ms,
            "share_of_step": avg_ms * prof.passes / step_ms,
            "passes_timed": prof.launches,
            "passes_with_update": prof.passes,
            "levels_with_update": prof.levels,
            "pivots_per_pass": prof.pivots_timed / prof.launches,
            "ms_per_pivot": avg_ms * prof.launches / prof.pivots_timed,
            "pivot_work_ms_per_pivot": (prof.pivot_ms / prof.pivot_levels) if prof.pivot_levels else None,
            "peak_source": peak_note,
            "algorithmic_per_launch": per_launch,
            "algorithmic_unit": "flop" if bound == "tensor" else "byte",
            "tflops_fp_equivalent": tflops,
            "gbs_algorithmic": gbs,
        }

    rf64 = roofline(
        fp64_prof, "tensor", fp64_peak, "TFLOP/s", 8, "cuBLAS DGEMM 8192^3 measured in this run (FP64 DMMA)",
        fp64_ms, "k_update64_f64 (FP64 DMMA m8n8k4, bulk-copy staged operands)",
    )
    hbm = float(peaks.get("hbm_gbs") or 6650.0)
    rmix = roofline(
        mixed_prof, "hbm", hbm, "GB/s", 4,
        f"MEASURED_PEAKS.json hbm_gbs ({peak_src})", mixed_ms,
        "k_update64_tc (tcgen05 split-BF16, persistent, bulk-copy C ring)",
        traffic_per_block=TC_DRAM_BYTES_PER_TARGET_BLOCK,
    )
    if rmix is not None and rmix["pivots_per_pass"] > 1.5:
        rmix["kernel"] = (
            "k_update64_tc2 (tcgen05 split-BF16, two pivots per pass: K = 128, targets staged in registers, "
            "persistent)"
        )
        rmix["traffic"] = TC2_DRAM_BYTES_PER_TARGET_BLOCK * mixed_prof.c_elems / mixed_prof.launches / 4096.0
    if rf64 is not None:
        rf64["traffic_note"] = (
            "null: the FP64 update's DRAM bytes were captured only at 32x32 (profiles/k_update64_f64_mesh32_p8.md), "
            "where a stage's targets stay in L2; the bound here is the FP64 tensor pipe, not DRAM"
        )
    if rmix is not None:
        rmix["traffic_note"] = (
            "dram__bytes_read.sum + dram__bytes_write.sum of one pass (both launches) from a 1-pass ncu capture "
            "at 96x96 p=8 (profiles/k_update64_tc2_mesh48_p8.md for the two-pivot pass: 26.4 KB per 64x64 target "
            "block per pair; profiles/k_update64_tc_dram_mesh96_p8.md for one pivot per pass: 27.2 KB per target "
            "block per stage), scaled to this pass's target blocks"
        )
    if rmix is not None:
        # three BF16 MMAs per FP32 product on the tensor cores, against the sustained peak
        bf16 = float(peaks.get("bf16_tflops_sustained") or 1390.5)
        rmix["tensor_bf16_tflops"] = 3 * rmix["tflops_fp_equivalent"]
        rmix["tensor_bf16_frac_of_sustained"] = 3 * rmix["tflops_fp_equivalent"] / bf16
    cpu, pair = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not reduced:
        from oracle import oracle as O

        if O.reference_available():
            try:
                cpu, x_ref = cpu_baseline(flops, args.p, args.cpu_sample_mesh, args.ref_threads)
                pair = same_mesh_pair(args, x_ref, cpu["sample_ms"])
            except RuntimeError as e:
                cpu = {"unavailable": str(e)}
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": mixed_ms,
            "unit": "ms",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": mixed_ms,
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 factors + f64 refinement",
            "data": "synthetic",
            "config": workload_config(
                args.mesh,
                args.p,
                {
                    "dof": int(pm.dof),
                    "blocks": int(pm.n_blocks),
                    "blocks_after_fill": int(ana["filled_blocks"]),
                    "levels": int(ana["n_levels"]),
                    "factor_gflop": flops / 1e9,
                    "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                    "alpha": args.alpha,
                    "nrhs": args.nrhs,
                },
            ),
            "fp64_ms": fp64_ms,
            "mixed_speedup_vs_fp64": fp64_ms / mixed_ms,
            "fp64_tflops": flops / (fp64_ms * 1e-3) / 1e12,
            "mixed_tflops": flops / (mixed_ms * 1e-3) / 1e12,
            "accuracy": {
                "fp64_relative_residual": fp64_relres,
                "fp64_refinement_iterations": fp64_info["iterations"],
                "mixed_relative_residual": mixed_info["relative_residual"],
                "mixed_refinement_iterations": mixed_info["iterations"],
                "mixed_krylov_iterations": mixed_info["krylov_iterations"],
                "mixed_converged": mixed_info["converged"],
                "mixed_rel_err_vs_fp64_solution": err_vs_fp64,
            },
            "analysis_ms": analysis_ms,
            "workload_build_s": gen_s,
            "e2e": {
                "value": e2e_ms,
                "unit": "ms",
                "h2d_bytes_per_step": int(h_vals.numel() * 8 + h_b.numel() * 8),
                "d2h_bytes_per_step": int(h_x.numel() * 8),
                "path": "C ABI with pinned host buffers: hyb_system_set_values + hyb_decompose(mixed) + hyb_solve",
            },
            "gpu_launches": int(mixed_launches),
            "gpu_launches_fp64": int(fp64_launches),
            "roofline": rmix,
            "roofline_fp64": rf64,
            "peaks": {"fp64_tflops_cublas": fp64_peak, "fp32_tflops_cublas": fp32_peak, "source": peak_src, **peaks},
            "clocks": clk,
            "cpu_baseline": cpu,
            "same_mesh_pair": pair,
        }
        print(json.dumps(line))
    ns.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse_args()
    if args.ref_child:
        return reference_child(args)
    if args.many:
        return run_many(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.single:
        return run_single(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
