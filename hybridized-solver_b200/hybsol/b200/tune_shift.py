"""Reduced-shift value sets on the GPU: the diagonal-shift scale of a mesh system at which
its 1-norm condition number is about a target (1e6 for the ill-conditioned set).

For each trial scale the values are re-shifted in place (``meshgen.shifted_values``),
factored in FP64 on the device and the condition number is estimated from the factors
(``hyb_condition_estimate``: Hager's method with Higham's refinements, solves with A and
A^T). ``meshgen.tune_shift`` bisects the scale. The results for the large meshes are
recorded in ``meshgen.REDUCED_SHIFT``.

    python -m hybsol.b200.tune_shift N P [--target 1e6] [--seed 0]
"""

from __future__ import annotations

import argparse
import json
import time

from . import meshgen, native


def tune(n: int, p, seed: int = 0, target: float = 1e6, tol_decades: float = 0.1):
    """(alpha, kappa_1 estimate, history) for the n x n mesh of order p (seed `seed`)."""
    mat, _ = meshgen.mesh_system(n, p, seed=seed, shift=1.0)
    order = native.compute_ordering(mat.row_ptr, mat.cols, "first")
    pm = mat.permuted(order)
    weights = meshgen.diagonal_weights(pm, meshgen.row_shift_amounts(pm, n))
    ns = native.NativeSystem(pm.sizes, pm.row_ptr, pm.cols)
    try:

        def kappa(alpha):
            ns.set_values(meshgen.shifted_values(pm, 1.0, alpha, weights))
            ns.decompose(native.FP64)
            return ns.condition_estimate()["kappa1"]

        return meshgen.tune_shift(kappa, target=target, tol_decades=tol_decades)
    finally:
        ns.close()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("n", type=int)
    ap.add_argument("p", type=int)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--target", type=float, default=1e6)
    args = ap.parse_args()
    t0 = time.perf_counter()
    alpha, kappa, history = tune(args.n, args.p, args.seed, args.target)
    print(
        json.dumps(
            {
                "n": args.n,
                "p": args.p,
                "seed": args.seed,
                "alpha": alpha,
                "kappa1_estimate": kappa,
                "history": history,
                "seconds": time.perf_counter() - t0,
            }
        )
    )


if __name__ == "__main__":
    main()
