"""The ill-conditioned value sets (reduced diagonal shift) on the host.

The generator scales the diagonal shift by alpha and ``tune_shift`` bisects alpha to a
target 1-norm condition number. These tests re-check the recorded small-mesh values with
the exact kappa_1 (dense inverse) and the bisection itself on a known curve.
"""

from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize(("n", "p"), [(8, 8), (16, 4)])
def test_recorded_reduced_shift_gives_kappa_1e6(n, p):
    from hybsol.b200 import meshgen

    alpha = meshgen.reduced_shift(n, p)
    mat, _ = meshgen.mesh_system(n, p, seed=0, shift=alpha)
    kappa = meshgen.exact_kappa1(mat)
    assert abs(np.log10(kappa) - 6.0) <= 0.1, kappa
    # the dominant set of the same draws is far better conditioned
    mat1, _ = meshgen.mesh_system(n, p, seed=0, shift=1.0)
    assert meshgen.exact_kappa1(mat1) < 1e3


def test_shifted_values_match_regeneration():
    from hybsol.b200 import meshgen

    mat, _ = meshgen.mesh_system(6, 4, seed=2, shift=1.0)
    m2, _ = meshgen.mesh_system(6, 4, seed=2, shift=0.37)
    w = meshgen.diagonal_weights(mat, meshgen.row_shift_amounts(mat, 6))
    v = meshgen.shifted_values(mat, 1.0, 0.37, w)
    assert np.allclose(v, m2.vals, rtol=0, atol=1e-13)
    off_diag = np.ones(len(v), dtype=bool)
    off_diag[w[0]] = False
    assert np.array_equal(v[off_diag], m2.vals[off_diag])


def test_tune_shift_bisects_to_the_target():
    from hybsol.b200 import meshgen

    # kappa(alpha) = 10 / alpha^4: 1e6 at alpha = 0.01778
    alpha, kappa, hist = meshgen.tune_shift(lambda a: 10.0 / a**4, target=1e6, tol_decades=0.02)
    assert abs(np.log10(kappa) - 6) <= 0.02 and abs(alpha - 10 ** (-1.25)) / 10 ** (-1.25) < 0.02
    assert hist[0] == (1.0, 10.0)
    with pytest.raises(ValueError):
        meshgen.tune_shift(lambda a: 1e9, target=1e6)
    with pytest.raises(KeyError, match="tune_shift"):
        meshgen.reduced_shift(1000, 8)
