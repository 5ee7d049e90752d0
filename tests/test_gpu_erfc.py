"""The FP64 erfc of the real-space Ewald kernels (erfc_ex2 in common.cuh:
e^{-x^2} times degree-13 Chebyshev interpolants of erfc(x) e^{x^2} on
[j/2, j/2 + 1/2), j = 0..8; coefficients from mdff_b200/csrc/fit_erfcx.py)
against CUDA's erfc and against 30-digit mpmath on [0, 4.5) and beyond.

Bound, pointwise: the fit's own error is 2.1e-16 relative in FP64 Horner, and
e^{-x^2} computed from the rounded x^2 carries x^2 u relative (u = 2^-53: the
argument's rounding, 2.2e-15 at x = 4.5; the real-space kernels reach
x = alpha rc = 3), plus a few ulp for exp and the product.  So erfc_ex2 is held
to (x^2 + 6) u relative of the 30-digit value and to (x^2 + 12) u of CUDA's
erfc (whose documented error is a few ulp)."""
import mpmath as mp
import numpy as np
import pytest

import mdff_b200

pytestmark = pytest.mark.gpu


def test_erfc_ex2_against_cuda_and_mpmath():
    rng = np.random.default_rng(5)
    x = np.concatenate([np.linspace(0.0, 4.5, 9001, endpoint=False), rng.uniform(0.0, 4.5, 4000),
                        np.arange(1, 9) * 0.5, np.arange(1, 9) * 0.5 - 1e-15, [4.5, 5.0, 6.0]])
    ex2, ref = mdff_b200.erfc_check(x)
    mp.mp.dps = 30
    exact = np.array([float(mp.erfc(mp.mpf(float(v)))) for v in x])
    inside = x < 4.5
    rel_exact = np.abs(ex2 - exact) / exact
    rel_cuda = np.abs(ex2 - ref) / ref
    u = 2.0 ** -53
    xi = x[inside]
    assert np.all(rel_exact[inside] <= (xi * xi + 6.0) * u), (rel_exact[inside] / ((xi * xi + 6.0) * u)).max()
    assert np.all(rel_cuda[inside] <= (xi * xi + 12.0) * u), (rel_cuda[inside] / ((xi * xi + 12.0) * u)).max()
    assert np.array_equal(ex2[~inside], ref[~inside])   # CUDA's erfc outside the fitted range
