"""The screened kernels' modified Bessel functions on the device
(wos_special_functions) against scipy.special.

* FP64 (PLAIN_FP64, FAST_FP64): the series / quadrature / Hankel sums agree
  with scipy's Cephes-based i0e / k0e to 1e-14 relative in ln I0 and ln K0
  (the C oracle's identical code matches libstdc++, the reference's
  std::cyl_bessel_i/k, to 5e-15: tests/test_oracle_golden.py).
* FP32 (FAST_FP32): Abramowitz & Stegun 9.8.1-9.8.6, absolute error < 1.9e-7
  on the scaled forms, i.e. < 1e-6 relative in I0 and K0, plus the FP32
  rounding of x and of the logarithm (|ln| up to ~50 here).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

scipy_special = pytest.importorskip("scipy.special")

X = np.concatenate([np.geomspace(1e-4, 60.0, 700), [0.5, 1.0, 2.0, 3.75, 10.0, 49.9, 50.0]])


def reference(x):
    # ln I0 = x + ln(i0e), ln K0 = ln(k0e) - x
    return x + np.log(scipy_special.i0e(x)), np.log(scipy_special.k0e(x)) - x


def test_fp64_matches_scipy(solver):
    li, lk = solver.special_functions(X, precision=64)
    ri, rk = reference(X)
    assert np.allclose(li, ri, rtol=1e-14, atol=1e-15)
    assert np.allclose(lk, rk, rtol=1e-14, atol=1e-14)


def test_fp32_within_the_published_bounds(solver):
    li, lk = solver.special_functions(X, precision=32)
    xf = X.astype(np.float32).astype(np.float64)   # the kernels see x in float
    ri, rk = reference(xf)
    # 1e-6 relative in the function -> 1e-6 absolute in its log, plus FP32
    # rounding of the log itself (ulp of |ln| <= 60 is 3.8e-6)
    tol_i = 1.2e-6 + 2.4e-7 * np.abs(ri)
    tol_k = 1.2e-6 + 2.4e-7 * np.abs(rk)
    assert np.all(np.abs(li - ri) <= tol_i), np.max(np.abs(li - ri) / tol_i)
    assert np.all(np.abs(lk - rk) <= tol_k), np.max(np.abs(lk - rk) / tol_k)
    # the screened walk's weight 1/I0(alpha R) and acceptance ratios
    w32, w64 = np.exp(-li), np.exp(-reference(xf)[0])
    assert np.allclose(w32, w64, rtol=5e-5)
