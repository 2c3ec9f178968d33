"""The device Boys function (sqb::boys<M>, the routine every class kernel calls) on a grid of
T in [0, 60] that crosses the switches of both implementations -- T = 0.0005 (the reference's
three-term series below it), T = 36 (the device's Taylor grid below, asymptote with upward
recursion above) -- for every order m <= 8:

  * against the exact function (its series summed in 60-digit decimal arithmetic):
    relative 1e-14;
  * against the reference's own fgamma_set (src/fgamma.c:172-206, from
    oracle/_ref/libsqref.so): relative 1e-12 for T >= 0.0005, where the reference itself
    departs from the exact values by up to about 2e-13 (forward recursion near T = 0.5, for
    instance); below T = 0.0005 within the truncation error of its series,
    x^3 / (6 (2m + 7)) (about 3e-12 at the switch)."""
import ctypes
import json
import os
from decimal import Decimal, getcontext

import numpy as np
import pytest

from conftest import ROOT, load_sqb200, results_path

LIBREF = os.path.join(ROOT, "oracle", "_ref", "libsqref.so")


def _grid():
    T = np.concatenate([[0.0, 1e-12, 1e-8, 1e-6, 1e-5, 1e-4, 2.5e-4, 4.99e-4, 5.0e-4, 5.01e-4, 1e-3],
                        np.linspace(0.001, 1.0, 97), np.linspace(1.0, 35.95, 300),
                        [35.999, 36.0, 36.001], np.linspace(36.05, 60.0, 120)])
    rng = np.random.default_rng(5)
    return np.concatenate([T, rng.uniform(0.0, 60.0, 150)])


def _exact(mmax, t):
    """F_0..F_mmax(t): F_mmax = e^-t sum_i (2t)^i / ((2m+1)(2m+3)...(2m+2i+1)) (all terms
    positive), then the stable downward recursion, in 60-digit decimal arithmetic."""
    getcontext().prec = 60
    x = Decimal(float(t))
    term = Decimal(1) / (2 * mmax + 1)
    acc = Decimal(0)
    i = 0
    while True:
        acc += term
        i += 1
        term = term * 2 * x / (2 * mmax + 2 * i + 1)
        if term < acc * Decimal(10) ** -50:
            break
    e = (-x).exp()
    F = [Decimal(0)] * (mmax + 1)
    F[mmax] = e * acc
    for m in range(mmax - 1, -1, -1):
        F[m] = (2 * x * F[m + 1] + e) / (2 * m + 1)
    return [float(v) for v in F]


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(LIBREF), reason="oracle/_ref not built")
def test_boys_matches_exact_and_reference():
    sqb = load_sqb200()
    ref = ctypes.CDLL(LIBREF)
    ref.fgamma_set.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    T = _grid()
    exact = [_exact(8, t) for t in T]
    worst_exact, worst_ref = {}, {}
    for M in range(9):
        F = sqb.engine.boys_eval(M, T)
        buf = (ctypes.c_double * (M + 1))()
        for i, t in enumerate(T):
            ref.fgamma_set(M, float(t), buf)
            for m in range(M + 1):
                d, x, r = F[i, m], exact[i][m], buf[m]
                e1 = abs(d - x) / abs(x)
                worst_exact[m] = max(worst_exact.get(m, 0.0), e1)
                assert e1 <= 1e-14, ("exact", M, m, t, d, x)
                if t < 0.0005:
                    assert abs(d - r) <= t ** 3 / (6 * (2 * m + 7)) + 1e-15 * abs(r), ("reference", M, m, t, d, r)
                else:
                    e2 = abs(d - r) / abs(r)
                    worst_ref[m] = max(worst_ref.get(m, 0.0), e2)
                    assert e2 <= 1e-12, ("reference", M, m, t, d, r)
    with open(results_path("boys_vs_exact_and_fgamma_set.json"), "w") as f:
        json.dump({"max_rel_err_vs_exact": worst_exact, "max_rel_err_vs_reference_T_ge_5e-4": worst_ref,
                   "points": len(T)}, f)
