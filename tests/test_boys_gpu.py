"""The device Boys function (sqb::boys<M>, the routine every class kernel calls) against the
reference's own fgamma_set (src/fgamma.c:172-206, from oracle/_ref/libsqref.so) on a grid of T
in [0, 60] that crosses both of its switches: T = 0.0005 (the reference's three-term series
below) and T = 36 (the device's Taylor grid below, asymptote with upward recursion above), for
every order m <= 8.

Tolerance: relative 1e-13 where the reference is exact to rounding.  Below T = 0.0005 the
reference truncates its series after x^2, an error up to x^3 / (6 (2m + 7)) (about 3e-12 at
the switch); there the device values are checked against the exact series at 1e-15 and against
the reference within its truncation bound."""
import ctypes
import json
import os
from math import factorial

import numpy as np
import pytest

from conftest import ROOT, load_sqb200, results_path

LIBREF = os.path.join(ROOT, "oracle", "_ref", "libsqref.so")


def _grid():
    T = np.concatenate([[0.0, 1e-12, 1e-8, 1e-6, 1e-5, 1e-4, 2.5e-4, 4.99e-4, 5.0e-4, 5.01e-4, 1e-3],
                        np.linspace(0.001, 1.0, 97), np.linspace(1.0, 35.95, 700),
                        [35.999, 36.0, 36.001], np.linspace(36.05, 60.0, 240)])
    rng = np.random.default_rng(5)
    return np.concatenate([T, rng.uniform(0.0, 60.0, 400)])


def _series(m, x, terms=12):
    return sum((-x) ** k / (factorial(k) * (2 * m + 2 * k + 1)) for k in range(terms))


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(LIBREF), reason="oracle/_ref not built")
def test_boys_matches_reference_fgamma_set():
    sqb = load_sqb200()
    ref = ctypes.CDLL(LIBREF)
    ref.fgamma_set.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    T = _grid()
    worst = {}
    for M in range(9):
        F = sqb.engine.boys_eval(M, T)
        buf = (ctypes.c_double * (M + 1))()
        for i, t in enumerate(T):
            ref.fgamma_set(M, float(t), buf)
            for m in range(M + 1):
                r, d = buf[m], F[i, m]
                if t < 0.0005:
                    exact = _series(m, t)
                    assert abs(d - exact) <= 1e-15 * abs(exact), (M, m, t, d, exact)
                    assert abs(d - r) <= t ** 3 / (6 * (2 * m + 7)) + 1e-15 * abs(r), (M, m, t, d, r)
                else:
                    rel = abs(d - r) / abs(r)
                    worst[m] = max(worst.get(m, 0.0), rel)
                    assert rel <= 1e-13, (M, m, t, d, r)
    with open(results_path("boys_vs_fgamma_set.json"), "w") as f:
        json.dump({"max_rel_err_by_order": worst, "points": len(T)}, f)
