"""The truncated-Coulomb coefficient table produced by the workload driver.

G_m(T,R) = (-d/dT)^m G_0(T,R) with G_0 = sqrt(pi)/(4 sqrt T) [2 erf(sqrt T) + erf(R - sqrt T)
- erf(R + sqrt T)]. The driver's direct evaluation is checked against high-precision
derivatives (mpmath); the per-patch Chebyshev fit against the direct evaluation, evaluated
through the oracle's restatement of the reference evaluator.
"""
import ctypes

import numpy as np
import pytest

from conftest import ORACLE_SO
from libgint_b200.workload import _dp, driver

mp = pytest.importorskip("mpmath")


def test_exact_Gm_against_mpmath():
    mp.mp.dps = 40
    g = np.zeros(13)

    def G0(T, R):
        s = mp.sqrt(T)
        return mp.sqrt(mp.pi) / (4 * s) * (2 * mp.erf(s) + mp.erf(R - s) - mp.erf(R + s))

    for T, R in [(0.5, 0.3), (3.0, 2.0), (10.0, 5.0), (40.0, 11.0), (150.0, 12.0), (1.0, 10.0)]:
        driver().gd_tcg_exact(12, T, R, _dp(g))
        ders = mp.diffs(lambda t: G0(t, mp.mpf(R)), mp.mpf(T), 12)
        ref = np.array([float((-1) ** m * v) for m, v in enumerate(ders)])
        assert np.abs(ref - g).max() < 1e-14, (T, R)


def test_Gm_limits():
    g = np.zeros(13)
    F = np.zeros(13)
    # R -> large at moderate T: the operator is the full Coulomb one
    driver().gd_tcg_exact(12, 5.0, 60.0, _dp(g))
    driver().gd_boys(12, 5.0, _dp(F))
    assert np.abs(g - F).max() < 1e-14
    # R -> 0: the truncated operator vanishes
    driver().gd_tcg_exact(12, 5.0, 1e-9, _dp(g))
    assert np.abs(g).max() < 1e-12


def test_fit_accuracy():
    C0 = np.zeros(207 * 13 * 105)
    assert driver().gd_tcg_table(12, _dp(C0)) == 13 * 105
    ora = ctypes.CDLL(ORACLE_SO)
    ora.oracle_tcg.restype = ctypes.c_int
    rng = np.random.default_rng(3)
    f = np.zeros(30)
    g = np.zeros(13)
    worst = 0.0
    for k in range(3000):
        R = rng.uniform(0, 11) if k % 2 else 11 / rng.uniform(0.02, 1)
        lo = 0 if R <= 11 else R * R - 11 * R
        T = rng.uniform(lo, R * R + 11 * R + 50)
        if ora.oracle_tcg(ctypes.c_double(0), _dp(C0), 13 * 105, ctypes.c_double(R), ctypes.c_double(T), 12,
                          ctypes.c_double(1.0), _dp(f)):
            continue
        driver().gd_tcg_exact(12, T, R, _dp(g))
        worst = max(worst, np.abs(f[:13] - g).max())
    assert worst < 1e-10, worst
