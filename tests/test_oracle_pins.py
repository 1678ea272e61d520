"""The CPU oracle's building blocks against the reference's own host code.

Golden vectors (tests/golden/ref_host_vectors.npz, made by tests/golden/make_golden.py from the
reference sources) always run; when oracle/_ref/libref_host.so is present the same checks run
live against it as well. Every comparison is bit-exact: the oracle restates the reference's
formulas in the same operation order.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN, ORACLE_SO, REF_HOST_SO

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def dp(a):
    return a.ctypes.data_as(_D)


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLDEN, "ref_host_vectors.npz"))


@pytest.fixture(scope="module")
def ora():
    lib = ctypes.CDLL(ORACLE_SO)
    lib.oracle_tcg.restype = ctypes.c_int
    return lib


def test_boys_table_bitwise(gold, ora):
    ft = np.zeros(121 * 28)
    ora.oracle_ftable(dp(ft))
    assert np.array_equal(ft, gold["ftable"])


def test_patch_maps_bitwise(gold, ora):
    lo = np.zeros(128 * 128, np.int32)
    hi = lo.copy()
    ora.oracle_lut(lo.ctypes.data_as(_I), hi.ctypes.data_as(_I))
    assert np.array_equal(lo.astype(np.uint8), gold["lut_low"])
    assert np.array_equal(hi.astype(np.uint8), gold["lut_high"])


def test_patch_rectangles_reproduce_bias_weight(gold):
    """The rectangle table (tcg_patches.h) encodes exactly the reference's BW_by_patch."""
    import re
    txt = open(os.path.join(os.path.dirname(ORACLE_SO), "..", "..", "libgint_b200", "csrc", "tcg_patches.h")).read()
    rects = [tuple(map(int, m)) for m in re.findall(r"\{(\d+),(\d+),(\d+),(\d+)\}", txt)]
    assert len(rects) == 207
    bw = np.array([[(a + b) / 128.0, 128.0 / (b - a), (c + d) / 128.0, 128.0 / (d - c)] for a, b, c, d in rects])
    assert np.array_equal(bw.ravel(), gold["bw"])


def test_c2s_bitwise(gold, ora):
    off = [0, 1, 10, 40]
    for l in range(4):
        nc, ns = (l + 1) * (l + 2) // 2, 2 * l + 1
        m = np.zeros(ns * nc)
        ora.oracle_c2s(l, dp(m))
        assert np.array_equal(m, gold["c2s"][off[l]:off[l] + ns * nc]), l


def test_fgamma0_bitwise(gold, ora):
    f = np.zeros(30)
    for i, T in enumerate(gold["fg_T"]):
        for j, n in enumerate([0, 3, 8, 12]):
            ora.oracle_fgamma0(n, ctypes.c_double(T), dp(f), ctypes.c_double(1.3))
            assert np.array_equal(f[:n + 1], gold["fg_val"][i, j, :n + 1]), (T, n)


def test_truncated_coulomb_bitwise(gold, ora):
    from golden.make_golden import tcg_C0
    C0 = tcg_C0()
    f = np.zeros(30)
    for i, (R, T) in enumerate(zip(gold["tcg_R"], gold["tcg_T"])):
        g = ora.oracle_tcg(ctypes.c_double(0), dp(C0), 13 * 105, ctypes.c_double(R), ctypes.c_double(T), 12,
                           ctypes.c_double(0.7), dp(f))
        assert g == gold["tcg_gamma"][i]
        assert np.array_equal(f[:13], gold["tcg_val"][i]), (R, T)


def test_pbc_bitwise(gold, ora):
    x = np.zeros(3)
    cc = np.ascontiguousarray(gold["pbc_cell"])
    for A, B, AB in zip(gold["pbc_A"], gold["pbc_B"], gold["pbc_AB"]):
        ora.oracle_pbc(dp(np.ascontiguousarray(A)), dp(np.ascontiguousarray(B)), dp(cc), dp(x))
        assert np.array_equal(x, AB)


@pytest.mark.skipif(not os.path.exists(REF_HOST_SO), reason="reference host library not built")
def test_live_reference_matches_golden(gold):
    """The committed fixture still matches the reference build of this tree."""
    r = ctypes.CDLL(REF_HOST_SO)
    ft = np.zeros(121 * 28)
    r.ref_ftable(dp(ft))
    assert np.array_equal(ft, gold["ftable"])
    c = np.zeros(245)
    r.ref_c2s(dp(c))
    assert np.array_equal(c, gold["c2s"])
