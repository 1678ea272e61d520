"""The engine's per-class recursion plan against the reference planner (src/plan.cpp:217).

The VRR workspace holds the same (a|c)^(m) blocks with the same m ranges, and the HRR workspace
the same intermediate blocks, so their sizes equal the reference's pr_size and sh_size for every
class with l <= 3.
"""
import ctypes
import itertools
import os

import numpy as np

from conftest import GOLDEN


def test_plan_sizes_match_reference():
    from libgint_b200.capi import load_engine
    lib = load_engine()
    gold = np.load(os.path.join(GOLDEN, "ref_host_vectors.npz"))["plan"]
    out = np.zeros(8, np.int32)
    for la, lb, lc, ld in itertools.product(range(4), repeat=4):
        assert lib.libgint_plan_sizes(la, lb, lc, ld, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        pr, sh = gold[la * 64 + lb * 16 + lc * 4 + ld][:2]
        assert out[0] == pr and out[2] == sh, (la, lb, lc, ld, out[:3], pr, sh)
        nc = lambda l: (l + 1) * (l + 2) // 2
        assert out[3] == nc(la) * nc(lb) * nc(lc) * nc(ld)
        assert out[4] == (2 * la + 1) * (2 * lb + 1) * (2 * lc + 1) * (2 * ld + 1)


def test_flop_model_positive():
    from libgint_b200.capi import load_engine
    lib = load_engine()
    fl = (ctypes.c_double * 8)()
    assert lib.libgint_plan_flops(0, 0, 0, 0, fl)
    assert fl[0] == 2 * 105 + 2 * 14 + 52 and fl[2] == 0.0
    assert lib.libgint_plan_flops(2, 2, 2, 2, fl)
    assert fl[2] > 0 and fl[5] > 0
    assert not lib.libgint_plan_flops(4, 0, 0, 0, fl)


def test_engine_host_tables_match_reference():
    """Boys table, c2s, patch maps and (B,W) that the engine uploads equal the reference's."""
    from libgint_b200.capi import load_engine
    lib = load_engine()
    gold = np.load(os.path.join(GOLDEN, "ref_host_vectors.npz"))
    ft = np.zeros(121 * 28); c2s = np.zeros(4 * 70); lut = np.zeros(2 * 128 * 128, np.uint8); bw = np.zeros(207 * 4)
    D = ctypes.POINTER(ctypes.c_double)
    lib.libgint_host_tables(ft.ctypes.data_as(D), c2s.ctypes.data_as(D),
                            lut.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), bw.ctypes.data_as(D))
    assert np.array_equal(ft, gold["ftable"])
    assert np.array_equal(lut[:16384], gold["lut_low"]) and np.array_equal(lut[16384:], gold["lut_high"])
    assert np.array_equal(bw, gold["bw"])
    off = [0, 1, 10, 40]
    for l in range(4):
        nc, ns = (l + 1) * (l + 2) // 2, 2 * l + 1
        assert np.array_equal(c2s[l * 70:l * 70 + ns * nc], gold["c2s"][off[l]:off[l] + ns * nc]), l
