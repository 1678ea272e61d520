"""The HRR instructions of the interpreted group kernel (one record per HRR workspace element,
built on the host for every class and copied to each GPU) reproduce the HRR recursion: run on
random inputs they give the cartesian block, bit for bit, that the straight-line HRR written by
gen_grp.py gives (the generated group kernel's code, which the GPU tests check against the oracle
for the classes it is compiled for). Both sides run here in Python with the same operations in the
same order. Reference recursion: src/compute_HRR.cpp:7-99."""
import ctypes
import re

import numpy as np
import pytest

from libgint_b200.gen_grp import gen_class
from libgint_b200.gen_vrr import ncart


def _program(lib, la, lb, lc, ld):
    info = (ctypes.c_int * 4)()
    n = lib.libgint_hrr_program(la, lb, lc, ld, None, 0, info)
    assert n >= 0
    buf = (ctypes.c_uint * (2 * max(n, 1)))()
    assert lib.libgint_hrr_program(la, lb, lc, ld, buf, n, info) == n
    return np.frombuffer(buf, dtype=np.uint32).reshape(-1, 2)[:n].astype(np.int64), list(info)


def _run_program(rec, info, T, AB, CD):
    S, H, out_off, ket = info
    assert S + len(rec) == H
    w = np.zeros(H)
    w[:S] = T
    wl = w.tolist()
    in1 = (rec[:, 0] & 0x3FFFFFFF).tolist()
    ax = (rec[:, 0] >> 30).tolist()
    in2 = rec[:, 1].tolist()
    for i in range(len(in1)):
        R = CD if i < ket else AB
        wl[S + i] = wl[in1[i]] + R[ax[i]] * wl[in2[i]]
    return wl, out_off


def _run_generated(la, lb, lc, ld, T, AB, CD):
    code = gen_class(la, lb, lc, ld)
    body = code.split("void hrr(")[1].split("static __device__")[0]
    lines = []
    for ln in body.splitlines():
        ln = ln.strip()
        m = re.match(r"const (?:double|R) (\w+) = (.*);$", ln)
        if m:
            lines.append(f"{m.group(1)} = {m.group(2)}")
            continue
        m = re.match(r"cart\[(\d+)\] \+= (.*);$", ln)
        if m:
            lines.append(f"cart[{m.group(1)}] += {m.group(2)}")
    nc = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    env = {"T": T, "AB": AB, "CD": CD, "cart": [0.0] * nc}
    exec(compile("\n".join(lines), f"hrr_{la}{lb}{lc}{ld}", "exec"), env)
    return env["cart"]


CLASSES = [(la, lb, lc, ld) for la in range(4) for lb in range(4) for lc in range(4) for ld in range(4)]


@pytest.mark.parametrize("cls", CLASSES, ids=lambda c: "%d%d%d%d" % c)
def test_hrr_program_matches_generated_hrr(cls):
    from libgint_b200.capi import load_engine
    lib = load_engine()
    la, lb, lc, ld = cls
    rec, info = _program(lib, la, lb, lc, ld)
    rng = np.random.default_rng(la * 64 + lb * 16 + lc * 4 + ld)
    T = rng.standard_normal(info[0]).tolist()
    AB = rng.standard_normal(3).tolist()
    CD = rng.standard_normal(3).tolist()
    w, out_off = _run_program(rec, info, T, AB, CD)
    cart = _run_generated(la, lb, lc, ld, T, AB, CD)
    assert w[out_off:out_off + len(cart)] == cart


def test_hrr_program_rejects_unsupported_class():
    from libgint_b200.capi import load_engine
    lib = load_engine()
    assert lib.libgint_hrr_program(4, 0, 0, 0, None, 0, None) == -1
