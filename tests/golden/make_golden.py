"""Generates tests/golden/ref_host_vectors.npz from the reference's own host-callable code.

Needs oracle/_ref/libref_host.so, built by `make -C oracle ref` from the reference sources
(src/plan.cpp, src/fgamma.cpp, src/t_c_g0_n.cpp, src/util.cpp, src/BW_by_patch.h, src/c2s.h).
The fixture pins the CPU oracle and the engine's tables without the reference tree:
  ftable       create_md_ftable(21, 0, 12, 0.1)                 (src/fgamma.cpp:109)
  lut_low/high fill_x12_to_patch(128, 128)                      (src/t_c_g0_n.cpp:53)
  bw           BW_by_patch                                      (src/BW_by_patch.h)
  c2s          c2s[245]                                         (src/c2s.h:36)
  fg_*         fgamma0(n, T, fac) samples                       (src/fgamma.cpp:196)
  tcg_*        t_c_g0_n_v2 (+fgamma0) samples with a seeded C0  (src/t_c_g0_n.cpp:67)
  pbc_*        compute_pbc samples                              (src/util.cpp:132)
  plan         pr_size, sh_size, numV, numVC, numVCH of plan(la,lb,lc,ld), l<=3 (src/plan.cpp:217)
Run: python tests/golden/make_golden.py
"""
import ctypes
import itertools
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def dp(a):
    return a.ctypes.data_as(_D)


def ip(a):
    return a.ctypes.data_as(_I)


def tcg_C0():
    """The seeded coefficient table used for the t_c_g0_n_v2 samples (13 orders)."""
    return np.random.default_rng(20240607).normal(size=207 * 13 * 105)


def main():
    r = ctypes.CDLL(REF)
    out = {}
    ft = np.zeros(121 * 28); r.ref_ftable(dp(ft)); out["ftable"] = ft
    lo = np.zeros(128 * 128, np.int32); hi = lo.copy(); r.ref_lut(ip(lo), ip(hi))
    out["lut_low"] = lo.astype(np.uint8); out["lut_high"] = hi.astype(np.uint8)
    bw = np.zeros(207 * 4); r.ref_bw(dp(bw)); out["bw"] = bw
    c2s = np.zeros(245); r.ref_c2s(dp(c2s)); out["c2s"] = c2s
    rng = np.random.default_rng(7)
    Ts = np.concatenate([rng.uniform(0, 40, 400), [0.0, 1e-14, 0.05, 0.15, 11.95, 12.0, 12.05, 29.9, 30.1]])
    fg = np.zeros((len(Ts), 4, 13))
    f = np.zeros(30)
    for i, T in enumerate(Ts):
        for j, n in enumerate([0, 3, 8, 12]):
            r.ref_fgamma0(n, ctypes.c_double(T), dp(f), ctypes.c_double(1.3))
            fg[i, j, :n + 1] = f[:n + 1]
    out["fg_T"] = Ts; out["fg_val"] = fg
    C0 = tcg_C0()
    R = np.concatenate([rng.uniform(0, 11, 300), rng.uniform(11, 60, 300), [0.0, 11.0, 11.000001]])
    T = np.array([rng.uniform(0, x * x + 11 * x + 60) for x in R])
    T[-3:] = [0.0, 121.0 + 121.0 + 50.0, 121.0 - 121.0]
    tv = np.zeros((len(R), 13)); tg = np.zeros(len(R), np.int32)
    r.ref_tcg.restype = ctypes.c_int
    for i in range(len(R)):
        tg[i] = r.ref_tcg(dp(C0), 13 * 105, ctypes.c_double(R[i]), ctypes.c_double(T[i]), 12,
                          ctypes.c_double(0.7), dp(f))
        tv[i] = f[:13]
    out["tcg_R"] = R; out["tcg_T"] = T; out["tcg_val"] = tv; out["tcg_gamma"] = tg
    cell = np.array([9.0, 0.3, 0.1, 0.2, 8.0, 0.0, 0.1, 0.0, 10.0])
    cc = np.concatenate([cell, np.linalg.inv(cell.reshape(3, 3)).ravel()])
    A = rng.uniform(-20, 20, (200, 3)); B = rng.uniform(-20, 20, (200, 3)); AB = np.zeros((200, 3))
    x = np.zeros(3)
    for i in range(200):
        r.ref_pbc(dp(np.ascontiguousarray(A[i])), dp(np.ascontiguousarray(B[i])), dp(cc), dp(x)); AB[i] = x
    out["pbc_cell"] = cc; out["pbc_A"] = A; out["pbc_B"] = B; out["pbc_AB"] = AB
    plan = np.zeros((256, 5), np.int32)
    buf = np.zeros(300000, np.int32); info = np.zeros(5, np.int32)
    for la, lb, lc, ld in itertools.product(range(4), repeat=4):
        r.ref_plan(la, lb, lc, ld, ip(buf), buf.size, ip(info))
        plan[la * 64 + lb * 16 + lc * 4 + ld] = info
    out["plan"] = plan
    np.savez_compressed(os.path.join(HERE, "ref_host_vectors.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_host_vectors.npz"))


if __name__ == "__main__":
    main()
