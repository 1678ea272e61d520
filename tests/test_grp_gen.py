"""The generated HRR + spherical transform (libgint_b200/csrc/grp_gen.cuh) against an independent
evaluation on the host.

The header is compiled as host C++ (g++); for every generated class, random contracted targets
and AB/CD go through the generated code and through a memoised HRR recursion over cartesian
exponent triples (same direction rule: first axis with a nonzero exponent) followed by the
spherical transform as a tensor contraction with the engine's own coefficients
(libgint_host_tables). Also checks that the committed header is current, that the HRR
workspace sizes are the planner's and that the literal coefficients are the engine's, bit for bit.
"""
import ctypes
import functools
import os
import subprocess
import tempfile

import numpy as np
import pytest

from libgint_b200 import gen_grp, gen_vrr

HEADER = gen_grp.OUT


def _engine_c2s():
    from libgint_b200.capi import load_engine
    lib = load_engine()
    ft, cs = np.zeros(121 * 28), np.zeros(4 * 70)
    lut, bw = np.zeros(2 * 128 * 128, np.uint8), np.zeros(207 * 4)
    dp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    lib.libgint_host_tables.argtypes = [ctypes.c_void_p] * 4
    lib.libgint_host_tables(dp(ft), dp(cs), dp(lut), dp(bw))
    cs = cs.reshape(4, 70)
    return [cs[l][:(2 * l + 1) * gen_vrr.ncart(l)].reshape(2 * l + 1, gen_vrr.ncart(l)) for l in range(4)]


def test_header_is_current():
    text, _ = gen_grp.generate()
    with open(HEADER) as f:
        assert f.read() == text, "csrc/grp_gen.cuh is stale: run python -m libgint_b200.gen_grp"


def test_sizes_and_coefficients_match_engine():
    from libgint_b200.capi import load_engine
    lib = load_engine()
    out = (ctypes.c_int * 8)()
    for c in range(256):
        la, lb, lc, ld = c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3
        assert lib.libgint_plan_sizes(la, lb, lc, ld, out)
        assert gen_grp.hrr_size(la, lb, lc, ld) == out[2], (la, lb, lc, ld)
    eng = _engine_c2s()
    for l in range(4):
        assert np.array_equal(np.array(gen_grp.c2s(l)), eng[l]), l


@pytest.fixture(scope="module")
def harness():
    _, classes = gen_grp.generate()
    d = tempfile.mkdtemp()
    src = os.path.join(d, "h.cpp")
    cases = "\n".join(
        f"      case {c}: {{ using G = gint::GrpGen<{c >> 6}, {(c >> 4) & 3}, {(c >> 2) & 3}, {c & 3}>;"
        f" double cart[G::Nc] = {{}}; G::hrr(T, AB, CD, cart); for (int q = 0; q < G::Nc; q++) cart_out[q] = cart[q];"
        f" G::sph(cart, sph_out); return 1; }}"
        for c in classes)
    with open(src, "w") as f:
        f.write(f"""
#define __device__
#define __forceinline__ inline
#define __restrict__
#include "{HEADER}"
extern "C" int grp_gen_eval(int cls, const double *T, const double *AB, const double *CD, double *cart_out,
                            double *sph_out) {{
   switch (cls) {{
{cases}
      default: return 0;
   }}
}}
""")
    so = os.path.join(d, "h.so")
    subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-w", "-o", so, src], check=True)
    lib = ctypes.CDLL(so)
    lib.grp_gen_eval.restype = ctypes.c_int
    return lib, classes


def _reference(la, lb, lc, ld, T, AB, CD, c2s):
    p = gen_vrr.plan(la, lb, lc, ld)
    nc = gen_vrr.ncart

    def row(e, ie):
        return p["Eoff"][e] + ie

    @functools.lru_cache(maxsize=None)
    def ket(e, ie, c, d):           # (e0 | c d), c and d exponent triples
        if sum(d) == 0:
            f = sum(c)
            return T[p["Foff"][f] + row(e, ie) * nc(f) + gen_vrr.cidx(c)]
        t = gen_vrr.first_dir(d)
        c1 = list(c); c1[t] += 1
        return ket(e, ie, tuple(c1), gen_vrr.lowered(d, t)) + CD[t] * ket(e, ie, c, gen_vrr.lowered(d, t))

    @functools.lru_cache(maxsize=None)
    def bra(a, b, c, d):
        if sum(b) == 0:
            return ket(sum(a), gen_vrr.cidx(a), c, d)
        t = gen_vrr.first_dir(b)
        a1 = list(a); a1[t] += 1
        return bra(tuple(a1), gen_vrr.lowered(b, t), c, d) + AB[t] * bra(a, gen_vrr.lowered(b, t), c, d)

    cart = np.zeros((nc(la), nc(lb), nc(lc), nc(ld)))
    for i in range(nc(la)):
        for j in range(nc(lb)):
            for k in range(nc(lc)):
                for l in range(nc(ld)):
                    cart[i, j, k, l] = bra(gen_vrr.cart(la, i), gen_vrr.cart(lb, j), gen_vrr.cart(lc, k),
                                           gen_vrr.cart(ld, l))
    sph = np.einsum("ai,bj,ck,dl,ijkl->abcd", c2s[la], c2s[lb], c2s[lc], c2s[ld], cart)
    return cart.ravel(), sph.ravel()


def test_generated_hrr_and_sph_match_reference(harness):
    lib, classes = harness
    c2s = _engine_c2s()
    rng = np.random.default_rng(11)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for c in classes:
        la, lb, lc, ld = c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3
        S = gen_vrr.plan(la, lb, lc, ld)["S"]
        T = np.ascontiguousarray(rng.uniform(-1, 1, S))
        AB = np.ascontiguousarray(rng.uniform(-2, 2, 3))
        CD = np.ascontiguousarray(rng.uniform(-2, 2, 3))
        cart_ref, sph_ref = _reference(la, lb, lc, ld, tuple(T), tuple(AB), tuple(CD), c2s)
        cart = np.zeros(cart_ref.size)
        sph = np.zeros(sph_ref.size)
        assert lib.grp_gen_eval(c, dp(T), dp(AB), dp(CD), dp(cart), dp(sph)) == 1
        assert np.array_equal(cart, cart_ref), (c, np.abs(cart - cart_ref).max())
        scale = max(1.0, np.abs(sph_ref).max())
        assert np.abs(sph - sph_ref).max() <= 1e-13 * scale, (c, np.abs(sph - sph_ref).max())
