"""The generated straight-line VRR (libgint_b200/csrc/vrr_gen.cuh) against an independent
recursive evaluation of the same Obara-Saika relations, on the host.

The header is compiled as host C++ (g++), every generated class is evaluated on random inputs,
and each target element is compared with a memoised recursion over cartesian exponent triples
that uses the same direction rule (first axis with a nonzero exponent). Also checks that the
committed header is what the generator writes, and that its workspace and target sizes are
the planner's (libgint_plan_sizes).
"""
import ctypes
import functools
import os
import subprocess
import tempfile

import numpy as np
import pytest

from libgint_b200 import gen_vrr

HEADER = gen_vrr.OUT


def test_header_is_current():
    text, _ = gen_vrr.generate()
    with open(HEADER) as f:
        assert f.read() == text, "csrc/vrr_gen.cuh is stale: run python -m libgint_b200.gen_vrr"


def test_sizes_match_planner():
    from libgint_b200.capi import load_engine
    lib = load_engine()
    out = (ctypes.c_int * 8)()
    for la in range(4):
        for lb in range(4):
            for lc in range(4):
                for ld in range(4):
                    p = gen_vrr.plan(la, lb, lc, ld)
                    assert lib.libgint_plan_sizes(la, lb, lc, ld, out)
                    assert (p["V"], p["S"]) == (out[0], out[1]), (la, lb, lc, ld)


@pytest.fixture(scope="module")
def harness():
    _, classes = gen_vrr.generate()
    d = tempfile.mkdtemp()
    src = os.path.join(d, "h.cpp")
    cases = "\n".join(
        f"      case {c}: {{ gint::VrrGen<{c >> 6}, {(c >> 4) & 3}, {(c >> 2) & 3}, {c & 3}>::run(F, z, o); return 1; }}"
        for c in classes)
    with open(src, "w") as f:
        f.write(f"""
#define __device__
#define __forceinline__ inline
#define __restrict__
#include "{HEADER}"
struct Collect {{ double *o; void operator()(int s, double v) {{ o[s] = v; }} }};
extern "C" int vrr_gen_eval(int cls, const double *F, const double *z, double *out) {{
   Collect o{{out}};
   switch (cls) {{
{cases}
      default: return 0;
   }}
}}
""")
    so = os.path.join(d, "h.so")
    subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-w", "-o", so, src], check=True)
    lib = ctypes.CDLL(so)
    lib.vrr_gen_eval.restype = ctypes.c_int
    return lib, classes


def _reference(la, lb, lc, ld, F, z):
    PA, WP, QC, WQ = z[0:3], z[3:6], z[6:9], z[9:12]
    i2ab, mrab, i2cd, mrcd, i2z = z[12:17]

    @functools.lru_cache(maxsize=None)
    def v(a, c, m):
        if sum(c) == 0:
            if sum(a) == 0:
                return F[m]
            d = gen_vrr.first_dir(a)
            a1 = gen_vrr.lowered(a, d)
            r = PA[d] * v(a1, c, m) + WP[d] * v(a1, c, m + 1)
            if a[d] >= 2:
                a2 = gen_vrr.lowered(a, d, 2)
                inner = i2ab * v(a2, c, m) + mrab * v(a2, c, m + 1)
                r = r + (inner if a[d] == 2 else float(a[d] - 1) * inner)
            return r
        d = gen_vrr.first_dir(c)
        c1 = gen_vrr.lowered(c, d)
        r = QC[d] * v(a, c1, m) + WQ[d] * v(a, c1, m + 1)
        if c[d] >= 2:
            c2 = gen_vrr.lowered(c, d, 2)
            inner = i2cd * v(a, c2, m) + mrcd * v(a, c2, m + 1)
            r = r + (inner if c[d] == 2 else float(c[d] - 1) * inner)
        if sum(a) > 0 and a[d] >= 1:
            x3 = v(gen_vrr.lowered(a, d), c1, m + 1)
            r = r + (i2z * x3 if a[d] == 1 else (float(a[d]) * i2z) * x3)
        return r

    p = gen_vrr.plan(la, lb, lc, ld)
    out = np.full(p["S"], np.nan)
    for e in range(la, la + lb + 1):
        for f in range(lc, lc + ld + 1):
            if la == 0 and lc == 0 and e == 0 and f == 0:
                continue
            for i in range(gen_vrr.ncart(e)):
                for k in range(gen_vrr.ncart(f)):
                    s = p["Foff"][f] + (p["Eoff"][e] + i) * gen_vrr.ncart(f) + k
                    out[s] = v(gen_vrr.cart(e, i), gen_vrr.cart(f, k), 0)
    return out


def test_generated_vrr_matches_recursion(harness):
    lib, classes = harness
    rng = np.random.default_rng(7)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for c in classes:
        la, lb, lc, ld = c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3
        L = la + lb + lc + ld
        F = np.ascontiguousarray(rng.uniform(0.1, 1.0, L + 1))
        z = np.ascontiguousarray(rng.uniform(-1.0, 1.0, 17))
        ref = _reference(la, lb, lc, ld, tuple(F), tuple(z))
        got = np.full(ref.size, np.nan)
        assert lib.vrr_gen_eval(c, dp(F), dp(z), dp(got)) == 1
        mask = ~np.isnan(ref)
        assert np.array_equal(np.isnan(got), ~mask), c
        assert np.array_equal(got[mask], ref[mask]), (c, np.abs(got[mask] - ref[mask]).max())


_VOP = np.dtype([("out", "<i2"), ("i0", "<i2"), ("i1", "<i2"), ("i2", "<i2"), ("i3", "<i2"), ("i4", "<i2"),
                 ("zA", "u1"), ("kind", "u1"), ("f1", "i1"), ("f2", "i1")])


def _run_vops(lib, la, lb, lc, ld, F, z):
    """Runs the engine's precompiled VRR instructions of one class (libgint_vrr_program) in order,
    with the formula the large-class primitive kernels apply, and gathers the targets."""
    info = (ctypes.c_int * (4 + 5 * 64))()
    n = lib.libgint_vrr_program(la, lb, lc, ld, None, 0, info, len(info))
    buf = np.zeros(max(n, 1), dtype=_VOP)
    assert lib.libgint_vrr_program(la, lb, lc, ld, buf.ctypes.data, n, info, len(info)) == n
    V, S, n00, ntg = info[0], info[1], info[2], info[3]
    w = [0.0] * (V + 1)
    for q in range(n00):
        w[q] = F[q]
    for o in buf[:n].tolist():
        out, i0, i1, i2, i3, i4, zA, kind, f1, f2 = o
        v = z[zA] * w[i0] + z[zA + 3] * w[i1]
        if f1:
            v += f1 * (z[12 + 2 * kind] * w[i2] + z[13 + 2 * kind] * w[i3])
        if f2:
            v += f2 * z[16] * w[i4]
        w[out] = v
    got = np.full(S, np.nan)
    for t in range(ntg):
        voff, soff, cnt, e, f = info[4 + 5 * t:9 + 5 * t]
        if la == 0 and lc == 0 and e == 0 and f == 0:
            continue          # the (00|00) target is summed over every image by the kernels
        got[soff:soff + cnt] = w[voff:voff + cnt]
    return got


@pytest.mark.parametrize("c", range(256), ids=lambda c: "%d%d%d%d" % (c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3))
def test_vrr_instructions_match_recursion(c):
    """The VRR instruction table of every class (k_prim2 and the team kernel run it on the GPU)
    gives the recursion's targets bit for bit: same operations in the same order."""
    from libgint_b200.capi import load_engine
    lib = load_engine()
    la, lb, lc, ld = c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3
    rng = np.random.default_rng(1000 + c)
    F = tuple(rng.uniform(0.1, 1.0, la + lb + lc + ld + 1).tolist())
    z = tuple(rng.uniform(-1.0, 1.0, 17).tolist())
    ref = _reference(la, lb, lc, ld, F, z)
    got = _run_vops(lib, la, lb, lc, ld, F, z)
    mask = ~np.isnan(ref)
    assert np.array_equal(np.isnan(got), ~mask), c
    assert np.array_equal(got[mask], ref[mask]), (c, np.abs(got[mask] - ref[mask]).max())
