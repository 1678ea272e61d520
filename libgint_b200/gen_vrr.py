"""Generates csrc/vrr_gen.cuh: straight-line Obara-Saika VRR code, one function per class.

For a class (la, lb, lc, ld) the primitive kernel needs, per surviving image, the targets
(e0|f0)^(0) for e in [la, la+lb] and f in [lc, lc+ld] (reference src/plan.cpp:56-146 builds
the same DAG; src/compute_VRR.cpp:111-345 evaluates it as VRR1..VRR6). The runtime planner
(csrc/plan.cpp) lays the blocks (a|c)^(m) out in a workspace and the interpreted kernels walk
that layout; this generator instead unrolls the same recursion, with the same m ranges and the
same formula per element, into one expression per element, so the compiler keeps the workspace
in registers and every index is resolved at compile time.

Element formulas (pqz layout: PA[3] WP[3] QC[3] WQ[3] i2ab mrab i2cd mrcd i2z; d is the first
axis on which the cartesian function has a nonzero exponent, "-1_d" lowers that exponent):
  (a|0)^m = PA_d (a-1_d|0)^m + WP_d (a-1_d|0)^(m+1)
            + (e_d - 1) (i2ab (a-2_d|0)^m + mrab (a-2_d|0)^(m+1))          if e_d >= 2
  (a|c)^m = QC_d (a|c-1_d)^m + WQ_d (a|c-1_d)^(m+1)
            + (f_d - 1) (i2cd (a|c-2_d)^m + mrcd (a|c-2_d)^(m+1))          if f_d >= 2
            + a_d i2z (a-1_d|c-1_d)^(m+1)                                  if a_d >= 1

Output: for every class with at most VMAX workspace elements, a specialisation
  template <> struct VrrGen<la, lb, lc, ld> {
     static constexpr bool kHas = true; static constexpr int S, s00;
     template <class R, class Out> static __device__ void run(const R *F, const R *z, Out &out);
  };
where F holds (0|0)^(m), m = 0..L, and out(s, v) receives target element s of the contracted-
target layout (one panel per ket shell f over every bra cartesian e, as csrc/plan.cpp). The
(00|00) target is not emitted when la = lc = 0: the kernel sums it over every image itself.

Run:  python -m libgint_b200.gen_vrr     (rewrites csrc/vrr_gen.cuh)
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "csrc", "vrr_gen.cuh")
VMAX = 300     # classes up to this VRR size get generated code (larger ones compile too slowly)
VREG = 300     # above this size the workspace is a per-lane array instead of named values
LMAX = 3


def ncart(l):
    return (l + 1) * (l + 2) // 2


def cart(l, i):
    """Exponents (x, y, z) of cartesian i of shell l (index a(a+1)/2 + z with a = y + z)."""
    a = 0
    while (a + 1) * (a + 2) // 2 <= i:
        a += 1
    z = i - a * (a + 1) // 2
    return (l - a, a - z, z)


def cidx(e):
    a = e[1] + e[2]
    return a * (a + 1) // 2 + e[2]


def first_dir(e):
    return 0 if e[0] else (1 if e[1] else 2)


def lowered(e, d, n=1):
    f = list(e)
    f[d] -= n
    return tuple(f)


def plan(la, lb, lc, ld):
    """Blocks (a, c, lo, hi) in level order and the target layout, as csrc/plan.cpp."""
    LAB, LCD = la + lb, lc + ld
    L = LAB + LCD
    lo = {}
    hi = {}

    def upd(a, c, l0, h0):
        lo[(a, c)] = min(lo.get((a, c), 99), l0)
        hi[(a, c)] = max(hi.get((a, c), -1), h0)

    for e in range(la, LAB + 1):
        for f in range(lc, LCD + 1):
            upd(e, f, 0, 0)
    for t in range(L, 0, -1):
        for a in range(0, min(t, LAB) + 1):
            c = t - a
            if c > LCD or (a, c) not in hi:
                continue
            l0, h0 = lo[(a, c)], hi[(a, c)]
            if c == 0:
                upd(a - 1, 0, l0, h0 + 1)
                if a >= 2:
                    upd(a - 2, 0, l0, h0 + 1)
            else:
                upd(a, c - 1, l0, h0 + 1)
                if c >= 2:
                    upd(a, c - 2, l0, h0 + 1)
                if a >= 1:
                    upd(a - 1, c - 1, l0 + 1, h0 + 1)
    blocks = []
    for t in range(0, L + 1):
        for a in range(0, min(t, LAB) + 1):
            c = t - a
            if c > LCD or (a, c) not in hi:
                continue
            blocks.append((a, c, lo[(a, c)], hi[(a, c)]))
    V = sum((h - l + 1) * ncart(a) * ncart(c) for a, c, l, h in blocks)
    nE = sum(ncart(e) for e in range(la, LAB + 1))
    Eoff, off = {}, 0
    for e in range(la, LAB + 1):
        Eoff[e] = off
        off += ncart(e)
    Foff, s = {}, 0
    for f in range(lc, LCD + 1):
        Foff[f] = s
        s += nE * ncart(f)
    return dict(blocks=blocks, V=V, S=s, Eoff=Eoff, Foff=Foff, L=L, LAB=LAB, LCD=LCD)


def _num(x):
    return f"R({float(x):.1f})"


def gen_class(la, lb, lc, ld, vreg=VREG):
    p = plan(la, lb, lc, ld)
    if p["V"] <= vreg:
        # named values: the compiler keeps the live ones in registers
        name = lambda a, c, i, k, m: f"x{a}_{c}_{i}_{k}_{m}"
        decl = "const R "
    else:
        # one per-lane array with compile-time indices (too many values for registers; this also
        # keeps the register allocator's work linear in the number of elements)
        off = {}
        o = 0
        for a, c, l0, h0 in p["blocks"]:
            for m in range(l0, h0 + 1):
                for i in range(ncart(a)):
                    for k in range(ncart(c)):
                        off[(a, c, i, k, m)] = o
                        o += 1
        name = lambda a, c, i, k, m: f"w[{off[(a, c, i, k, m)]}]"
        decl = ""
    lines = [] if p["V"] <= vreg else [f"      R w[{p['V']}];"]
    for a, c, l0, h0 in p["blocks"]:
        for m in range(l0, h0 + 1):
            for i in range(ncart(a)):
                for k in range(ncart(c)):
                    n = name(a, c, i, k, m)
                    if a == 0 and c == 0:
                        lines.append(f"      {decl}{n} = F[{m}];")
                        continue
                    if c == 0:
                        e = cart(a, i)
                        d = first_dir(e)
                        im = cidx(lowered(e, d))
                        expr = f"PA{d} * {name(a - 1, 0, im, 0, m)} + WP{d} * {name(a - 1, 0, im, 0, m + 1)}"
                        if e[d] >= 2:
                            iw = cidx(lowered(e, d, 2))
                            inner = f"i2ab * {name(a - 2, 0, iw, 0, m)} + mrab * {name(a - 2, 0, iw, 0, m + 1)}"
                            expr += f" + ({inner})" if e[d] == 2 else f" + {_num(e[d] - 1)} * ({inner})"
                    else:
                        ea, fc = cart(a, i), cart(c, k)
                        d = first_dir(fc)
                        km = cidx(lowered(fc, d))
                        expr = f"QC{d} * {name(a, c - 1, i, km, m)} + WQ{d} * {name(a, c - 1, i, km, m + 1)}"
                        if fc[d] >= 2:
                            kw = cidx(lowered(fc, d, 2))
                            inner = f"i2cd * {name(a, c - 2, i, kw, m)} + mrcd * {name(a, c - 2, i, kw, m + 1)}"
                            expr += f" + ({inner})" if fc[d] == 2 else f" + {_num(fc[d] - 1)} * ({inner})"
                        if a > 0 and ea[d] >= 1:
                            im = cidx(lowered(ea, d))
                            t3 = f"i2z * {name(a - 1, c - 1, im, km, m + 1)}"
                            expr += f" + {t3}" if ea[d] == 1 else f" + {_num(ea[d])} * {t3}"
                    lines.append(f"      {decl}{n} = {expr};")
    want00 = la == 0 and lc == 0
    outs = []
    for e in range(la, p["LAB"] + 1):
        for f in range(lc, p["LCD"] + 1):
            if want00 and e == 0 and f == 0:
                continue
            for i in range(ncart(e)):
                for k in range(ncart(f)):
                    s = p["Foff"][f] + (p["Eoff"][e] + i) * ncart(f) + k
                    outs.append((s, name(e, f, i, k, 0)))
    outs.sort()
    body = "\n".join(lines)
    s00 = p["Foff"][0] + p["Eoff"][0] * 1 if want00 else -1
    head = [
        f"// class ({la}{lb}|{lc}{ld}): L = {p['L']}, {p['V']} VRR elements, {p['S']} targets",
        "template <>",
        f"struct VrrGen<{la}, {lb}, {lc}, {ld}> {{",
        "   static constexpr bool kHas = true;",
        f"   static constexpr int S = {p['S']};",
        f"   static constexpr int s00 = {s00};",
        f"   static constexpr int nout = {len(outs)};",
        "   template <class R, class Out>",
        "   static __device__ __forceinline__ void run(const R *__restrict__ F, const R *__restrict__ z, Out &out) {",
    ]
    if p["V"] > 1:
        head.append("      const R PA0 = z[0], PA1 = z[1], PA2 = z[2], WP0 = z[3], WP1 = z[4], WP2 = z[5];")
        head.append("      const R QC0 = z[6], QC1 = z[7], QC2 = z[8], WQ0 = z[9], WQ1 = z[10], WQ2 = z[11];")
        head.append("      const R i2ab = z[12], mrab = z[13], i2cd = z[14], mrcd = z[15], i2z = z[16];")
    tail = [f"      out({s}, {n});" for s, n in outs]
    unused = ("      (void)PA0; (void)PA1; (void)PA2; (void)WP0; (void)WP1; (void)WP2; (void)QC0; (void)QC1;"
              " (void)QC2; (void)WQ0; (void)WQ1; (void)WQ2; (void)i2ab; (void)mrab; (void)i2cd; (void)mrcd;"
              " (void)i2z;") if p["V"] > 1 else "      (void)z; (void)out; (void)F;"
    return "\n".join(head + [body] + tail + [unused, "   }", "};", ""]), p


def generate(vmax=VMAX):
    parts = [
        "// vrr_gen.cuh -- GENERATED by libgint_b200/gen_vrr.py; do not edit.",
        "// Straight-line Obara-Saika VRR per angular-momentum class (see the generator's docstring).",
        "#pragma once",
        "// generated intermediates that a class never reads are left to the compiler to drop",
        "#pragma nv_diagnostic push",
        "#pragma nv_diag_suppress 177",
        "",
        "namespace gint {",
        "",
        "template <int LA, int LB, int LC, int LD>",
        "struct VrrGen {",
        "   static constexpr bool kHas = false;",
        "   static constexpr int S = 0, s00 = -1, nout = 0;",
        "};",
        "",
    ]
    classes = []
    for la in range(LMAX + 1):
        for lb in range(LMAX + 1):
            for lc in range(LMAX + 1):
                for ld in range(LMAX + 1):
                    p = plan(la, lb, lc, ld)
                    if p["V"] <= vmax:
                        code, _ = gen_class(la, lb, lc, ld)
                        parts.append(code)
                        classes.append(la * 64 + lb * 16 + lc * 4 + ld)
    parts.append("// classes with generated code, c = la*64 + lb*16 + lc*4 + ld")
    parts.append(f"constexpr int kVrrGenCount = {len(classes)};")
    parts.append("constexpr int kVrrGenClasses[kVrrGenCount] = {" + ", ".join(map(str, classes)) + "};")
    parts.append("")
    parts.append("}  // namespace gint")
    parts.append("")
    parts.append("#pragma nv_diagnostic pop")
    parts.append("")
    return "\n".join(parts), classes


def main():
    text, classes = generate()
    with open(OUT, "w") as f:
        f.write(text)
    print(f"wrote {OUT}: {len(classes)} classes")


if __name__ == "__main__":
    main()
