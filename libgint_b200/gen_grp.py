"""Generates csrc/grp_gen.cuh: straight-line HRR and cartesian -> spherical code per class.

After the contraction over primitives, each shell quartet of a set quartet goes through the HRR
(reference src/compute_HRR.cpp:7-99: HRR1 on the ket, then HRR2 on the bra) and the sum over
image pairs; the sum is transformed to real solid harmonics one centre at a time (reference
src/compute_SPH.cpp:58-237 with the coefficients of src/c2s.h). csrc/plan.cpp lays these steps
out for the interpreted group kernel; this generator unrolls the same steps, in the same order and
with the same formula per element, for the per-lane group kernel:
  ket  (e0|c d)[x][k][l] = (e0|c+1_t d-1_t)[x][k+1_t][l-1_t] + CD_t (e0|c d-1_t)[x][k][l-1_t]
  bra  (a b|cd)[i][j][q] = (a+1_t b-1_t|cd)[i+1_t][j-1_t][q] + AB_t (a b-1_t|cd)[i][j-1_t][q]
where t is the first axis on which cartesian l (of d) or j (of b) has a nonzero exponent.

The spherical coefficients are written as literals, zero entries skipped. They are computed by
the formula the engine's host tables use (CP2K's normalisation, l = 3 entries rounded to nine
decimals); tests/test_grp_gen.py checks them bit for bit against libgint_host_tables.

Output per class with L = la+lb+lc+ld <= LGMAX and an HRR workspace of at most HMAX doubles:
  template <> struct GrpGen<la, lb, lc, ld> {
     static constexpr bool kHas = true; static constexpr int S, Nc, Ns;
     template <class R> static __device__ void hrr(const R *T, const R *AB, const R *CD, R *cart);  // cart += ...
     template <class R> static __device__ void sph(const R *cart, R *out);
  };

Run:  python -m libgint_b200.gen_grp     (rewrites csrc/grp_gen.cuh)
"""
import math
import os

from libgint_b200.gen_vrr import cart, cidx, first_dir, lowered, ncart, plan

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "csrc", "grp_gen.cuh")
HMAX = 140
LGMAX = 3      # one lane per contraction row up to L = 3; at L = 4 (up to 100 targets per lane,
               # 255 registers with spills) it was slower than the warp kernels for most classes
LMAX = 3

# unnormalised real solid harmonics as integer coefficients on the cartesian monomials, rows
# m = -l..l (CP2K order; the same rows as the engine's make_c2s)
_SH = {
    1: [[0, 1, 0], [0, 0, 1], [1, 0, 0]],
    2: [[0, 1, 0, 0, 0, 0], [0, 0, 0, 0, 1, 0], [-1, 0, 0, -1, 0, 2], [0, 0, 1, 0, 0, 0], [1, 0, 0, -1, 0, 0]],
    3: [[0, 3, 0, 0, 0, 0, -1, 0, 0, 0], [0, 0, 0, 0, 1, 0, 0, 0, 0, 0], [0, -1, 0, 0, 0, 0, -1, 0, 4, 0],
        [0, 0, -3, 0, 0, 0, 0, -3, 0, 2], [-1, 0, 0, -1, 0, 4, 0, 0, 0, 0], [0, 0, 1, 0, 0, 0, 0, -1, 0, 0],
        [1, 0, 0, -3, 0, 0, 0, 0, 0, 0]],
}


def _dfact(n):
    r = 1.0
    k = n
    while k > 1:
        r *= k
        k -= 2
    return r


def _round_half_away(x):
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def c2s(l):
    """[2l+1][ncart(l)] coefficients, evaluated as the engine's make_c2s does."""
    if l == 0:
        return [[1.0]]
    nc = ncart(l)
    out = []
    for row in _SH[l]:
        n2 = 0.0
        for i in range(nc):
            for j in range(nc):
                if not row[i] or not row[j]:
                    continue
                e1, e2 = cart(l, i), cart(l, j)
                o = 1.0
                for d in range(3):
                    s = e1[d] + e2[d]
                    if s & 1:
                        o = 0.0
                        break
                    o *= _dfact(s - 1)
                n2 += row[i] * row[j] * o
        nr = math.sqrt(n2)
        vals = []
        for i in range(nc):
            v = row[i] / nr
            if l >= 3:
                v = _round_half_away(v * 1e9) / 1e9
            vals.append(v)
        out.append(vals)
    return out


def hrr_size(la, lb, lc, ld):
    """Workspace doubles of the HRR (targets + intermediates), as csrc/plan.cpp counts H."""
    p = plan(la, lb, lc, ld)
    nE = sum(ncart(e) for e in range(la, la + lb + 1))
    h = p["S"]
    LCD = lc + ld
    for d in range(1, ld + 1):
        for c in range(lc, LCD - d + 1):
            h += nE * ncart(c) * ncart(d)
    ncd = ncart(lc) * ncart(ld)
    LAB = la + lb
    for b in range(1, lb + 1):
        for a in range(la, LAB - b + 1):
            h += ncart(a) * ncart(b) * ncd
    return h


def _inc(e, d):
    f = list(e)
    f[d] += 1
    return tuple(f)


def gen_class(la, lb, lc, ld):
    p = plan(la, lb, lc, ld)
    LAB, LCD = la + lb, lc + ld
    Eoff = p["Eoff"]
    nE = sum(ncart(e) for e in range(la, LAB + 1))
    Erows = []          # E row x -> (e, ie)
    for e in range(la, LAB + 1):
        for ie in range(ncart(e)):
            Erows.append((e, ie))
    lines = []
    # ket values K[(c, d)][(x, k, l)] -> expression name
    K = {}
    for c in range(lc, LCD + 1):
        for x in range(nE):
            for k in range(ncart(c)):
                K[(c, 0, x, k, 0)] = f"T[{p['Foff'][c] + x * ncart(c) + k}]"
    for d in range(1, ld + 1):
        for c in range(lc, LCD - d + 1):
            for x in range(nE):
                for k in range(ncart(c)):
                    for l in range(ncart(d)):
                        ed = cart(d, l)
                        t = first_dir(ed)
                        lm = cidx(lowered(ed, t))
                        kp = cidx(_inc(cart(c, k), t))
                        n = f"k{c}_{d}_{x}_{k}_{l}"
                        lines.append(f"      const R {n} = {K[(c + 1, d - 1, x, kp, lm)]} + CD[{t}] * "
                                     f"{K[(c, d - 1, x, k, lm)]};")
                        K[(c, d, x, k, l)] = n
    ncd = ncart(lc) * ncart(ld)
    Bv = {}
    for a in range(la, LAB + 1):
        for i in range(ncart(a)):
            x = Eoff[a] + i
            for kk in range(ncart(lc)):
                for l in range(ncart(ld)):
                    Bv[(a, 0, i, 0, kk * ncart(ld) + l)] = K[(lc, ld, x, kk, l)]
    for b in range(1, lb + 1):
        for a in range(la, LAB - b + 1):
            for i in range(ncart(a)):
                for j in range(ncart(b)):
                    eb = cart(b, j)
                    t = first_dir(eb)
                    jm = cidx(lowered(eb, t))
                    ip = cidx(_inc(cart(a, i), t))
                    for q in range(ncd):
                        n = f"b{a}_{b}_{i}_{j}_{q}"
                        lines.append(f"      const R {n} = {Bv[(a + 1, b - 1, ip, jm, q)]} + AB[{t}] * "
                                     f"{Bv[(a, b - 1, i, jm, q)]};")
                        Bv[(a, b, i, j, q)] = n
    nca, ncb = ncart(la), ncart(lb)
    Nc = nca * ncb * ncd
    for i in range(nca):
        for j in range(ncb):
            for q in range(ncd):
                lines.append(f"      cart[{(i * ncb + j) * ncd + q}] += {Bv[(la, lb, i, j, q)]};")
    hrr_body = "\n".join(lines)

    # cartesian -> spherical, centre a, b, c, d in turn
    ls = [la, lb, lc, ld]
    dims = [ncart(l) for l in ls]
    cur = {}
    for idx in range(Nc):
        cur[idx] = f"cart[{idx}]"
    slines = []
    for ctr in range(4):
        cc = c2s(ls[ctr])
        nd = list(dims)
        nd[ctr] = 2 * ls[ctr] + 1
        stride = 1
        for q in range(ctr + 1, 4):
            stride *= dims[q]
        nxt = {}
        tot = nd[0] * nd[1] * nd[2] * nd[3]
        for t in range(tot):
            rem, id4 = t, [0] * 4
            for q in range(3, -1, -1):
                id4[q] = rem % nd[q]
                rem //= nd[q]
            mi = id4[ctr]
            id4[ctr] = 0
            base = ((id4[0] * dims[1] + id4[1]) * dims[2] + id4[2]) * dims[3] + id4[3]
            if ls[ctr] == 0:
                nxt[t] = cur[base]
                continue
            terms = [(cc[mi][k], cur[base + k * stride]) for k in range(dims[ctr]) if cc[mi][k] != 0.0]
            n = f"s{ctr}_{t}"
            expr = " + ".join(f"R({repr(float(v))}) * {x}" for v, x in terms) if terms else "R(0)"
            slines.append(f"      const R {n} = {expr};")
            nxt[t] = n
        cur = nxt
        dims = nd
    Ns = dims[0] * dims[1] * dims[2] * dims[3]
    for t in range(Ns):
        slines.append(f"      out[{t}] = {cur[t]};")
    sph_body = "\n".join(slines)
    H = hrr_size(la, lb, lc, ld)
    return "\n".join([
        f"// class ({la}{lb}|{lc}{ld}): S = {p['S']}, HRR workspace {H}, Nc = {Nc}, Ns = {Ns}",
        "template <>",
        f"struct GrpGen<{la}, {lb}, {lc}, {ld}> {{",
        "   static constexpr bool kHas = true;",
        f"   static constexpr int S = {p['S']}, Nc = {Nc}, Ns = {Ns};",
        "   template <class R>",
        "   static __device__ __forceinline__ void hrr(const R *__restrict__ T, const R *AB, const R *CD, R *cart) {",
        hrr_body,
        "      (void)AB; (void)CD;",
        "   }",
        "   template <class R>",
        "   static __device__ __forceinline__ void sph(const R *cart, R *out) {",
        sph_body,
        "   }",
        "};",
        "",
    ])


def generate(hmax=HMAX):
    parts = [
        "// grp_gen.cuh -- GENERATED by libgint_b200/gen_grp.py; do not edit.",
        "// Straight-line HRR and cartesian -> spherical transform per class (see the generator).",
        "#pragma once",
        "",
        "namespace gint {",
        "",
        "template <int LA, int LB, int LC, int LD>",
        "struct GrpGen {",
        "   static constexpr bool kHas = false;",
        "};",
        "",
    ]
    classes = []
    for la in range(LMAX + 1):
        for lb in range(LMAX + 1):
            for lc in range(LMAX + 1):
                for ld in range(LMAX + 1):
                    if la + lb + lc + ld <= LGMAX and hrr_size(la, lb, lc, ld) <= hmax:
                        parts.append(gen_class(la, lb, lc, ld))
                        classes.append(la * 64 + lb * 16 + lc * 4 + ld)
    parts.append("// classes with generated code, c = la*64 + lb*16 + lc*4 + ld")
    parts.append(f"constexpr int kGrpGenCount = {len(classes)};")
    parts.append("constexpr int kGrpGenClasses[kGrpGenCount] = {" + ", ".join(map(str, classes)) + "};")
    parts.append("")
    parts.append("}  // namespace gint")
    parts.append("")
    return "\n".join(parts), classes


def main():
    text, classes = generate()
    with open(OUT, "w") as f:
        f.write(text)
    print(f"wrote {OUT}: {len(classes)} classes")


if __name__ == "__main__":
    main()
