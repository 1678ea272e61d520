// engine_types.h -- records and per-class plans shared by the host engine and the kernels.
#pragma once
#include <cstdint>

namespace gint {

constexpr int kMaxL = 3;             // per centre (reference limit, src/define.h:42-55)
constexpr int kMaxLL = 4 * kMaxL;    // la+lb+lc+ld
constexpr int kMaxPrm = 16;          // primitives per set
constexpr int kMaxNl = 4;            // contractions per set
constexpr int kMaxCell = 256;        // periodic images

// One basis entry = (set, angular-momentum slot): centre, exponents and normalised coefficients.
struct BasisEnt {
   double R[3];
   int z_off;        // exponents in the double pool
   int k_off;        // coefficients (nl rows of np) in the double pool
   int np, nl, l, pad;
};

// One shell quartet (an add_shell for one l-combination): four basis entries and the image
// pair of b (n1) and d (n2).
struct ShellRec {
   uint32_t ent[4];
   uint32_t prm_off;    // first primitive quartet of this shell in the batch
   uint32_t nprm;
   uint16_t n1, n2;
   uint32_t group;      // owning group in the class segment (for the primitive kernel's records: the
                        // set quartet's first group)
};

// All image pairs of one set quartet for one class, and its contraction rows.
struct GroupRec {
   uint32_t shell_off, nshell;
   uint32_t qrtt_off;   // first KS record; the group owns nla*nlb*nlc*nld consecutive rows
   uint8_t nl[4];
   float bound;         // largest Schwarz bound of its shell quartets given by the caller (+inf: none)
};

// One row of the exchange update (reference KS record, src/define.h:172-179, decoded).
struct QrttRec {
   uint32_t off[4];     // ac, ad, bc, bd
   uint8_t ld[4];       // ld_ac, ld_ad, ld_bc, ld_bd (< 256 as in the reference encoding)
   uint8_t T;           // bit0 Tac, bit1 Tad, bit2 Tbc, bit3 Tbd
   uint8_t idx_fac;     // 0..4 -> {2, 1, 0.5, 0.25, 0}
   uint8_t pad[2];
};

// ---------------------------------------------------------------------------------------
// Per-class plan (built on the host by plan.cpp, read by the kernels from global memory).
// ---------------------------------------------------------------------------------------
// VRR block (a|c)^(m), m = lo..lo+nm-1, stored [m][i][k] at off in the VRR workspace.
struct VBlock {
   int8_t a, c, lo, nm;
   int off;
   int in1, in2, in3;     // offsets of (a-1|c)/(a|c-1), (a-2|c)/(a|c-2), (a-1|c-1); -1 if absent
   int8_t lo1, lo2, lo3, pad;
   int nelem;
};

// HRR step on a contracted block. type 0 = ket (e0|c d) from (e0|c+1 d-1), (e0|c d-1) for
// all e at once; type 1 = bra (a b|LC LD) from (a+1 b-1|), (a b-1|).
struct HOp {
   int8_t type, x, y, pad;   // ket: x=c, y=d ; bra: x=a, y=b
   int out, in1, in2;
   int n0;                   // leading (batch) extent: nE for ket, ncart(a) for bra
   int nelem;
};

// One VRR element as a precompiled instruction (see build_vops in plan.cpp): the element's
// workspace offset, its inputs, the pqz slot of its first factor and its integer multipliers.
//   A form (kind 0):  w[out] = z[zA] w[i0] + z[zA+3] w[i1] + f1 (z[12] w[i2] + z[13] w[i3])
//   C form (kind 1):  w[out] = z[zA] w[i0] + z[zA+3] w[i1] + f1 (z[14] w[i2] + z[15] w[i3])
//                              + f2 z[16] w[i4]
// Absent inputs point at a zero slot (offset V) and carry a zero multiplier.
struct VOp {
   int16_t out, i0, i1, i2, i3, i4;
   uint8_t zA, kind;
   int8_t f1, f2;
};

constexpr int kMaxVB = 64;
constexpr int kMaxLev = 16;
constexpr int kMaxTgt = 16;
constexpr int kMaxHop = 32;

struct ClassPlan {
   int la, lb, lc, ld, L;
   int V;                  // VRR workspace doubles
   int S;                  // contracted-target doubles (HRR input)
   int H;                  // HRR workspace doubles (S region first)
   int Nc, Ns, nE;
   int out_off;            // offset of the final cartesian block in the HRR workspace
   int nvb, nlev;
   int lev_off[kMaxLev + 1];
   int ntg;                // VRR targets (e,f), m = 0
   int tg_voff[kMaxTgt * 4], tg_soff[kMaxTgt * 4], tg_n[kMaxTgt * 4], tg_e[kMaxTgt * 4], tg_f[kMaxTgt * 4];
   int nhop, nhlev;
   int hlev_off[kMaxLev + 1];
   int vop_off, nvop;      // the class's VRR instructions in the engine's VOp table
   int vop_lev[kMaxLev + 1];   // level l (1..nlev) is instructions [vop_lev[l-1], vop_lev[l])
   int want00;             // la == 0 && lc == 0: the (00|00) target collects every image
   int s00;                // offset of the (00|00) target in S (if want00)
   VBlock vb[kMaxVB];
   HOp hop[kMaxHop];
};

}  // namespace gint
