// plan.cpp -- per-class recursion plan (host).
//
// The Obara-Saika DAG is the one of the reference planner (src/plan.cpp:56-146: HRR2 on the
// bra, HRR1 on the ket, VRR1..6 on (a0|c0)^(m)); the layout is this engine's own:
//  * VRR blocks (a|c)^(m) are grouped by level a+c; all blocks of one level are independent,
//    so a team evaluates a whole level in one pass. Each block keeps only the m range that the
//    targets need, propagated downwards from the targets (e0|f0)^(0).
//  * The contracted targets are stored per ket shell f as one [nE][ncart(f)] panel over every
//    bra shell e in [la, la+lb] (nE cartesians), so each ket HRR step runs over all e at once.
//  * HRR: ket steps (e0|c d) for d = 1..ld, then bra steps (a b|lc ld) for b = 1..lb.
#include <algorithm>
#include <cstring>
#include <vector>
#include "engine_types.h"

namespace gint {

static inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

bool build_class_plan(int la, int lb, int lc, int ld, ClassPlan &p) {
   std::memset(&p, 0, sizeof(p));
   if (la < 0 || lb < 0 || lc < 0 || ld < 0 || la > kMaxL || lb > kMaxL || lc > kMaxL || ld > kMaxL) return false;
   p.la = la; p.lb = lb; p.lc = lc; p.ld = ld;
   const int LAB = la + lb, LCD = lc + ld, L = LAB + LCD;
   p.L = L;
   p.Nc = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
   p.Ns = (2 * la + 1) * (2 * lb + 1) * (2 * lc + 1) * (2 * ld + 1);
   // ---- m ranges needed per (a|c)
   int lo[7][7], hi[7][7];
   for (int a = 0; a < 7; a++) for (int c = 0; c < 7; c++) { lo[a][c] = 99; hi[a][c] = -1; }
   auto upd = [&](int a, int c, int l0, int h0) {
      lo[a][c] = std::min(lo[a][c], l0); hi[a][c] = std::max(hi[a][c], h0);
   };
   for (int e = la; e <= LAB; e++) for (int f = lc; f <= LCD; f++) upd(e, f, 0, 0);
   for (int t = L; t >= 1; t--) {
      for (int a = 0; a <= std::min(t, LAB); a++) {
         int c = t - a;
         if (c > LCD || hi[a][c] < 0) continue;
         int l0 = lo[a][c], h0 = hi[a][c];
         if (c == 0) {
            upd(a - 1, 0, l0, h0 + 1);
            if (a >= 2) upd(a - 2, 0, l0, h0 + 1);
         } else {
            upd(a, c - 1, l0, h0 + 1);
            if (c >= 2) upd(a, c - 2, l0, h0 + 1);
            if (a >= 1) upd(a - 1, c - 1, l0 + 1, h0 + 1);
         }
      }
   }
   // ---- VRR blocks, level by level
   int off = 0, boff[7][7];
   for (int a = 0; a < 7; a++) for (int c = 0; c < 7; c++) boff[a][c] = -1;
   p.nvb = 0;
   int lev = 0;
   p.lev_off[0] = 0;
   for (int t = 0; t <= L; t++) {
      for (int a = 0; a <= std::min(t, LAB); a++) {
         int c = t - a;
         if (c > LCD || hi[a][c] < 0) continue;
         VBlock &b = p.vb[p.nvb++];
         b.a = (int8_t)a; b.c = (int8_t)c; b.lo = (int8_t)lo[a][c]; b.nm = (int8_t)(hi[a][c] - lo[a][c] + 1);
         b.off = off; boff[a][c] = off;
         b.nelem = b.nm * ncart(a) * ncart(c);
         off += b.nelem;
      }
      if (t == 0) p.lev_off[0] = p.nvb;    // level 0 is the (0|0) block, filled from Fm
      else { lev++; p.lev_off[lev] = p.nvb; }
   }
   p.nlev = lev;   // levels 1..nlev are blocks [lev_off[l-1], lev_off[l])
   p.V = off;
   for (int i = 0; i < p.nvb; i++) {
      VBlock &b = p.vb[i];
      int a = b.a, c = b.c;
      b.in1 = b.in2 = b.in3 = -1; b.lo1 = b.lo2 = b.lo3 = 0;
      if (a == 0 && c == 0) continue;
      if (c == 0) {
         b.in1 = boff[a - 1][0]; b.lo1 = (int8_t)lo[a - 1][0];
         if (a >= 2) { b.in2 = boff[a - 2][0]; b.lo2 = (int8_t)lo[a - 2][0]; }
      } else {
         b.in1 = boff[a][c - 1]; b.lo1 = (int8_t)lo[a][c - 1];
         if (c >= 2) { b.in2 = boff[a][c - 2]; b.lo2 = (int8_t)lo[a][c - 2]; }
         if (a >= 1) { b.in3 = boff[a - 1][c - 1]; b.lo3 = (int8_t)lo[a - 1][c - 1]; }
      }
   }
   // ---- contracted targets: panel per f, rows over all bra cartesians e in [la, LAB]
   int Eoff[8] = {0};
   p.nE = 0;
   for (int e = la; e <= LAB; e++) { Eoff[e] = p.nE; p.nE += ncart(e); }
   int Foff[8] = {0}, s = 0;
   for (int f = lc; f <= LCD; f++) { Foff[f] = s; s += p.nE * ncart(f); }
   p.S = s;
   p.ntg = 0;
   p.want00 = (la == 0 && lc == 0) ? 1 : 0;
   p.s00 = 0;
   for (int e = la; e <= LAB; e++) for (int f = lc; f <= LCD; f++) {
      int t = p.ntg++;
      p.tg_e[t] = e; p.tg_f[t] = f;
      p.tg_voff[t] = boff[e][f] + 0;   // m = 0 slice (lo == 0 for every target)
      p.tg_soff[t] = Foff[f] + Eoff[e] * ncart(f);
      p.tg_n[t] = ncart(e) * ncart(f);
   }
   // ---- HRR steps
   int hoff = p.S;
   int kloc[8][4];   // (c, d) -> offset of (e0|c d) panel [nE][nc][nd]
   for (int c = 0; c < 8; c++) for (int d = 0; d < 4; d++) kloc[c][d] = -1;
   for (int c = lc; c <= LCD; c++) kloc[c][0] = Foff[c];
   p.nhop = 0; p.nhlev = 0; p.hlev_off[0] = 0;
   for (int d = 1; d <= ld; d++) {
      for (int c = lc; c <= LCD - d; c++) {
         HOp &h = p.hop[p.nhop++];
         h.type = 0; h.x = (int8_t)c; h.y = (int8_t)d;
         h.out = hoff; h.in1 = kloc[c + 1][d - 1]; h.in2 = kloc[c][d - 1];
         h.n0 = p.nE;
         h.nelem = p.nE * ncart(c) * ncart(d);
         kloc[c][d] = hoff; hoff += h.nelem;
      }
      p.hlev_off[++p.nhlev] = p.nhop;
   }
   const int ncd = ncart(lc) * ncart(ld);
   const int kfin = kloc[lc][ld];
   int bloc[8][4];
   for (int a = 0; a < 8; a++) for (int b = 0; b < 4; b++) bloc[a][b] = -1;
   for (int a = la; a <= LAB; a++) bloc[a][0] = kfin + Eoff[a] * ncd;
   for (int b = 1; b <= lb; b++) {
      for (int a = la; a <= LAB - b; a++) {
         HOp &h = p.hop[p.nhop++];
         h.type = 1; h.x = (int8_t)a; h.y = (int8_t)b;
         h.out = hoff; h.in1 = bloc[a + 1][b - 1]; h.in2 = bloc[a][b - 1];
         h.n0 = ncart(a);
         h.nelem = ncart(a) * ncart(b) * ncd;
         bloc[a][b] = hoff; hoff += h.nelem;
      }
      p.hlev_off[++p.nhlev] = p.nhop;
   }
   p.out_off = bloc[la][lb];
   p.H = hoff;
   return true;
}

// ---- precompiled VRR instructions -------------------------------------------------------
static void cart_exps(int l, int i, int e[3]) {
   int a = 0;
   while ((a + 1) * (a + 2) / 2 <= i) a++;
   e[0] = l - a; e[2] = i - a * (a + 1) / 2; e[1] = a - e[2];
}
static int cart_idx(const int e[3]) { const int a = e[1] + e[2]; return a * (a + 1) / 2 + e[2]; }
static int first_dir(const int e[3]) { return e[0] ? 0 : (e[1] ? 1 : 2); }
static int lowered_idx(const int e[3], int d, int n) { int f[3] = {e[0], e[1], e[2]}; f[d] -= n; return cart_idx(f); }

// Appends the VRR of class p as one instruction per workspace element, level by level, with the
// same inputs and multipliers as the element formulas of the interpreted kernels
// (reference VRR1..VRR6, src/compute_VRR.cpp:111-345), and records the level boundaries.
void build_vops(ClassPlan &p, std::vector<VOp> &out) {
   const int16_t zero = (int16_t)p.V;   // the workspace's zero slot
   p.vop_off = (int)out.size();
   p.vop_lev[0] = 0;
   for (int lv = 1; lv <= p.nlev; lv++) {
      for (int bb = p.lev_off[lv - 1]; bb < p.lev_off[lv]; bb++) {
         const VBlock &b = p.vb[bb];
         const int a = b.a, c = b.c, na = ncart(a), nc = ncart(c);
         for (int mm = 0; mm < b.nm; mm++) for (int i = 0; i < na; i++) for (int k = 0; k < nc; k++) {
            const int m = b.lo + mm;
            VOp o;
            o.out = (int16_t)(b.off + (mm * na + i) * nc + k);
            o.i2 = o.i3 = o.i4 = zero;
            o.f1 = o.f2 = 0;
            int ea[3];
            cart_exps(a, i, ea);
            if (c == 0) {
               const int d = first_dir(ea), im = lowered_idx(ea, d, 1), na1 = ncart(a - 1);
               o.kind = 0; o.zA = (uint8_t)d;
               o.i0 = (int16_t)(b.in1 + (m - b.lo1) * na1 + im);
               o.i1 = (int16_t)(b.in1 + (m + 1 - b.lo1) * na1 + im);
               if (ea[d] >= 2) {
                  const int iw = lowered_idx(ea, d, 2), na2 = ncart(a - 2);
                  o.f1 = (int8_t)(ea[d] - 1);
                  o.i2 = (int16_t)(b.in2 + (m - b.lo2) * na2 + iw);
                  o.i3 = (int16_t)(b.in2 + (m + 1 - b.lo2) * na2 + iw);
               }
            } else {
               int ec[3];
               cart_exps(c, k, ec);
               const int d = first_dir(ec), km = lowered_idx(ec, d, 1), nc1 = ncart(c - 1);
               o.kind = 1; o.zA = (uint8_t)(6 + d);
               o.i0 = (int16_t)(b.in1 + ((m - b.lo1) * na + i) * nc1 + km);
               o.i1 = (int16_t)(b.in1 + ((m + 1 - b.lo1) * na + i) * nc1 + km);
               if (ec[d] >= 2) {
                  const int kw = lowered_idx(ec, d, 2), nc2 = ncart(c - 2);
                  o.f1 = (int8_t)(ec[d] - 1);
                  o.i2 = (int16_t)(b.in2 + ((m - b.lo2) * na + i) * nc2 + kw);
                  o.i3 = (int16_t)(b.in2 + ((m + 1 - b.lo2) * na + i) * nc2 + kw);
               }
               if (a > 0 && ea[d] >= 1) {
                  const int im = lowered_idx(ea, d, 1);
                  o.f2 = (int8_t)ea[d];
                  o.i4 = (int16_t)(b.in3 + ((m + 1 - b.lo3) * ncart(a - 1) + im) * nc1 + km);
               }
            }
            out.push_back(o);
         }
      }
      p.vop_lev[lv] = (int)out.size() - p.vop_off;
   }
   p.nvop = (int)out.size() - p.vop_off;
}

}  // namespace gint
