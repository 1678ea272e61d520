// TEST INFRASTRUCTURE ONLY. Thin extern "C" wrappers around host-callable functions of the
// reference libGint sources, compiled from the reference tree by oracle/Makefile into
// oracle/_ref/libref_host.so. The tests use them to pin the oracle's restatements:
//   plan()                 src/plan.cpp:217-642
//   create_md_ftable()     src/fgamma.cpp:109-123
//   fgamma0()              src/fgamma.cpp:196-243
//   fill_x12_to_patch()    src/t_c_g0_n.cpp:53-64
//   t_c_g0_n_v2()          src/t_c_g0_n.cpp:67-180
//   compute_pbc()          src/util.cpp:235-265
//   BW_by_patch[], c2s[]   src/BW_by_patch.h, src/c2s.h
#include <vector>
#include <cstdio>
#include <cstdlib>
#include "define.h"
#include "plan.h"
#include "fgamma.h"
#include "t_c_g0_n.h"
#include "util.h"
#include "BW_by_patch.h"
#include "c2s.h"

extern "C" {

int ref_plan(int la, int lb, int lc, int ld, int *out, int cap, int *info) {
   int pr, sh, nV, nVC, nVCH;
   std::vector<int> p = plan(la, lb, lc, ld, &pr, &sh, &nV, &nVC, &nVCH);
   info[0] = pr; info[1] = sh; info[2] = nV; info[3] = nVC; info[4] = nVCH;
   int n = (int)p.size();
   for (int i = 0; i < n && i < cap; i++) out[i] = p[i];
   return n;
}

void ref_ftable(double *out) {
   int ld = 0;
   double *t = create_md_ftable(21, 0., 12., 0.1, &ld);
   for (int i = 0; i < 121 * 28; i++) out[i] = t[i];
   free(t);
}

void ref_fgamma0(int nmax, double T, double *f, double fac) {
   static double *t = nullptr;
   int ld = 0;
   if (!t) t = create_md_ftable(21, 0., 12., 0.1, &ld);
   fgamma0(nmax, T, f, t, 28, fac);
}

void ref_lut(int *low, int *high) { fill_x12_to_patch(128, 128, low, high); }

void ref_bw(double *out) { for (int i = 0; i < 207 * 4; i++) out[i] = BW_by_patch[i]; }

void ref_c2s(double *out) { for (int i = 0; i < 245; i++) out[i] = c2s[i]; }

int ref_tcg(const double *C0, int ld_C0, double R, double T, int Nder, double Kfac, double *res) {
   static int *low = nullptr, *high = nullptr;
   static double *ft = nullptr;
   int ld = 0;
   if (!low) {
      low = (int *)malloc(128 * 128 * sizeof(int));
      high = (int *)malloc(128 * 128 * sizeof(int));
      fill_x12_to_patch(128, 128, low, high);
      ft = create_md_ftable(21, 0., 12., 0.1, &ld);
   }
   bool g = t_c_g0_n_v2(res, R, T, Nder, C0, ld_C0, 128, 128, low, high, BW_by_patch, 0, Kfac);
   if (g) fgamma0(Nder, T, res, ft, 28, Kfac);
   return g ? 1 : 0;
}

void ref_pbc(const double *A, const double *B, const double *cell, double *AB) {
   compute_pbc(A, B, cell, AB);
}

}  // extern "C"
