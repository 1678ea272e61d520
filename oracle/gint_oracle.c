/*
 * gint_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C, CPU restatement of libGint's exchange-matrix (K) build, used only by the tests,
 * by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker of the
 * CUDA engine in libgint_b200/. It is never linked into, loaded by, or called from the
 * product path.
 *
 * It exports the same C-ABI as the engine (include/libgint.h), so one recorded call
 * stream can be replayed into either library. Each stage cites the reference function
 * it restates (paths are relative to the libGint source tree):
 *
 *   normalisation of contraction coefficients  src/extern_functions.cpp:95-136
 *   add_prm / add_shell / add_qrt / add_qrtt  src/libGint.cpp:151-283
 *   primitive geometry and Kfac               src/compute_Fm.cpp:20-166 (prepare_Fm)
 *   minimum-image wrap                        src/util.cpp:132-162 (compute_pbc)
 *   truncated-Coulomb G_m(T,R)                src/t_c_g0_n.cpp:53-180 (fill_x12_to_patch,
 *                                             t_c_g0_n_v2)
 *   Boys function table and evaluation        src/fgamma.cpp:53-123 (fgamma_ref,
 *                                             create_md_ftable), :196-243 (fgamma0)
 *   per-image Fm and VRR factors              src/compute_Fm.cpp:168-326
 *   Obara-Saika VRR + screening               src/compute_VRR.cpp:111-458
 *   sum over the third image (SFT)            src/compute_ECO.cpp:216-272
 *   contraction over primitives (ECO)         src/compute_ECO.cpp:12-214
 *   HRR and the sum over image pairs          src/compute_HRR.cpp:7-225
 *   cartesian -> spherical (c2s, CP2K order)  src/compute_SPH.cpp:58-237, src/c2s.h:36-100
 *   exchange update of K                      src/compute_KS.cpp:6-117
 *
 * Quantities that decide screening (T, R, Kfac, the patch index) are evaluated with the
 * same formula and operation order as the reference, with one explicit fma where the
 * reference's CUDA build contracts (wdist below). The recursions themselves are written
 * directly from the Obara-Saika relations (no op-list interpreter); their results agree with
 * the reference's to rounding.
 */
#include <math.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../libgint_b200/csrc/tcg_patches.h"

#define OR_MAX_L 3          /* l <= 3 per centre (src/define.h:42-55, README.md:44-50) */
#define OR_MAX_LL 12        /* la+lb+lc+ld */
#define OR_MAX_CELL 256
#define OR_MAX_PRM 16
#define OR_MAX_NL 4
#define OR_TEPS 1.e-13
#define OR_SQRT2 1.4142135623730950488016887242096980785696718753

/* ------------------------------------------------------------------------------------ */
/* growable arrays                                                                       */
/* ------------------------------------------------------------------------------------ */
#define VEC(T) struct { T *d; size_t n, cap; }
#define VEC_PUSH(v, x) do { if ((v).n == (v).cap) { (v).cap = (v).cap ? 2*(v).cap : 64; \
   (v).d = realloc((v).d, (v).cap*sizeof(*(v).d)); } (v).d[(v).n++] = (x); } while (0)
#define VEC_FREE(v) do { free((v).d); (v).d = NULL; (v).n = (v).cap = 0; } while (0)

typedef struct {
   double R[3];
   int np;
   double Z[OR_MAX_PRM];
   int nL;
   int l[8], nl[8];
   double *K[8];            /* normalised, nl*np, row = contraction */
   int defined;
} or_set;

typedef struct {
   int set[4], lidx[4];
   int n1, n2;
   size_t prm_off;
   int nprm;
   int cls;                 /* la*64+lb*16+lc*4+ld */
} or_shell;

typedef struct {
   unsigned idx_fac;
   int inl[4];
   int ld[4];               /* ld_ac, ld_ad, ld_bc, ld_bd */
   unsigned off[4];         /* off_ac, off_ad, off_bc, off_bd */
   int T[4];                /* Tac, Tad, Tbc, Tbd */
   int cls;
} or_qrtt;

typedef struct {
   int cls, nl[4];
   size_t shell_off; int nshell;
   size_t qrtt_off;  int nqrtt;
} or_group;

typedef struct {
   /* basis */
   or_set *sets; int nsets;
   /* potential */
   double R_cut; double *C0; int ld_C0; int C0_size; int have_pot;
   int lut_low[128*128], lut_high[128*128];
   double hf_fac;
   /* cell */
   int periodic; double cell[18];
   double *neighs; int Ng;
   /* density / K */
   int nspin; size_t FP_size;
   double *P[2], *K[2];
   /* stream */
   VEC(uint32_t) prm_tmp;
   VEC(or_shell) set_shells;   VEC(uint32_t) set_prms;
   VEC(or_qrtt) set_qrtts;     VEC(or_group) set_groups;
   VEC(or_shell) shells;       VEC(uint32_t) prms;
   VEC(or_qrtt) qrtts;         VEC(or_group) groups;
   /* Boys table */
   double ftable[121*28];
   int nthreads;
   int error;
   /* optional screening-decision counters per class (the engine's libgint_get_counters layout):
      [cls*4 + 0] Chebyshev evaluations, 1 Boys evaluations, 2 images through the VRR
      (Fm[0] > 1e-12, classes other than (ss|ss)), 3 primitive quartets */
   int counting;
   unsigned long long cnt[256*4];
   /* magnitude mode: every factor of every product replaced by its absolute value (the Chebyshev
      coefficients and polynomials of G_m, the VRR factors, the contraction coefficients, AB/CD,
      c2s, -fac and P), so that K holds, per element, the sum of the magnitudes of the terms its
      FP64 evaluation adds up: the scale of the rounding error any evaluation order makes, against
      which two FP64 implementations are compared. (The geometric factors themselves, P, Q, W and
      their differences, are evaluated with the same rounded operations on both sides.) */
   int absmode;
} or_handle;

/* ------------------------------------------------------------------------------------ */
/* cartesian helpers                                                                     */
/* ------------------------------------------------------------------------------------ */
static int ncart(int l) { return (l+1)*(l+2)/2; }
static int nsph(int l) { return 2*l+1; }
/* order xx..: lx descending, then ly descending (src/util.cpp:270-330) */
static void cart_xyz(int l, int i, int e[3]) {
   int a = 0; while ((a+1)*(a+2)/2 <= i) a++;      /* a = l - lx */
   e[0] = l - a; e[2] = i - a*(a+1)/2; e[1] = a - e[2];
}
static int cart_idx(int lx, int ly, int lz) { int a = ly + lz; return a*(a+1)/2 + lz; }

/* ------------------------------------------------------------------------------------ */
/* Boys function table (restates src/fgamma.cpp:53-123 fgamma_ref / create_md_ftable)   */
/* ------------------------------------------------------------------------------------ */
static void or_fgamma_ref(int nmax, double T, double *f) {
   const int kmax = 50;
   double r[50+10];
   if (T < OR_TEPS) {
      for (int n = 0; n <= nmax; n++) f[n] = 1.0/(2.*n + 1.);
   } else if (T <= 50.0) {
      r[kmax+9] = 0.0;
      for (int j = kmax+9; j >= 1; j--) r[j-1] = -T/((4.*j + 2.) - T*r[j+1-1]);
      double factor = 2.0*sinh(0.5*T)*exp(-0.5*T)/T;
      for (int n = 0; n <= nmax; n++) {
         double sumtot = factor/(2.*n + 1.);
         double term = 1.0;
         for (int k = 1; k <= kmax; k++) {
            term = term*(2.*n - 2.*k + 1.)/(2.*n + 2.*k + 1);
            double p = 1.0;
            for (int j = 1; j <= k; j++) p = p*r[j-1];
            double sumterm = factor*term*p*(2.*k + 1.)/(2.*n + 1.);
            if (fabs(sumterm) < 2.220446049250313e-16) break;
            else if (k == kmax) { /* not converged: the reference asserts here */ }
            else sumtot = sumtot + sumterm;
         }
         f[n] = sumtot;
      }
   } else {
      f[0] = 0.5*sqrt(M_PI/T);
      double expt = exp(-T);
      for (int n = 1; n <= nmax; n++) f[n] = 0.5*((2.*n-1.)*f[n-1] - expt)/T;
   }
}

static void or_make_ftable(double *ft) {
   /* nmax=21, n=27, tmin=0, tmax=12, tdelta=0.1 -> 121 rows of 28 (src/libGint.cpp:488-497) */
   for (int itab = 0; itab <= 120; itab++) {
      double T = (double)itab*0.1;
      or_fgamma_ref(27, T, &ft[itab*28]);
   }
}

/* restates fgamma0 (src/fgamma.cpp:196-243); result scaled by fac */
static void or_fgamma0(int nmax, double T, double *f, const double *ftable, double fac) {
   if (T < OR_TEPS) {
      for (int n = 0; n <= nmax; n++) f[n] = fac/(2.*n+1.);
      return;
   }
   if (T < 12.) {
      const double tdelta = 0.1;
      const int ld = 28;
      int itab = (int)(round(T/tdelta));
      double ttab = (double)itab*tdelta;
      double tmp = 1.0, inv_fac;
      double fL = ftable[itab*ld+nmax+0];
      tmp *= (ttab-T); inv_fac = 1.0    ; fL += ftable[itab*ld+nmax+1]*tmp*inv_fac;
      tmp *= (ttab-T); inv_fac = 0.5    ; fL += ftable[itab*ld+nmax+2]*tmp*inv_fac;
      tmp *= (ttab-T); inv_fac = 1./6.  ; fL += ftable[itab*ld+nmax+3]*tmp*inv_fac;
      tmp *= (ttab-T); inv_fac = 1./24. ; fL += ftable[itab*ld+nmax+4]*tmp*inv_fac;
      tmp *= (ttab-T); inv_fac = 1./120.; fL += ftable[itab*ld+nmax+5]*tmp*inv_fac;
      tmp *= (ttab-T); inv_fac = 1./720.; fL += ftable[itab*ld+nmax+6]*tmp*inv_fac;
      double expt = exp(-T);
      f[nmax] = fL;
      for (int n = nmax-1; n >= 0; n--) f[n] = (2.0*T*f[n + 1] + expt)/(2.*n + 1.);
   } else {
      double tmp = 1.0/T;
      double tmp2 = tmp*tmp;
      double tmp3 = tmp*tmp2;
      double g = 0.4999489092 - 0.2473631686*tmp + 0.321180909*tmp2 - 0.3811559346*tmp3;
      double expt = exp(-T);
      f[0] = 0.5*sqrt(M_PI*tmp) - g*expt*tmp;
      for (int n = 1; n <= nmax; n++) f[n] = (0.5*tmp)*((2.*n - 1.)*f[n - 1] - expt);
   }
   for (int n = 0; n <= nmax; n++) f[n] *= fac;
}

/* ------------------------------------------------------------------------------------ */
/* truncated Coulomb (restates src/t_c_g0_n.cpp:53-180)                                 */
/* ------------------------------------------------------------------------------------ */
static int or_locate(double X1, double X2, int first, int last) {
   for (int p = first; p < last; p++) {
      double lo1 = tcg_patch_rect[p][0]/128.0, hi1 = tcg_patch_rect[p][1]/128.0;
      double lo2 = tcg_patch_rect[p][2]/128.0, hi2 = tcg_patch_rect[p][3]/128.0;
      int in1 = (X1 <= hi1) && (X1 > lo1 || (lo1 == 0.0 && X1 >= 0.0));
      int in2 = (X2 <= hi2) && (X2 > lo2 || (lo2 == 0.0 && X2 >= 0.0));
      if (in1 && in2) return p;
   }
   return -1;
}

static void or_fill_lut(or_handle *h) {
   /* src/t_c_g0_n.cpp:53-64: the grid point i maps to X = i/(N-1) */
   for (int i1 = 0; i1 < 128; i1++) {
      double X1 = ((double)i1)/(double)(128-1.0);
      for (int i2 = 0; i2 < 128; i2++) {
         double X2 = ((double)i2)/(double)(128-1.0);
         h->lut_low[i1*128+i2]  = or_locate(X1, X2, 0, TCG_NPATCH_LOW);
         h->lut_high[i1*128+i2] = or_locate(X1, X2, TCG_NPATCH_LOW, TCG_NPATCH);
      }
   }
}

/* returns 1 if the Boys function must be used instead (then res is zeroed), 2 when the Chebyshev
   series was evaluated, 0 beyond the truncation (res zeroed) */
static int or_tcg(const or_handle *h, double *res, double R, double T, int Nder, double Kfac) {
   double upper = R*R + 11.0*R + 50.0;
   double lower = R*R - 11.0*R + 0.0;
   double X1, X2;
   int patch;
   const int N1 = 128, N2 = 128;
   if (T > upper) {
      for (int n = 0; n <= Nder; n++) res[n] = 0.0;
      return 0;
   }
   if (R <= 11.0) {
      X2 = R/11.0;
      upper = R*R + 11.0*R + 50.0;
      lower = 0.0;
      X1 = (T - lower)/(upper - lower);
      int i1 = (int)(X1 * N1), i2 = (int)(X2 * N2);
      if (i1 == N1) i1 = N1-1;
      if (i2 == N2) i2 = N2-1;
      patch = h->lut_low[i1*N2+i2];
   } else {
      if (T < lower) {
         for (int n = 0; n <= Nder; n++) res[n] = 0.0;
         return 1;
      }
      X2 = 11.0/R;
      X1 = (T-lower)/(upper-lower);
      int i1 = (int)(X1 * N1), i2 = (int)(X2 * N2);
      if (i1 == N1) i1 = N1-1;
      if (i2 == N2) i2 = N2-1;
      patch = h->lut_high[i1*N2+i2];
   }
   const double B1 = (tcg_patch_rect[patch][0] + tcg_patch_rect[patch][1]) / 128.0;
   const double W1 = 128.0 / (tcg_patch_rect[patch][1] - tcg_patch_rect[patch][0]);
   const double B2 = (tcg_patch_rect[patch][2] + tcg_patch_rect[patch][3]) / 128.0;
   const double W2 = 128.0 / (tcg_patch_rect[patch][3] - tcg_patch_rect[patch][2]);
   const double *C0_row = &h->C0[(size_t)h->ld_C0*patch];
   double TG1 = (2.*X1-B1)*W1;
   double TG2 = (2.*X2-B2)*W2;
   double T1[14], T2[14];
   T1[0] = 1.0; T2[0] = 1.0;
   T1[1] = OR_SQRT2*TG1; T2[1] = OR_SQRT2*TG2;
   T1[2] = 2.*TG1*T1[1] - OR_SQRT2; T2[2] = 2.*TG2*T2[1] - OR_SQRT2;
   for (int i = 3; i < 14; i++) {
      T1[i] = 2.*TG1*T1[i-1] - T1[i-2];
      T2[i] = 2.*TG2*T2[i-1] - T2[i-2];
   }
   if (h->absmode) {
      /* magnitude of the series: the scale of its rounding error, not of its value */
      for (int i = 0; i < 14; i++) { T1[i] = fabs(T1[i]); T2[i] = fabs(T2[i]); }
   }
   for (int k = 0; k <= Nder; k++) {
      double tmp = 0.0;
      int jl = 0;
      for (int j = 0; j < 14; j++) {
         double dot = 0.0;
         for (int l = 0; l < 14-j; l++) {
            const double cf = h->absmode ? fabs(C0_row[k*105+jl]) : C0_row[k*105+jl];
            dot += T1[l] * cf; jl++;
         }
         tmp += dot * T2[j];
      }
      res[k] = tmp*Kfac;
   }
   return 2;
}

/* ------------------------------------------------------------------------------------ */
/* periodic wrap (restates src/util.cpp:132-162)                                        */
/* ------------------------------------------------------------------------------------ */
static void or_pbc(const double A[3], const double B[3], const double *cell, double *AB) {
   const double *hm = &cell[0], *hi = &cell[9];
   AB[0] = B[0]-A[0]; AB[1] = B[1]-A[1]; AB[2] = B[2]-A[2];
   double s0 = hi[0*3+0]*AB[0] + hi[1*3+0]*AB[1] + hi[2*3+0]*AB[2];
   double s1 = hi[0*3+1]*AB[0] + hi[1*3+1]*AB[1] + hi[2*3+1]*AB[2];
   double s2 = hi[0*3+2]*AB[0] + hi[1*3+2]*AB[1] + hi[2*3+2]*AB[2];
   s0 -= round(s0); s1 -= round(s1); s2 -= round(s2);
   AB[0] = hm[0*3+0]*s0 + hm[1*3+0]*s1 + hm[2*3+0]*s2;
   AB[1] = hm[0*3+1]*s0 + hm[1*3+1]*s1 + hm[2*3+1]*s2;
   AB[2] = hm[0*3+2]*s0 + hm[1*3+2]*s1 + hm[2*3+2]*s2;
}

/* weighted distance (c1 X1 + c2 X2) c12 (src/util.h:62-68). The reference's CUDA build
 * contracts the first product into the sum, fma(c1, X1, c2 X2) c12, and that rounding decides
 * the minimum image of P - Q when it lies on half a lattice vector (symmetric quartets such as
 * (ab|ab') with b' an image of b and equal exponents), so the oracle states the fma. */
static void wdist(double X[3], const double X1[3], const double X2[3], double c1, double c2,
                  double c12) {
   X[0] = fma(c1, X1[0], c2*X2[0]) * c12;
   X[1] = fma(c1, X1[1], c2*X2[1]) * c12;
   X[2] = fma(c1, X1[2], c2*X2[2]) * c12;
}

/* ------------------------------------------------------------------------------------ */
/* cartesian -> spherical coefficients in CP2K's convention (values of src/c2s.h)       */
/* ------------------------------------------------------------------------------------ */
/* unnormalised real solid harmonics, rows m=-l..l, as integer coefficients on the
 * cartesian monomials in the order above. */
static const int or_sh_l1[3][3] = { {0,1,0}, {0,0,1}, {1,0,0} };
static const int or_sh_l2[5][6] = {
   {0,1,0,0,0,0}, {0,0,0,0,1,0}, {-1,0,0,-1,0,2}, {0,0,1,0,0,0}, {1,0,0,-1,0,0} };
static const int or_sh_l3[7][10] = {
   {0,3,0,0,0,0,-1,0,0,0},     /* 3x^2y - y^3        */
   {0,0,0,0,1,0,0,0,0,0},      /* xyz                */
   {0,-1,0,0,0,0,-1,0,4,0},    /* y(4z^2-x^2-y^2)    */
   {0,0,-3,0,0,0,0,-3,0,2},    /* z(2z^2-3x^2-3y^2)  */
   {-1,0,0,-1,0,4,0,0,0,0},    /* x(4z^2-x^2-y^2)    */
   {0,0,1,0,0,0,0,-1,0,0},     /* z(x^2-y^2)         */
   {1,0,0,-3,0,0,0,0,0,0} };   /* x^3-3xy^2          */

static double dfact(int n) { double r = 1.0; for (int k = n; k > 1; k -= 2) r *= k; return r; }

/* <x^a1 y^b1 z^c1 | x^a2 y^b2 z^c2> up to a common factor */
static double mono_ovl(const int e1[3], const int e2[3]) {
   double r = 1.0;
   for (int d = 0; d < 3; d++) {
      int s = e1[d] + e2[d];
      if (s & 1) return 0.0;
      r *= dfact(s-1);
   }
   return r;
}

static double or_c2s[4][7][10];

static void or_make_c2s(void) {
   memset(or_c2s, 0, sizeof(or_c2s));
   or_c2s[0][0][0] = 1.0;
   for (int l = 1; l <= 3; l++) {
      int nc = ncart(l), ns = nsph(l);
      for (int m = 0; m < ns; m++) {
         const int *row = (l == 1) ? or_sh_l1[m] : (l == 2) ? or_sh_l2[m] : or_sh_l3[m];
         double n2 = 0.0;
         for (int i = 0; i < nc; i++) for (int j = 0; j < nc; j++) {
            if (!row[i] || !row[j]) continue;
            int e1[3], e2[3]; cart_xyz(l, i, e1); cart_xyz(l, j, e2);
            n2 += row[i]*row[j]*mono_ovl(e1, e2);
         }
         double nrm = sqrt(n2);
         for (int i = 0; i < nc; i++) {
            double v = row[i]/nrm;
            if (l >= 3) v = round(v*1e9)/1e9;   /* 9-decimal literals of the CP2K table */
            or_c2s[l][m][i] = v;
         }
      }
   }
}

/* ------------------------------------------------------------------------------------ */
/* integral of one class for one (set quartet, l-combination) group                     */
/* ------------------------------------------------------------------------------------ */
typedef struct {
   int la, lb, lc, ld, L;
   int LAB, LCD;
   /* VRR block table: (a,c) block offset and size, m in [0, L-a-c] */
   int voff[7][7];
   int vsize;
   /* CP2S targets: (e,f) for e in [la,la+lb], f in [lc,lc+ld] (m=0) */
   int toff[7][7];
   int tsize;
} or_cls;

static void or_cls_init(or_cls *c, int la, int lb, int lc, int ld) {
   c->la = la; c->lb = lb; c->lc = lc; c->ld = ld;
   c->LAB = la+lb; c->LCD = lc+ld; c->L = c->LAB + c->LCD;
   int off = 0;
   for (int a = 0; a <= c->LAB; a++) for (int cc = 0; cc <= c->LCD; cc++) {
      c->voff[a][cc] = off;
      off += ncart(a)*ncart(cc)*(c->L - a - cc + 1);
   }
   c->vsize = off;
   off = 0;
   for (int e = la; e <= c->LAB; e++) for (int f = lc; f <= c->LCD; f++) {
      c->toff[e][f] = off;
      off += ncart(e)*ncart(f);
   }
   c->tsize = off;
}

/* VRR (a|c)^(m) (restates the recurrences of src/compute_VRR.cpp:111-345) */
static void or_vrr(const or_cls *c, double *V, const double *Fm, const double pqz[17]) {
   const double *PA = pqz+0, *WP = pqz+3, *QC = pqz+6, *WQ = pqz+9;
   const double i2ab = pqz[12], mrab = pqz[13], i2cd = pqz[14], mrcd = pqz[15], i2z = pqz[16];
   const int L = c->L;
   for (int m = 0; m <= L; m++) V[c->voff[0][0] + m] = Fm[m];
   for (int a = 0; a <= c->LAB; a++) {
      for (int cc = 0; cc <= c->LCD; cc++) {
         if (a == 0 && cc == 0) continue;
         int na = ncart(a), nc = ncart(cc), nm = L - a - cc + 1;
         double *out = V + c->voff[a][cc];
         for (int m = 0; m < nm; m++) for (int i = 0; i < na; i++) for (int k = 0; k < nc; k++) {
            int ea[3], ec[3]; cart_xyz(a, i, ea); cart_xyz(cc, k, ec);
            double v;
            if (cc == 0) {
               int d = ea[0] ? 0 : (ea[1] ? 1 : 2);
               int em[3] = {ea[0], ea[1], ea[2]}; em[d]--;
               int im = cart_idx(em[0], em[1], em[2]);
               const double *b1 = V + c->voff[a-1][0];
               int n1 = ncart(a-1);
               v = PA[d]*b1[m*n1+im] + WP[d]*b1[(m+1)*n1+im];
               if (ea[d] >= 2) {
                  int ew[3] = {em[0], em[1], em[2]}; ew[d]--;
                  int iw = cart_idx(ew[0], ew[1], ew[2]);
                  const double *b2 = V + c->voff[a-2][0];
                  int n2 = ncart(a-2);
                  v += (ea[d]-1)*(i2ab*b2[m*n2+iw] + mrab*b2[(m+1)*n2+iw]);
               }
            } else {
               int d = ec[0] ? 0 : (ec[1] ? 1 : 2);
               int cm[3] = {ec[0], ec[1], ec[2]}; cm[d]--;
               int km = cart_idx(cm[0], cm[1], cm[2]);
               const double *b1 = V + c->voff[a][cc-1];
               int n1 = na*ncart(cc-1);
               int ncm = ncart(cc-1);
               v = QC[d]*b1[m*n1 + i*ncm + km] + WQ[d]*b1[(m+1)*n1 + i*ncm + km];
               if (ec[d] >= 2) {
                  int cw[3] = {cm[0], cm[1], cm[2]}; cw[d]--;
                  int kw = cart_idx(cw[0], cw[1], cw[2]);
                  const double *b2 = V + c->voff[a][cc-2];
                  int ncw = ncart(cc-2);
                  int n2 = na*ncw;
                  v += (ec[d]-1)*(i2cd*b2[m*n2 + i*ncw + kw] + mrcd*b2[(m+1)*n2 + i*ncw + kw]);
               }
               if (a > 0 && ea[d] >= 1) {
                  int em[3] = {ea[0], ea[1], ea[2]}; em[d]--;
                  int im = cart_idx(em[0], em[1], em[2]);
                  const double *b3 = V + c->voff[a-1][cc-1];
                  int n3 = ncart(a-1)*ncm;
                  v += ea[d]*i2z*b3[(m+1)*n3 + im*ncm + km];
               }
            }
            out[m*na*nc + i*nc + k] = v;
         }
      }
   }
}

/* HRR on one contracted block (restates src/compute_HRR.cpp:7-99; ket first, then bra).
 * in: targets (e0|f0) at c->toff; out: cart[(ia*nb+ib)*nc*nd + ic*nd + id] */
static void or_hrr(const or_cls *c, const double *tin, const double AB[3], const double CD[3],
                   double *out, double *ws) {
   const int la = c->la, lb = c->lb, lc = c->lc, ld = c->ld;
   /* ket: for each e, X_e[c][d] blocks; store (e0|LC LD) in Y[ie][cd] */
   int nE = 0; for (int e = la; e <= c->LAB; e++) nE += ncart(e);
   int ncd = ncart(lc)*ncart(ld);
   double *Y = ws; ws += nE*ncd;
   int ie0 = 0;
   for (int e = la; e <= c->LAB; e++) {
      int ne = ncart(e);
      /* level buffers: lev[cc] holds (e0|cc, d) for current d, size ne*ncart(cc)*ncart(d) */
      double *lev[7], *nxt[7];
      int cap = 0;
      for (int cc = lc; cc <= c->LCD; cc++) cap += ne*ncart(cc)*ncart(ld);
      double *bufA = ws, *bufB = ws + cap;
      int o = 0;
      for (int cc = lc; cc <= c->LCD; cc++) {
         lev[cc] = bufA + o; o += ne*ncart(cc);
         const double *src = tin + c->toff[e][cc];
         memcpy(lev[cc], src, sizeof(double)*ne*ncart(cc));
      }
      for (int d = 1; d <= ld; d++) {
         o = 0;
         double *dst = (d & 1) ? bufB : bufA;
         int nd = ncart(d), ndm = ncart(d-1);
         for (int cc = lc; cc <= c->LCD - d; cc++) {
            nxt[cc] = dst + o; o += ne*ncart(cc)*nd;
            int nc = ncart(cc), ncp = ncart(cc+1);
            for (int i = 0; i < ne; i++) for (int k = 0; k < nc; k++) for (int l = 0; l < nd; l++) {
               int ed[3], ecc[3]; cart_xyz(d, l, ed); cart_xyz(cc, k, ecc);
               int dir = ed[0] ? 0 : (ed[1] ? 1 : 2);
               int dm[3] = {ed[0], ed[1], ed[2]}; dm[dir]--;
               int cp[3] = {ecc[0], ecc[1], ecc[2]}; cp[dir]++;
               int lm = cart_idx(dm[0], dm[1], dm[2]), kp = cart_idx(cp[0], cp[1], cp[2]);
               nxt[cc][(i*nc+k)*nd+l] = lev[cc+1][(i*ncp+kp)*ndm+lm] + CD[dir]*lev[cc][(i*nc+k)*ndm+lm];
            }
         }
         for (int cc = lc; cc <= c->LCD - d; cc++) lev[cc] = nxt[cc];
      }
      memcpy(Y + ie0*ncd, lev[lc], sizeof(double)*ne*ncd);
      ie0 += ne;
   }
   /* bra: (a,b|) from Y */
   double *bl[7], *bn[7];
   int capb = 0;
   for (int a = la; a <= c->LAB; a++) capb += ncart(a)*ncart(lb)*ncd;
   double *bA = ws, *bB = ws + capb;
   ie0 = 0;
   for (int a = la; a <= c->LAB; a++) { bl[a] = Y + ie0*ncd; ie0 += ncart(a); }
   for (int b = 1; b <= lb; b++) {
      double *dst = (b & 1) ? bA : bB;
      int o = 0, nb = ncart(b), nbm = ncart(b-1);
      for (int a = la; a <= c->LAB - b; a++) {
         bn[a] = dst + o; o += ncart(a)*nb*ncd;
         int na = ncart(a), nap = ncart(a+1);
         for (int i = 0; i < na; i++) for (int j = 0; j < nb; j++) for (int q = 0; q < ncd; q++) {
            int eb[3], ea[3]; cart_xyz(b, j, eb); cart_xyz(a, i, ea);
            int dir = eb[0] ? 0 : (eb[1] ? 1 : 2);
            int bm[3] = {eb[0], eb[1], eb[2]}; bm[dir]--;
            int ap[3] = {ea[0], ea[1], ea[2]}; ap[dir]++;
            int jm = cart_idx(bm[0], bm[1], bm[2]), ip = cart_idx(ap[0], ap[1], ap[2]);
            bn[a][(i*nb+j)*ncd+q] = bl[a+1][(ip*nbm+jm)*ncd+q] + AB[dir]*bl[a][(i*nbm+jm)*ncd+q];
         }
      }
      for (int a = la; a <= c->LAB - b; a++) bl[a] = bn[a];
   }
   memcpy(out, bl[la], sizeof(double)*ncart(la)*ncart(lb)*ncd);
}

/* cart -> spherical, one centre at a time: a, then b, c, d (src/compute_SPH.cpp:127-234) */
static void or_sph(int la, int lb, int lc, int ld, const double *cart, double *sph, double *ws, int absmode) {
   int n[4] = {ncart(la), ncart(lb), ncart(lc), ncart(ld)};
   int s[4] = {nsph(la), nsph(lb), nsph(lc), nsph(ld)};
   int l[4] = {la, lb, lc, ld};
   /* current tensor dims: dims[0..3], one of which has been converted */
   int dims[4] = {n[0], n[1], n[2], n[3]};
   const double *src = cart;
   double *bufs[2] = { ws, ws + 10000 };
   for (int ctr = 0; ctr < 4; ctr++) {
      double *dst = (ctr == 3) ? sph : bufs[ctr & 1];
      int od[4] = {dims[0], dims[1], dims[2], dims[3]}; od[ctr] = s[ctr];
      int tot = od[0]*od[1]*od[2]*od[3];
      for (int t = 0; t < tot; t++) {
         int id[4], r = t;
         for (int q = 3; q >= 0; q--) { id[q] = r % od[q]; r /= od[q]; }
         double acc = 0.0;
         for (int k = 0; k < n[ctr]; k++) {
            int jd[4] = {id[0], id[1], id[2], id[3]}; jd[ctr] = k;
            int si = ((jd[0]*dims[1] + jd[1])*dims[2] + jd[2])*dims[3] + jd[3];
            const double cf = or_c2s[l[ctr]][id[ctr]][k];
            acc += (absmode ? fabs(cf) : cf) * src[si];
         }
         dst[t] = acc;
      }
      dims[ctr] = s[ctr];
      src = dst;
   }
}

static const double or_symm_factors[5] = {2.0, 1.0, 0.5, 0.25, 0.0};

/* ------------------------------------------------------------------------------------ */
/* one group: all image pairs of one set quartet for one l-combination                  */
/* ------------------------------------------------------------------------------------ */
static void or_group_compute(or_handle *h, const or_group *g, double *Kout[2], double *scratch,
                             unsigned long long *cnt) {
   const int la = g->cls >> 6, lb = (g->cls >> 4) & 3, lc = (g->cls >> 2) & 3, ld = g->cls & 3;
   or_cls c; or_cls_init(&c, la, lb, lc, ld);
   const int L = c.L;
   const int nlabcd = g->nl[0]*g->nl[1]*g->nl[2]*g->nl[3];
   const int Nc = ncart(la)*ncart(lb)*ncart(lc)*ncart(ld);
   const int Ns = nsph(la)*nsph(lb)*nsph(lc)*nsph(ld);
   const int want00 = (la == 0 && lc == 0);

   double *V = scratch;                      /* c.vsize */
   double *ssum = V + c.vsize;               /* c.tsize */
   double *contr = ssum + c.tsize;           /* nlabcd * tsize */
   double *abcd0 = contr + (size_t)nlabcd*c.tsize;  /* nlabcd * Nc */
   double *cart = abcd0 + (size_t)nlabcd*Nc;       /* Nc */
   double *ws = cart + 10000;                      /* HRR/SPH workspace */
   memset(abcd0, 0, sizeof(double)*(size_t)nlabcd*Nc);

   double Fm[OR_MAX_LL+1];
   for (int is = 0; is < g->nshell; is++) {
      const or_shell *sh = &h->shells.d[g->shell_off + is];
      const or_set *sa = &h->sets[sh->set[0]], *sb = &h->sets[sh->set[1]];
      const or_set *sc = &h->sets[sh->set[2]], *sd = &h->sets[sh->set[3]];
      const double *Ka = sa->K[sh->lidx[0]], *Kb = sb->K[sh->lidx[1]];
      const double *Kc = sc->K[sh->lidx[2]], *Kd = sd->K[sh->lidx[3]];
      const int n1 = sh->n1, n2 = sh->n2;
      memset(contr, 0, sizeof(double)*(size_t)nlabcd*c.tsize);

      /* shell geometry (src/compute_Fm.cpp:79-95, src/compute_HRR.cpp:142-166) */
      double A[3], B[3], C[3], D[3], ABs[3], CDs[3];
      or_pbc(sa->R, sb->R, h->cell, ABs);
      for (int q = 0; q < 3; q++) { A[q] = sa->R[q]; B[q] = sa->R[q] + ABs[q] + h->neighs[n1*3+q]; }
      or_pbc(sc->R, sd->R, h->cell, CDs);
      for (int q = 0; q < 3; q++) { C[q] = sc->R[q]; D[q] = sc->R[q] + CDs[q] + h->neighs[n2*3+q]; }

      cnt[g->cls*4 + 3] += (unsigned long long)sh->nprm;
      for (int ip = 0; ip < sh->nprm; ip++) {
         uint32_t code = h->prms.d[sh->prm_off + ip];
         int ipa = code >> 24, ipb = (code >> 16) & 255, ipc = (code >> 8) & 255, ipd = code & 255;
         const double za = sa->Z[ipa], zb = sb->Z[ipb], zc = sc->Z[ipc], zd = sd->Z[ipd];
         /* prepare_Fm (src/compute_Fm.cpp:66-159) */
         const double zab = za+zb, inv_zab = 1./zab, zcd = zc+zd, inv_zcd = 1./zcd;
         const double z = zab + zcd, inv_z = 1./z;
         double P[3], Q[3], PQs[3], shift[3], Cs[3], Ds[3];
         wdist(P, A, B, za, zb, inv_zab);
         wdist(Q, C, D, zc, zd, inv_zcd);
         or_pbc(Q, P, h->cell, PQs);
         for (int q = 0; q < 3; q++) shift[q] = P[q] - Q[q] - PQs[q];
         double normf = 2. * pow(M_PI, 5./2.) * inv_zab * inv_zcd;
         double dx = A[0]-B[0], dy = A[1]-B[1], dz = A[2]-B[2];
         double RAB2 = dx*dx + dy*dy + dz*dz;
         double expon_ab = - (za*zb)/(za+zb) * RAB2;
         dx = C[0]-D[0]; dy = C[1]-D[1]; dz = C[2]-D[2];
         double RCD2 = dx*dx + dy*dy + dz*dz;
         double expon_cd = - (zc*zd)/(zc+zd) * RCD2;
         double Zn = 1./sqrt(z);
         double Kfactor = Zn * normf * exp(expon_ab+expon_cd);
         for (int q = 0; q < 3; q++) {
            Cs[q] = C[q] + shift[q];
            Ds[q] = C[q] + CDs[q] + h->neighs[n2*3+q] + shift[q];
         }
         wdist(Q, Cs, Ds, zc, zd, inv_zcd);
         double PA[3] = {P[0]-A[0], P[1]-A[1], P[2]-A[2]};
         double QC[3] = {Q[0]-Cs[0], Q[1]-Cs[1], Q[2]-Cs[2]};
         /* compute_Fm / compute_Vm constants (src/compute_Fm.cpp:202-210, 281-290) */
         const double Kfac = Kfactor, invz = inv_z;
         const double zcd2 = zc + zd;
         const double rho = zab * zcd2 * invz;
         const double R = h->R_cut * sqrt(rho);
         const double izab = 1. / zab, i2ab = 0.5 * izab, mrab = -1. * rho * izab * i2ab;
         const double izcd = 1. / zcd2, i2cd = 0.5 * izcd, mrcd = -1. * rho * izcd * i2cd;
         const double i2z = 0.5 * invz;

         memset(ssum, 0, sizeof(double)*c.tsize);
         for (int n3 = 0; n3 < h->Ng; n3++) {
            const double *g3 = &h->neighs[n3*3];
            double PQ[3] = {P[0]-Q[0]-g3[0], P[1]-Q[1]-g3[1], P[2]-Q[2]-g3[2]};
            double rpq2 = (PQ[0]*PQ[0] + PQ[1]*PQ[1] + PQ[2]*PQ[2]);
            double T = rho * rpq2;
            const int branch = or_tcg(h, Fm, R, T, L, Kfac);
            if (branch == 1) or_fgamma0(L, T, Fm, h->ftable, Kfac);
            cnt[g->cls*4 + 0] += (branch == 2);
            cnt[g->cls*4 + 1] += (branch == 1);
            const int survives = Fm[0] > 1.e-12;
            if (h->absmode) for (int m = 0; m <= L; m++) Fm[m] = fabs(Fm[m]);
            /* the (00|00) value enters the s-type target unscreened
               (src/compute_VRR.cpp:381-389 writes Fm[0] for every visited primitive) */
            if (want00) ssum[c.toff[0][0]] += Fm[0];
            if (!survives) continue;                  /* Fm[0] > 1e-12, src/compute_VRR.cpp:387 */
            cnt[g->cls*4 + 2] += (g->cls != 0);
            double Qp[3] = {Q[0]+g3[0], Q[1]+g3[1], Q[2]+g3[2]};
            double W[3]; wdist(W, P, Qp, zab, zcd2, invz);
            double pqz[17] = { PA[0], PA[1], PA[2], W[0]-P[0], W[1]-P[1], W[2]-P[2],
                               QC[0], QC[1], QC[2], W[0]-Qp[0], W[1]-Qp[1], W[2]-Qp[2],
                               i2ab, mrab, i2cd, mrcd, i2z };
            if (h->absmode) for (int q = 0; q < 17; q++) pqz[q] = fabs(pqz[q]);
            or_vrr(&c, V, Fm, pqz);
            for (int e = la; e <= c.LAB; e++) for (int f = lc; f <= c.LCD; f++) {
               if (e == 0 && f == 0) continue;      /* added above, unscreened */
               const double *blk = V + c.voff[e][f];  /* m = 0 slice */
               double *dst = ssum + c.toff[e][f];
               int nn = ncart(e)*ncart(f);
               for (int q = 0; q < nn; q++) dst[q] += blk[q];
            }
         }
         /* contraction (src/compute_ECO.cpp:131-212) */
         for (int l = 0; l < nlabcd; l++) {
            int a = l / (g->nl[1]*g->nl[2]*g->nl[3]);
            int b = (l / (g->nl[2]*g->nl[3])) % g->nl[1];
            int cc = (l / g->nl[3]) % g->nl[2];
            int d = l % g->nl[3];
            double Kp = Ka[a*sa->np + ipa] * Kb[b*sb->np + ipb] * Kc[cc*sc->np + ipc] * Kd[d*sd->np + ipd];
            if (h->absmode) Kp = fabs(Kp);
            double *dst = contr + (size_t)l*c.tsize;
            for (int q = 0; q < c.tsize; q++) dst[q] += Kp*ssum[q];
         }
      }
      /* HRR per contracted block + sum over (n1,n2) (src/compute_HRR.cpp:190-223) */
      double ABv[3] = {A[0]-B[0], A[1]-B[1], A[2]-B[2]};
      double CDv[3] = {C[0]-D[0], C[1]-D[1], C[2]-D[2]};
      if (h->absmode) for (int q = 0; q < 3; q++) { ABv[q] = fabs(ABv[q]); CDv[q] = fabs(CDv[q]); }
      for (int l = 0; l < nlabcd; l++) {
         or_hrr(&c, contr + (size_t)l*c.tsize, ABv, CDv, cart, ws);
         double *dst = abcd0 + (size_t)l*Nc;
         for (int q = 0; q < Nc; q++) dst[q] += cart[q];
      }
   }

   /* SPH + KS per contraction row (src/compute_KS.cpp:26-115) */
   const int nsa = nsph(la), nsb = nsph(lb), nsc = nsph(lc), nsd = nsph(ld);
   const int nscd = nsc*nsd, nsbcd = nsb*nscd;
   double *sph = cart;
   for (int r = 0; r < g->nqrtt && r < nlabcd; r++) {
      const or_qrtt *k = &h->qrtts.d[g->qrtt_off + r];
      or_sph(la, lb, lc, ld, abcd0 + (size_t)r*Nc, sph, ws, h->absmode);
      const double fac = or_symm_factors[k->idx_fac] * h->hf_fac;
      for (int t = 0; t < Ns; t++) {
         const int isa = t / nsbcd, isb = (t / nscd) % nsb, isc = (t / nsd) % nsc, isd = t % nsd;
         const int iac = !k->T[0] ? isc*k->ld[0] + isa : isa*k->ld[0] + isc;
         const int iad = !k->T[1] ? isd*k->ld[1] + isa : isa*k->ld[1] + isd;
         const int ibc = !k->T[2] ? isc*k->ld[2] + isb : isb*k->ld[2] + isc;
         const int ibd = !k->T[3] ? isd*k->ld[3] + isb : isb*k->ld[3] + isd;
         const size_t Iac = k->off[0] + (size_t)iac, Iad = k->off[1] + (size_t)iad;
         const size_t Ibc = k->off[2] + (size_t)ibc, Ibd = k->off[3] + (size_t)ibd;
         if (Iac >= h->FP_size || Iad >= h->FP_size || Ibc >= h->FP_size || Ibd >= h->FP_size) {
            h->error = 3; continue;
         }
         const double iabcd = h->absmode ? fabs(fac * sph[t]) : - fac * sph[t];
         for (int s = 0; s < h->nspin; s++) {
            const double *Pm = h->P[s];
            double *Km = Kout[s];
            if (h->absmode) {
               Km[Ibd] += iabcd * fabs(Pm[Iac]);
               Km[Ibc] += iabcd * fabs(Pm[Iad]);
               Km[Iad] += iabcd * fabs(Pm[Ibc]);
               Km[Iac] += iabcd * fabs(Pm[Ibd]);
               continue;
            }
            Km[Ibd] += iabcd * Pm[Iac];
            Km[Ibc] += iabcd * Pm[Iad];
            Km[Iad] += iabcd * Pm[Ibc];
            Km[Iac] += iabcd * Pm[Ibd];
         }
      }
   }
}

static size_t or_scratch_size(int cls, const int nl[4]) {
   const int la = cls >> 6, lb = (cls >> 4) & 3, lc = (cls >> 2) & 3, ld = cls & 3;
   or_cls c; or_cls_init(&c, la, lb, lc, ld);
   size_t nlabcd = (size_t)nl[0]*nl[1]*nl[2]*nl[3];
   size_t Nc = (size_t)ncart(la)*ncart(lb)*ncart(lc)*ncart(ld);
   return c.vsize + c.tsize + nlabcd*c.tsize + nlabcd*Nc + 10000 + 200000;
}

static void or_compute_all(or_handle *h) {
   if (h->groups.n == 0 || h->nspin == 0) return;
   int nth = h->nthreads > 0 ? h->nthreads : 1;
#ifdef _OPENMP
   if (h->nthreads <= 0) nth = omp_get_max_threads();
#else
   nth = 1;
#endif
   size_t maxs = 0;
   for (size_t ig = 0; ig < h->groups.n; ig++) {
      size_t s = or_scratch_size(h->groups.d[ig].cls, h->groups.d[ig].nl);
      if (s > maxs) maxs = s;
   }
   double **Kp = calloc((size_t)nth*2, sizeof(double*));
   #pragma omp parallel num_threads(nth)
   {
      int tid = 0;
#ifdef _OPENMP
      tid = omp_get_thread_num();
#endif
      double *scr = malloc(sizeof(double)*maxs);
      unsigned long long *tcnt = calloc(256*4, sizeof(unsigned long long));
      double *Kloc[2] = {NULL, NULL};
      for (int s = 0; s < h->nspin; s++) {
         Kloc[s] = (tid == 0) ? h->K[s] : calloc(h->FP_size, sizeof(double));
         Kp[tid*2+s] = Kloc[s];
      }
      #pragma omp for schedule(dynamic, 4)
      for (long ig = 0; ig < (long)h->groups.n; ig++) or_group_compute(h, &h->groups.d[ig], Kloc, scr, tcnt);
      free(scr);
      if (h->counting) {
         #pragma omp critical
         for (int q = 0; q < 256*4; q++) h->cnt[q] += tcnt[q];
      }
      free(tcnt);
   }
   for (int t = 1; t < nth; t++) for (int s = 0; s < h->nspin; s++) {
      double *src = Kp[t*2+s];
      for (size_t q = 0; q < h->FP_size; q++) h->K[s][q] += src[q];
      free(src);
   }
   free(Kp);
   h->shells.n = 0; h->prms.n = 0; h->qrtts.n = 0; h->groups.n = 0;
}

/* ------------------------------------------------------------------------------------ */
/* C-ABI (same entry points as src/extern_functions.cpp:9-190)                          */
/* ------------------------------------------------------------------------------------ */
void *libgint_create_handle(void) {
   or_handle *h = calloc(1, sizeof(or_handle));
   or_make_ftable(h->ftable);
   or_make_c2s();
   h->Ng = 1; h->neighs = calloc(3, sizeof(double));
   for (int i = 0; i < 3; i++) { h->cell[i*3+i] = 1.e6; h->cell[9+i*3+i] = 1.e-6; }
   h->hf_fac = 1.0;
   return h;
}
void libgint_init(void *hh) { (void)hh; }
void libgint_set_Potential_Truncated(void *hh, double R_cut, double *C0, int ld_C0, int C0_size) {
   or_handle *h = hh;
   h->R_cut = R_cut; h->ld_C0 = ld_C0; h->C0_size = C0_size;
   free(h->C0); h->C0 = malloc(sizeof(double)*(size_t)C0_size);
   memcpy(h->C0, C0, sizeof(double)*(size_t)C0_size);
   or_fill_lut(h);
   h->have_pot = 1;
}
void libgint_set_hf_fac(void *hh, double fac) { ((or_handle*)hh)->hf_fac = fac; }
void libgint_set_max_mem(void *hh, int max_mem) { (void)hh; (void)max_mem; }
static void or_setP(or_handle *h, int nspin, double *Pa, double *Pb, int n) {
   h->nspin = nspin; h->FP_size = (size_t)n;
   for (int s = 0; s < 2; s++) { free(h->P[s]); free(h->K[s]); h->P[s] = h->K[s] = NULL; }
   double *src[2] = {Pa, Pb};
   for (int s = 0; s < nspin; s++) {
      h->P[s] = malloc(sizeof(double)*(size_t)n); memcpy(h->P[s], src[s], sizeof(double)*(size_t)n);
      h->K[s] = calloc((size_t)n, sizeof(double));
   }
}
void libgint_set_P(void *hh, double *P, int P_size) { or_setP(hh, 1, P, NULL, P_size); }
void libgint_set_P_polarized(void *hh, double *Pa, double *Pb, int P_size) { or_setP(hh, 2, Pa, Pb, P_size); }
void libgint_set_K(void *hh, double *K, int K_size) {
   or_handle *h = hh; if ((size_t)K_size != h->FP_size || !h->K[0]) { h->error = 2; return; }
   memcpy(h->K[0], K, sizeof(double)*(size_t)K_size);
}
void libgint_set_K_polarized(void *hh, double *Ka, double *Kb, int K_size) {
   or_handle *h = hh; if ((size_t)K_size != h->FP_size || !h->K[1]) { h->error = 2; return; }
   memcpy(h->K[0], Ka, sizeof(double)*(size_t)K_size);
   memcpy(h->K[1], Kb, sizeof(double)*(size_t)K_size);
}
void libgint_dispatch(void *hh) { or_compute_all(hh); }
void libgint_get_K(void *hh, double *K) {
   or_handle *h = hh; or_compute_all(h);
   if (h->K[0]) memcpy(K, h->K[0], sizeof(double)*h->FP_size);
}
void libgint_get_K_polarized(void *hh, double *Ka, double *Kb) {
   or_handle *h = hh; or_compute_all(h);
   if (h->K[0]) memcpy(Ka, h->K[0], sizeof(double)*h->FP_size);
   if (h->K[1]) memcpy(Kb, h->K[1], sizeof(double)*h->FP_size);
}
void libgint_set_cell(void *hh, bool periodic, double *cell_h, double *cell_i) {
   or_handle *h = hh; h->periodic = periodic;
   for (int i = 0; i < 9; i++) { h->cell[i] = cell_h[i]; h->cell[9+i] = cell_i[i]; }
}
void libgint_set_neighs(void *hh, double *neighs, int nneighs) {
   or_handle *h = hh; free(h->neighs);
   h->neighs = malloc(sizeof(double)*3*(size_t)nneighs);
   memcpy(h->neighs, neighs, sizeof(double)*3*(size_t)nneighs);
   h->Ng = nneighs;
}
void libgint_set_Atom(void *hh, int i, double *R, double *Z, int np) {
   or_handle *h = hh;
   if (i >= h->nsets) {
      h->sets = realloc(h->sets, sizeof(or_set)*(size_t)(i+1));
      memset(h->sets + h->nsets, 0, sizeof(or_set)*(size_t)(i+1-h->nsets));
      h->nsets = i+1;
   }
   or_set *s = &h->sets[i];
   for (int q = 0; q < s->nL; q++) free(s->K[q]);
   memset(s, 0, sizeof(*s));
   memcpy(s->R, R, 3*sizeof(double));
   s->np = np; memcpy(s->Z, Z, sizeof(double)*(size_t)np);
   s->defined = 1;
}
void libgint_set_Atom_L(void *hh, int i, int l, int nl, double *K) {
   or_handle *h = hh;
   or_set *s = &h->sets[i];
   int np = s->np;
   double *Kn = malloc(sizeof(double)*(size_t)(nl*np));
   for (int inl = 0; inl < nl; inl++) {
      /* compute_norm_psi, src/extern_functions.cpp:95-110 */
      const double *Kr = &K[inl*np];
      double ans = 0.0;
      for (int a = 0; a < np; a++) for (int b = 0; b < np; b++)
         ans += Kr[a] * Kr[b] / pow(s->Z[a]+s->Z[b], 1.5+l);
      ans *= pow(M_PI, 1.5) / pow(2.0, l);
      double norm = sqrt(ans);
      for (int ip = 0; ip < np; ip++) Kn[inl*np+ip] = K[inl*np+ip] / norm;
   }
   s->l[s->nL] = l; s->nl[s->nL] = nl; s->K[s->nL] = Kn; s->nL++;
}
void libgint_set_AtomInfo(void *hh, int i, double *R, double *Z, int np, int lmin, int Lmax,
                          int *nl, double *K) {
   libgint_set_Atom(hh, i, R, Z, np);
   int k_offset = 0;
   for (int l = lmin; l < Lmax; l++) {
      libgint_set_Atom_L(hh, i, l, nl[l-lmin], &K[k_offset]);
      k_offset += nl[l-lmin] * np;
   }
}
void libgint_add_prm(void *hh, int ipa, int ipb, int ipc, int ipd) {
   or_handle *h = hh;
   uint32_t code = ((uint32_t)ipa << 24) | ((uint32_t)ipb << 16) | ((uint32_t)ipc << 8) | (uint32_t)ipd;
   VEC_PUSH(h->prm_tmp, code);
}
void libgint_add_shell(void *hh, int i, int j, int k, int l, int n1, int n2) {
   or_handle *h = hh;
   if (h->prm_tmp.n == 0) return;
   const or_set *S[4] = {&h->sets[i], &h->sets[j], &h->sets[k], &h->sets[l]};
   for (int a = 0; a < S[0]->nL; a++) for (int b = 0; b < S[1]->nL; b++)
   for (int c = 0; c < S[2]->nL; c++) for (int d = 0; d < S[3]->nL; d++) {
      or_shell sh;
      sh.set[0] = i; sh.set[1] = j; sh.set[2] = k; sh.set[3] = l;
      sh.lidx[0] = a; sh.lidx[1] = b; sh.lidx[2] = c; sh.lidx[3] = d;
      sh.n1 = n1; sh.n2 = n2;
      sh.cls = S[0]->l[a]*64 + S[1]->l[b]*16 + S[2]->l[c]*4 + S[3]->l[d];
      sh.prm_off = h->set_prms.n; sh.nprm = (int)h->prm_tmp.n;
      for (size_t q = 0; q < h->prm_tmp.n; q++) VEC_PUSH(h->set_prms, h->prm_tmp.d[q]);
      VEC_PUSH(h->set_shells, sh);
   }
   h->prm_tmp.n = 0;
}
void libgint_add_cell(void *hh) { (void)hh; }
void libgint_add_qrt(void *hh, int la, int lb, int lc, int ld, int nla, int nlb, int nlc, int nld) {
   or_handle *h = hh;
   or_group g; memset(&g, 0, sizeof(g));
   g.cls = la*64 + lb*16 + lc*4 + ld;
   g.nl[0] = nla; g.nl[1] = nlb; g.nl[2] = nlc; g.nl[3] = nld;
   VEC_PUSH(h->set_groups, g);
}
void libgint_add_qrtt(void *hh, double symm_fac, int la, int lb, int lc, int ld,
                      int inla, int inlb, int inlc, int inld,
                      int ld_ac, int ld_ad, int ld_bc, int ld_bd,
                      unsigned int off_ac, unsigned int off_ad, unsigned int off_bc, unsigned int off_bd,
                      bool Tac, bool Tad, bool Tbc, bool Tbd) {
   or_handle *h = hh;
   or_qrtt q;
   /* src/libGint.cpp:262-267 */
   unsigned idx_fac = 0;
   if (symm_fac < 0.1) idx_fac = 4;
   else if (symm_fac < 0.3) idx_fac = 3;
   else if (symm_fac < 0.75) idx_fac = 2;
   else if (symm_fac < 1.5) idx_fac = 1;
   else idx_fac = 0;
   q.idx_fac = idx_fac;
   q.inl[0] = inla; q.inl[1] = inlb; q.inl[2] = inlc; q.inl[3] = inld;
   q.ld[0] = ld_ac; q.ld[1] = ld_ad; q.ld[2] = ld_bc; q.ld[3] = ld_bd;
   q.off[0] = off_ac; q.off[1] = off_ad; q.off[2] = off_bc; q.off[3] = off_bd;
   q.T[0] = Tac; q.T[1] = Tad; q.T[2] = Tbc; q.T[3] = Tbd;
   q.cls = la*64 + lb*16 + lc*4 + ld;
   VEC_PUSH(h->set_qrtts, q);
}
void libgint_add_set(void *hh) {
   or_handle *h = hh;
   for (size_t ig = 0; ig < h->set_groups.n; ig++) {
      or_group g = h->set_groups.d[ig];
      g.shell_off = h->shells.n; g.nshell = 0;
      for (size_t is = 0; is < h->set_shells.n; is++) {
         or_shell sh = h->set_shells.d[is];
         if (sh.cls != g.cls) continue;
         size_t off = h->prms.n;
         for (int q = 0; q < sh.nprm; q++) VEC_PUSH(h->prms, h->set_prms.d[sh.prm_off + q]);
         sh.prm_off = off;
         VEC_PUSH(h->shells, sh);
         g.nshell++;
      }
      g.qrtt_off = h->qrtts.n; g.nqrtt = 0;
      for (size_t iq = 0; iq < h->set_qrtts.n; iq++) {
         if (h->set_qrtts.d[iq].cls != g.cls) continue;
         VEC_PUSH(h->qrtts, h->set_qrtts.d[iq]);
         g.nqrtt++;
      }
      if (g.nshell > 0) VEC_PUSH(h->groups, g);
      else { h->shells.n = g.shell_off; h->qrtts.n = g.qrtt_off; }
   }
   h->set_groups.n = 0; h->set_shells.n = 0; h->set_prms.n = 0; h->set_qrtts.n = 0;
}

/* ---- oracle-only controls ---- */
int libgint_last_error(void *hh) { return ((or_handle*)hh)->error; }

/* The engine's bulk form of the call stream (no reference counterpart): the per-item calls of n
 * set quartets made in order, so the bulk path of the engine can be checked against the stream. */
int libgint_add_set_quartets(void *hh, int n, const int *sets, const int *shell_count, const int *shell_images,
                             const int *prm_count, const unsigned int *prm_codes, const int *qrt_count,
                             const int *qrt, const double *qrtt_fac, const int *qrtt_ld,
                             const unsigned int *qrtt_off, const unsigned char *qrtt_T) {
   size_t ish = 0, ip = 0, iqrt = 0, ir = 0;
   for (int q = 0; q < n; q++) {
      const int *s4 = sets + 4 * (size_t)q;
      for (int k = 0; k < shell_count[q]; k++, ish++) {
         for (int p = 0; p < prm_count[ish]; p++, ip++) {
            const unsigned c = prm_codes[ip];
            libgint_add_prm(hh, (int)(c >> 24), (int)((c >> 16) & 255), (int)((c >> 8) & 255), (int)(c & 255));
         }
         libgint_add_shell(hh, s4[0], s4[1], s4[2], s4[3], shell_images[2 * ish], shell_images[2 * ish + 1]);
      }
      for (int t = 0; t < qrt_count[q]; t++, iqrt++) {
         const int *r = qrt + 8 * iqrt;
         libgint_add_qrt(hh, r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]);
         for (int ia = 0; ia < r[4]; ia++) for (int ib = 0; ib < r[5]; ib++)
         for (int ic = 0; ic < r[6]; ic++) for (int id = 0; id < r[7]; id++, ir++) {
            const int *l4 = qrtt_ld + 4 * ir;
            const unsigned int *o4 = qrtt_off + 4 * ir;
            const unsigned char T = qrtt_T[ir];
            libgint_add_qrtt(hh, qrtt_fac[ir], r[0], r[1], r[2], r[3], ia, ib, ic, id, l4[0], l4[1], l4[2], l4[3],
                             o4[0], o4[1], o4[2], o4[3], (T & 1) != 0, (T & 2) != 0, (T & 4) != 0, (T & 8) != 0);
         }
      }
      libgint_add_set(hh);
   }
   return ((or_handle*)hh)->error;
}
void oracle_set_threads(void *hh, int n) { ((or_handle*)hh)->nthreads = n; }
/* magnitude mode (see or_handle.absmode): the following K builds accumulate sums of magnitudes */
void oracle_set_absmode(void *hh, int on) { ((or_handle*)hh)->absmode = on != 0; }
/* the screening-decision counters of the engine's extension (same layout as its
   libgint_get_counters): on = 1 zeroes and starts them */
void libgint_set_counters(void *hh, int on) {
   or_handle *h = hh;
   or_compute_all(h);
   if (on) memset(h->cnt, 0, sizeof(h->cnt));
   h->counting = on != 0;
}
void libgint_get_counters(void *hh, unsigned long long *out) {
   or_handle *h = hh;
   or_compute_all(h);
   memcpy(out, h->cnt, sizeof(h->cnt));
}
void oracle_destroy(void *hh) {
   or_handle *h = hh;
   for (int i = 0; i < h->nsets; i++) for (int q = 0; q < h->sets[i].nL; q++) free(h->sets[i].K[q]);
   free(h->sets); free(h->C0); free(h->neighs);
   for (int s = 0; s < 2; s++) { free(h->P[s]); free(h->K[s]); }
   VEC_FREE(h->prm_tmp); VEC_FREE(h->set_shells); VEC_FREE(h->set_prms); VEC_FREE(h->set_qrtts);
   VEC_FREE(h->set_groups); VEC_FREE(h->shells); VEC_FREE(h->prms); VEC_FREE(h->qrtts);
   VEC_FREE(h->groups);
   free(h);
}
void libgint_destroy_handle(void *hh) { oracle_destroy(hh); }

/* pinning hooks: expose the restated building blocks to the tests */
void oracle_ftable(double *out) { or_make_ftable(out); }
void oracle_fgamma0(int nmax, double T, double *f, double fac) {
   static double ft[121*28]; static int init = 0;
   if (!init) { or_make_ftable(ft); init = 1; }
   or_fgamma0(nmax, T, f, ft, fac);
}
void oracle_c2s(int l, double *out) {
   or_make_c2s();
   int nc = ncart(l), ns = nsph(l);
   for (int m = 0; m < ns; m++) for (int i = 0; i < nc; i++) out[m*nc+i] = or_c2s[l][m][i];
}
void oracle_lut(int *low, int *high) {
   or_handle h; memset(&h, 0, sizeof(h)); or_fill_lut(&h);
   memcpy(low, h.lut_low, sizeof(h.lut_low)); memcpy(high, h.lut_high, sizeof(h.lut_high));
}
/* G_m(T,R)*Kfac with the given table; returns 1 if the Boys branch was used */
int oracle_tcg(double R_cut_unused, const double *C0, int ld_C0, double R, double T, int Nder,
               double Kfac, double *res) {
   (void)R_cut_unused;
   static or_handle h; static int init = 0;
   if (!init) { memset(&h, 0, sizeof(h)); or_fill_lut(&h); or_make_ftable(h.ftable); init = 1; }
   h.C0 = (double*)C0; h.ld_C0 = ld_C0;
   int g = or_tcg(&h, res, R, T, Nder, Kfac);
   if (g == 1) or_fgamma0(Nder, T, res, h.ftable, Kfac);
   return g == 1;
}
void oracle_pbc(const double *A, const double *B, const double *cell, double *AB) { or_pbc(A, B, cell, AB); }
