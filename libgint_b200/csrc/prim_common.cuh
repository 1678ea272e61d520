// prim_common.cuh -- per-primitive-quartet device code shared by the primitive kernels:
// Boys function, truncated-Coulomb G_m, and the geometry whose rounding decides screening.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "engine_types.h"
#include "kernels.h"

namespace gint {

// ---------------------------------------------------------------------------------------
// Boys function (reference src/fgamma.cpp:196-243), result scaled by fac
// ---------------------------------------------------------------------------------------
// NT >= 0 fixes the highest order at compile time (the loops unroll); NT < 0 takes nmax.
template <int NT>
static __device__ __forceinline__ void boys_eval_t(int nmax_rt, double T, double *f, const double *__restrict__ ft,
                                                   double fac) {
   const int nmax = NT >= 0 ? NT : nmax_rt;
   if (T < 1.e-13) {
      for (int n = 0; n <= nmax; n++) f[n] = fac / (2. * n + 1.);
      return;
   }
   if (T < 12.) {
      const double tdelta = 0.1;
      int itab = (int)(round(T / tdelta));
      double ttab = (double)itab * tdelta;
      const double *row = ft + itab * 28 + nmax;
      double d = ttab - T, tmp = d;
      double fL = __ldg(row + 0);
      fL += __ldg(row + 1) * tmp;
      tmp *= d; fL += __ldg(row + 2) * tmp * 0.5;
      tmp *= d; fL += __ldg(row + 3) * tmp * (1. / 6.);
      tmp *= d; fL += __ldg(row + 4) * tmp * (1. / 24.);
      tmp *= d; fL += __ldg(row + 5) * tmp * (1. / 120.);
      tmp *= d; fL += __ldg(row + 6) * tmp * (1. / 720.);
      double expt = exp(-T);
      f[nmax] = fL;
      for (int n = nmax - 1; n >= 0; n--) f[n] = (2.0 * T * f[n + 1] + expt) / (2. * n + 1.);
   } else {
      double tmp = 1.0 / T, tmp2 = tmp * tmp, tmp3 = tmp * tmp2;
      double g = 0.4999489092 - 0.2473631686 * tmp + 0.321180909 * tmp2 - 0.3811559346 * tmp3;
      double expt = exp(-T);
      f[0] = 0.5 * sqrt(M_PI * tmp) - g * expt * tmp;
      for (int n = 1; n <= nmax; n++) f[n] = (0.5 * tmp) * ((2. * n - 1.) * f[n - 1] - expt);
   }
   for (int n = 0; n <= nmax; n++) f[n] *= fac;
}

static __device__ void boys_eval(int nmax, double T, double *f, const double *__restrict__ ft, double fac) {
   boys_eval_t<-1>(nmax, T, f, ft, fac);
}

// ---------------------------------------------------------------------------------------
// Geometry that feeds discrete decisions. The minimum-image rounding (which lattice shift
// brings Q next to P, and so which 27 images the image sum covers), the truncation test, the
// Boys/Chebyshev branch and the patch index all compare rounded doubles against thresholds;
// a one-ulp difference can flip them and change K by far more than one ulp. These values are
// therefore evaluated with explicitly rounded operations in the source's order, with an FMA
// only where the reference's CUDA build contracts one (the weighted distance), so every
// decision is the one the reference makes on the same inputs.
// ---------------------------------------------------------------------------------------
static __device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
static __device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
static __device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
static __device__ __forceinline__ double rdot3(double a0, double b0, double a1, double b1, double a2, double b2) {
   return radd(radd(rmul(a0, b0), rmul(a1, b1)), rmul(a2, b2));
}
// weighted distance (c1 x1 + c2 x2) c12 (reference src/util.h:62-68) as the reference's CUDA
// build evaluates it: the first product contracted into the sum, fma(c1, x1, c2 x2) c12. This
// rounding decides the minimum image of P - Q when P - Q lies on half a lattice vector, which
// happens for symmetric quartets such as (ab|ab') with b' an image of b and equal exponents.
static __device__ __forceinline__ double wdist(double c1, double x1, double c2, double x2, double c12) {
   return rmul(__fma_rn(c1, x1, rmul(c2, x2)), c12);
}

// minimum-image wrap (reference src/util.cpp:132-162)
static __device__ __forceinline__ void pbc(const double *A, const double *B, const double *cell, double *AB) {
   const double *hm = cell, *hi = cell + 9;
   AB[0] = rsub(B[0], A[0]); AB[1] = rsub(B[1], A[1]); AB[2] = rsub(B[2], A[2]);
   double s0 = rdot3(hi[0], AB[0], hi[3], AB[1], hi[6], AB[2]);
   double s1 = rdot3(hi[1], AB[0], hi[4], AB[1], hi[7], AB[2]);
   double s2 = rdot3(hi[2], AB[0], hi[5], AB[1], hi[8], AB[2]);
   s0 = rsub(s0, round(s0)); s1 = rsub(s1, round(s1)); s2 = rsub(s2, round(s2));
   AB[0] = rdot3(hm[0], s0, hm[3], s1, hm[6], s2);
   AB[1] = rdot3(hm[1], s0, hm[4], s1, hm[7], s2);
   AB[2] = rdot3(hm[2], s0, hm[5], s1, hm[8], s2);
}

// shell geometry: A, B (image n1), C, D (image n2) as the reference places them
static __device__ __forceinline__ void shell_geom(const DevCtx &ctx, const BasisEnt &ea, const BasisEnt &eb,
                                                  const BasisEnt &ec, const BasisEnt &ed, int n1, int n2,
                                                  double *A, double *B, double *C, double *D, double *CDs) {
   double ABs[3];
   pbc(ea.R, eb.R, ctx.cell, ABs);
   pbc(ec.R, ed.R, ctx.cell, CDs);
   for (int q = 0; q < 3; q++) {
      A[q] = ea.R[q];
      B[q] = radd(radd(ea.R[q], ABs[q]), __ldg(ctx.neighs + n1 * 3 + q));
      C[q] = ec.R[q];
      D[q] = radd(radd(ec.R[q], CDs[q]), __ldg(ctx.neighs + n2 * 3 + q));
   }
}

// Per-primitive-quartet quantities shared by every image n3. D = P - Q is rounded as the
// reference's T formula rounds it; upper, lower, X2 and i2 (the truncation bounds and the
// second patch coordinate, which depend on R only) are evaluated exactly as t_c_g0_n does.
struct PrimGeo {
   double P[3], Q[3], PA[3], QC[3], D[3];
   double Kfac, rho, R, upper, lower, X2;
   double zab, zcd, inv_z, i2ab, mrab, i2cd, mrcd, i2z;
   int i2, lowR;
};

// prepare_Fm and the image-independent part of compute_Vm (reference
// src/compute_Fm.cpp:66-159, :202-210, :281-290). Q is the ket centre shifted by the
// minimum-image lattice vector of P - Q, so that image n3 sits at Q + neighs[n3].
static __device__ __forceinline__ void prim_geometry(const DevCtx &ctx, const ShellRec &sh, uint32_t code,
                                                     PrimGeo &g) {
   const BasisEnt ea = ctx.ents[sh.ent[0]], eb = ctx.ents[sh.ent[1]];
   const BasisEnt ec = ctx.ents[sh.ent[2]], ed = ctx.ents[sh.ent[3]];
   double A[3], B[3], C[3], D[3], CDs[3];
   shell_geom(ctx, ea, eb, ec, ed, sh.n1, sh.n2, A, B, C, D, CDs);
   const double za = ctx.pool[ea.z_off + (code >> 24)], zb = ctx.pool[eb.z_off + ((code >> 16) & 255)];
   const double zc = ctx.pool[ec.z_off + ((code >> 8) & 255)], zd = ctx.pool[ed.z_off + (code & 255)];
   const double zab = za + zb, inv_zab = 1. / zab, zcd = zc + zd, inv_zcd = 1. / zcd;
   const double z = zab + zcd, inv_z = 1. / z;
   double P[3], Q[3], PQs[3], shift[3];
   for (int q = 0; q < 3; q++) {
      P[q] = wdist(za, A[q], zb, B[q], inv_zab);
      Q[q] = wdist(zc, C[q], zd, D[q], inv_zcd);
   }
   pbc(Q, P, ctx.cell, PQs);
   for (int q = 0; q < 3; q++) shift[q] = rsub(rsub(P[q], Q[q]), PQs[q]);
   const double normf = 2. * 17.493418327624862 * inv_zab * inv_zcd;   // 2 pi^(5/2) / (zab zcd)
   double dx = A[0] - B[0], dy = A[1] - B[1], dz = A[2] - B[2];
   const double RAB2 = dx * dx + dy * dy + dz * dz;
   const double expon_ab = -(za * zb) / (za + zb) * RAB2;
   dx = C[0] - D[0]; dy = C[1] - D[1]; dz = C[2] - D[2];
   const double RCD2 = dx * dx + dy * dy + dz * dz;
   const double expon_cd = -(zc * zd) / (zc + zd) * RCD2;
   g.Kfac = (1. / sqrt(z)) * normf * exp(expon_ab + expon_cd);
   for (int q = 0; q < 3; q++) {
      const double Cs = radd(C[q], shift[q]);
      const double Ds = radd(radd(radd(C[q], CDs[q]), __ldg(ctx.neighs + sh.n2 * 3 + q)), shift[q]);
      g.P[q] = P[q];
      g.Q[q] = wdist(zc, Cs, zd, Ds, inv_zcd);
      g.PA[q] = P[q] - A[q];
      g.QC[q] = g.Q[q] - Cs;
   }
   g.rho = rmul(rmul(zab, zcd), inv_z);
   g.R = rmul(ctx.R_cut, sqrt(g.rho));
   g.zab = zab; g.zcd = zcd; g.inv_z = inv_z;
   const double izab = 1. / zab, izcd = 1. / zcd;
   g.i2ab = 0.5 * izab; g.mrab = -1. * g.rho * izab * g.i2ab;
   g.i2cd = 0.5 * izcd; g.mrcd = -1. * g.rho * izcd * g.i2cd;
   g.i2z = 0.5 * inv_z;
   for (int q = 0; q < 3; q++) g.D[q] = rsub(g.P[q], g.Q[q]);
   // truncation bounds and X2 (reference src/t_c_g0_n.cpp:78-131)
   g.upper = radd(radd(rmul(g.R, g.R), rmul(11.0, g.R)), 50.0);
   g.lower = radd(rsub(rmul(g.R, g.R), rmul(11.0, g.R)), 0.0);
   g.lowR = g.R <= 11.0;
   g.X2 = g.lowR ? g.R / 11.0 : 11.0 / g.R;
   int i2 = (int)(g.X2 * 128);
   g.i2 = i2 == 128 ? 127 : i2;
}

// Incremental replays skip the primitives of screened groups: their truncation bound is set below
// every T, so no image of theirs is evaluated and their targets stay zero.
static __device__ __forceinline__ void kill_if_screened(const BatchArgs &bt, const ShellRec &sh, PrimGeo &g) {
   if (bt.gflags && !__ldg(bt.gflags + sh.group)) g.upper = -1.0;
}

// T = rho |P - Q - neighs[n3]|^2 (reference src/compute_Fm.cpp:204-210)
static __device__ __forceinline__ double image_T(const DevCtx &ctx, const PrimGeo &g, int n3) {
   const double PQ0 = rsub(g.D[0], __ldg(ctx.neighs + n3 * 3 + 0));
   const double PQ1 = rsub(g.D[1], __ldg(ctx.neighs + n3 * 3 + 1));
   const double PQ2 = rsub(g.D[2], __ldg(ctx.neighs + n3 * 3 + 2));
   return rmul(g.rho, rdot3(PQ0, PQ0, PQ1, PQ1, PQ2, PQ2));
}

// the truncation bound R^2 + 11 R + 50 (reference src/t_c_g0_n.cpp:78)
static __device__ __forceinline__ double trunc_upper(double R) {
   return radd(radd(rmul(R, R), rmul(11.0, R)), 50.0);
}

// four consecutive doubles from a 32-byte aligned, read-only global address
static __device__ __forceinline__ void ldg_v4(const double *p, double *v) {
   asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p));
}

// The degree-13 triangular Chebyshev series of one patch at (X1, X2), orders 0..L, times Kfac
// (reference src/t_c_g0_n.cpp:133-178).
template <int LT>
static __device__ __forceinline__ void cheb_eval(const DevCtx &ctx, int L_rt, int patch, double X1, double X2,
                                                 double Kfac, double *res) {
   const int L = LT >= 0 ? LT : L_rt;
   const double B1 = __ldg(ctx.bw + patch * 4 + 0), W1 = __ldg(ctx.bw + patch * 4 + 1);
   const double B2 = __ldg(ctx.bw + patch * 4 + 2), W2 = __ldg(ctx.bw + patch * 4 + 3);
   const double *C0_row = ctx.C0 + (size_t)ctx.ld_C0 * patch;
   const double SQ2 = 1.4142135623730950488016887242096980785696718753;
   double TG1 = (2. * X1 - B1) * W1;
   double TG2 = (2. * X2 - B2) * W2;
   double T1[14], T2[14];
   T1[0] = 1.0; T2[0] = 1.0;
   T1[1] = SQ2 * TG1; T2[1] = SQ2 * TG2;
   T1[2] = 2. * TG1 * T1[1] - SQ2; T2[2] = 2. * TG2 * T2[1] - SQ2;
#pragma unroll
   for (int i = 3; i < 14; i++) {
      T1[i] = 2. * TG1 * T1[i - 1] - T1[i - 2];
      T2[i] = 2. * TG2 * T2[i - 1] - T2[i - 2];
   }
   for (int k = 0; k <= L; k++) {
      // one 32-byte load per four coefficients (each lane reads its own patch, so a narrower
      // load would fetch every sector four times)
      const double *c = C0_row + k * kC0Row;
      double cf[kC0Row];
#pragma unroll
      for (int q = 0; q < kC0Row / 4; q++) ldg_v4(c + 4 * q, cf + 4 * q);
      double tmp = 0.0;
      int jl = 0;
#pragma unroll
      for (int j = 0; j < 14; j++) {
         double dot = 0.0;
#pragma unroll
         for (int l = 0; l < 14 - j; l++) { dot += T1[l] * cf[jl]; jl++; }
         tmp += dot * T2[j];
      }
      res[k] = tmp * Kfac;
   }
}

// four consecutive floats from a 16-byte aligned, read-only global address
static __device__ __forceinline__ void ldg_v4f(const float *p, float *v) {
   asm("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]) : "l"(p));
}

// cheb_eval in FP32 (the mixed-precision path): the patch and its mapped coordinates come from
// the same FP64 decisions; the polynomials, the FP32 copy of the coefficients and the sums are FP32.
template <int LT>
static __device__ __forceinline__ void cheb_eval_f(const DevCtx &ctx, int L_rt, int patch, double X1, double X2,
                                                   double Kfac, float *res) {
   const int L = LT >= 0 ? LT : L_rt;
   const double B1 = __ldg(ctx.bw + patch * 4 + 0), W1 = __ldg(ctx.bw + patch * 4 + 1);
   const double B2 = __ldg(ctx.bw + patch * 4 + 2), W2 = __ldg(ctx.bw + patch * 4 + 3);
   const float *C0_row = ctx.C0f + (size_t)ctx.ld_C0 * patch;
   const float SQ2 = 1.41421356237309505f;
   const float TG1 = (float)((2. * X1 - B1) * W1);
   const float TG2 = (float)((2. * X2 - B2) * W2);
   const float kf = (float)Kfac;
   float T1[14], T2[14];
   T1[0] = 1.0f; T2[0] = 1.0f;
   T1[1] = SQ2 * TG1; T2[1] = SQ2 * TG2;
   T1[2] = 2.f * TG1 * T1[1] - SQ2; T2[2] = 2.f * TG2 * T2[1] - SQ2;
#pragma unroll
   for (int i = 3; i < 14; i++) {
      T1[i] = 2.f * TG1 * T1[i - 1] - T1[i - 2];
      T2[i] = 2.f * TG2 * T2[i - 1] - T2[i - 2];
   }
   for (int k = 0; k <= L; k++) {
      const float *c = C0_row + k * kC0Row;
      float cf[kC0Row];
#pragma unroll
      for (int q = 0; q < kC0Row / 4; q++) ldg_v4f(c + 4 * q, cf + 4 * q);
      float tmp = 0.0f;
      int jl = 0;
#pragma unroll
      for (int j = 0; j < 14; j++) {
         float dot = 0.0f;
#pragma unroll
         for (int l = 0; l < 14 - j; l++) { dot += T1[l] * cf[jl]; jl++; }
         tmp += dot * T2[j];
      }
      res[k] = tmp * kf;
   }
}

// ---------------------------------------------------------------------------------------
// Truncated-Coulomb G_m(T,R) * Kfac (reference src/t_c_g0_n.cpp:67-180); falls back to the
// Boys function for R > 11 and T < R^2 - 11 R.
// ---------------------------------------------------------------------------------------
// returns 0 when T is beyond the truncation (zeros), 1 for the Chebyshev series, 2 for Boys
// LT >= 0 fixes L at compile time (the loops unroll); LT < 0 takes L_rt.
template <int LT>
static __device__ __forceinline__ int fm_eval_t(const DevCtx &ctx, int L_rt, double R, double T, double Kfac,
                                                double *res) {
   const int L = LT >= 0 ? LT : L_rt;
   double upper = trunc_upper(R);
   double lower = radd(rsub(rmul(R, R), rmul(11.0, R)), 0.0);
   double X1, X2;
   int patch;
   if (T > upper) {
      for (int n = 0; n <= L; n++) res[n] = 0.0;
      return 0;
   }
   if (R <= 11.0) {
      X2 = R / 11.0;
      lower = 0.0;
      X1 = rsub(T, lower) / rsub(upper, lower);
      int i1 = (int)(X1 * 128), i2 = (int)(X2 * 128);
      if (i1 == 128) i1 = 127;
      if (i2 == 128) i2 = 127;
      patch = __ldg(ctx.lut_low + i1 * 128 + i2);
   } else {
      if (T < lower) {
         boys_eval_t<LT>(L, T, res, ctx.ftable, Kfac);
         return 2;
      }
      X2 = 11.0 / R;
      X1 = rsub(T, lower) / rsub(upper, lower);
      int i1 = (int)(X1 * 128), i2 = (int)(X2 * 128);
      if (i1 == 128) i1 = 127;
      if (i2 == 128) i2 = 127;
      patch = __ldg(ctx.lut_high + i1 * 128 + i2);
   }
   cheb_eval<LT>(ctx, L, patch, X1, X2, Kfac, res);
   return 1;
}

static __device__ int fm_eval(const DevCtx &ctx, int L, double R, double T, double Kfac, double *res) {
   return fm_eval_t<-1>(ctx, L, R, T, Kfac, res);
}

// G_m * Kfac of one image from the primitive's precomputed bounds and X2; the same decisions and
// arithmetic as fm_eval_t. Returns 0 beyond the truncation, 1 for the series, 2 for Boys.
template <int LT>
static __device__ __forceinline__ int fm_eval_geo(const DevCtx &ctx, int L_rt, const PrimGeo &g, double T,
                                                  double *res) {
   const int L = LT >= 0 ? LT : L_rt;
   if (T > g.upper) {
      for (int n = 0; n <= L; n++) res[n] = 0.0;
      return 0;
   }
   double X1;
   int patch;
   if (g.lowR) {
      X1 = rsub(T, 0.0) / rsub(g.upper, 0.0);
      int i1 = (int)(X1 * 128);
      if (i1 == 128) i1 = 127;
      patch = __ldg(ctx.lut_low + i1 * 128 + g.i2);
   } else {
      if (T < g.lower) {
         boys_eval_t<LT>(L, T, res, ctx.ftable, g.Kfac);
         return 2;
      }
      X1 = rsub(T, g.lower) / rsub(g.upper, g.lower);
      int i1 = (int)(X1 * 128);
      if (i1 == 128) i1 = 127;
      patch = __ldg(ctx.lut_high + i1 * 128 + g.i2);
   }
   cheb_eval<LT>(ctx, L, patch, X1, g.X2, g.Kfac, res);
   return 1;
}

// ---------------------------------------------------------------------------------------
// Contraction rows (QrttRec) are the group kernels' work items; rows are stored in group order,
// group g owning rows [qrtt_off, qrtt_off + nla nlb nlc nld). bt.rowgrp[q / 32] is the group of
// row 32 (q / 32), and at most 32 groups start within one 32-row block.
// ---------------------------------------------------------------------------------------
// the group of row q0 + lane for every lane of a converged warp (q0 a multiple of 32)
static __device__ __forceinline__ uint32_t row_group_warp(const BatchArgs &bt, uint32_t q0, int lane) {
   const uint32_t g0 = __ldg(bt.rowgrp + (q0 >> 5));
   const uint32_t gi = g0 + (uint32_t)lane;
   unsigned bit = 0;
   if (lane > 0 && gi < bt.ngroup) {
      const uint32_t st = __ldg(&bt.groups[gi].qrtt_off);   // > q0: group g0 holds row q0
      if (st - q0 < 32u) bit = 1u << (st - q0);
   }
   const unsigned M = __reduce_or_sync(0xffffffffu, bit);
   return g0 + __popc(M & ((2u << lane) - 1u));
}

// the group of row q, the same in every lane of a converged warp
static __device__ __forceinline__ uint32_t row_group_one(const BatchArgs &bt, uint32_t q, int lane) {
   const uint32_t g0 = __ldg(bt.rowgrp + (q >> 5));
   const uint32_t gi = g0 + 1u + (uint32_t)lane;
   const bool later = gi < bt.ngroup && __ldg(&bt.groups[gi].qrtt_off) <= q;
   return g0 + __popc(__ballot_sync(0xffffffffu, later));
}

// fm_eval_geo for the FP32 path: the same decisions (truncation, branch, patch) in FP64, the
// Chebyshev series in FP32 and the rarely taken Boys branch in FP64, rounded to FP32.
template <int LT>
static __device__ __forceinline__ int fm_eval_geo_f(const DevCtx &ctx, int L_rt, const PrimGeo &g, double T,
                                                    float *res) {
   const int L = LT >= 0 ? LT : L_rt;
   if (T > g.upper) {
      for (int n = 0; n <= L; n++) res[n] = 0.0f;
      return 0;
   }
   double X1;
   int patch;
   if (g.lowR) {
      X1 = rsub(T, 0.0) / rsub(g.upper, 0.0);
      int i1 = (int)(X1 * 128);
      if (i1 == 128) i1 = 127;
      patch = __ldg(ctx.lut_low + i1 * 128 + g.i2);
   } else {
      if (T < g.lower) {
         double tmp[kMaxLL + 1];
         boys_eval_t<LT>(L, T, tmp, ctx.ftable, g.Kfac);
         for (int n = 0; n <= L; n++) res[n] = (float)tmp[n];
         return 2;
      }
      X1 = rsub(T, g.lower) / rsub(g.upper, g.lower);
      int i1 = (int)(X1 * 128);
      if (i1 == 128) i1 = 127;
      patch = __ldg(ctx.lut_high + i1 * 128 + g.i2);
   }
   cheb_eval_f<LT>(ctx, L, patch, X1, g.X2, g.Kfac, res);
   return 1;
}

}  // namespace gint
