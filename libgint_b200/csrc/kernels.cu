// kernels.cu -- sm_100a kernels of the K build.
//
// Two kernels per angular-momentum class (la,lb,lc,ld), launched on class-sorted segments of
// one batch:
//
//  k_prim<TS>   one team of TS lanes per primitive quartet. The lanes evaluate the images n3
//               in parallel (truncated-Coulomb G_m by the patch Chebyshev series, or the Boys
//               function), drop screened images, then run the Obara-Saika VRR of each
//               surviving image cooperatively, level by level, in the team's shared-memory
//               workspace, and sum the (e0|f0)^(0) targets over n3. The image-summed targets
//               of the primitive go to the AC buffer.
//               (reference: src/compute_Fm.cpp:20-326, src/compute_VRR.cpp:349-458,
//                src/compute_ECO.cpp:216-272)
//  k_group      one warp per group (all image pairs of one set quartet for one class): for
//               every contraction row, contract AC over the primitives of each shell, apply
//               the HRR with that shell's AB/CD, sum the shells, transform to spherical and
//               update K with atomics.
//               (reference: src/compute_ECO.cpp:12-214, src/compute_HRR.cpp:102-225,
//                src/compute_SPH.cpp:58-237, src/compute_KS.cpp:8-117)
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include "engine_types.h"
#include "kernels.h"
#include "group3.h"
#include "prim3.h"
#include "prim_common.cuh"

namespace gint {

__constant__ int8_t c_cart_exp[8][36][3];
__constant__ int8_t c_cart_dir[8][36];
__constant__ int8_t c_cart_dec[8][36][3];
__constant__ int8_t c_cart_inc[8][36][3];
__constant__ double c_c2s[4][70];
__constant__ double c_symm[5];

static __device__ __forceinline__ int ncart(int l) { return (l + 1) * (l + 2) / 2; }



// ---------------------------------------------------------------------------------------
// One VRR element of block b (reference VRR1..VRR6, src/compute_VRR.cpp:111-345)
// pqz: PA[3] WP[3] QC[3] WQ[3] i2ab mrab i2cd mrcd i2z
// ---------------------------------------------------------------------------------------
template <int ST>
static __device__ __forceinline__ void vrr_elem_s(const VBlock &b, int e, double *ws, const double *pqz) {
   // ws element x lives at ws[x * ST]: ST = 1 for a team-shared workspace, 32 for the
   // lane-interleaved per-lane workspaces
   const int a = b.a, c = b.c;
   const int na = ncart(a), nc = ncart(c);
   const int k = e % nc, i = (e / nc) % na, mm = e / (nc * na);
   const int m = b.lo + mm;
   double v;
   if (c == 0) {
      const int d = c_cart_dir[a][i];
      const int im = c_cart_dec[a][i][d];
      const int na1 = ncart(a - 1);
      const double *b1 = ws + b.in1 * ST;
      v = pqz[d * ST] * b1[((m - b.lo1) * na1 + im) * ST] + pqz[(3 + d) * ST] * b1[((m + 1 - b.lo1) * na1 + im) * ST];
      const int ed = c_cart_exp[a][i][d];
      if (ed >= 2) {
         const int iw = c_cart_dec[a - 1][im][d];
         const int na2 = ncart(a - 2);
         const double *b2 = ws + b.in2 * ST;
         v += (ed - 1) * (pqz[12 * ST] * b2[((m - b.lo2) * na2 + iw) * ST] + pqz[13 * ST] * b2[((m + 1 - b.lo2) * na2 + iw) * ST]);
      }
   } else {
      const int d = c_cart_dir[c][k];
      const int km = c_cart_dec[c][k][d];
      const int nc1 = ncart(c - 1);
      const double *b1 = ws + b.in1 * ST;
      v = pqz[(6 + d) * ST] * b1[(((m - b.lo1) * na + i) * nc1 + km) * ST] +
          pqz[(9 + d) * ST] * b1[(((m + 1 - b.lo1) * na + i) * nc1 + km) * ST];
      const int cd = c_cart_exp[c][k][d];
      if (cd >= 2) {
         const int kw = c_cart_dec[c - 1][km][d];
         const int nc2 = ncart(c - 2);
         const double *b2 = ws + b.in2 * ST;
         v += (cd - 1) * (pqz[14 * ST] * b2[(((m - b.lo2) * na + i) * nc2 + kw) * ST] +
                          pqz[15 * ST] * b2[(((m + 1 - b.lo2) * na + i) * nc2 + kw) * ST]);
      }
      if (a > 0) {
         const int ad = c_cart_exp[a][i][d];
         if (ad >= 1) {
            const int im = c_cart_dec[a][i][d];
            const double *b3 = ws + b.in3 * ST;
            v += ad * pqz[16 * ST] * b3[(((m + 1 - b.lo3) * ncart(a - 1) + im) * nc1 + km) * ST];
         }
      }
   }
   ws[(b.off + e) * ST] = v;
}

// One level of the precompiled VRR (VOp, see build_vops): instructions [e0, e1) spread over the
// lanes of a team; ws holds a zero at offset V.
static __device__ __forceinline__ void vops_level(const VOp *__restrict__ vop, int e0, int e1, int lane, int stride,
                                                  double *ws, const double *pqz) {
   for (int e = e0 + lane; e < e1; e += stride) {
      const int4 r = __ldg(reinterpret_cast<const int4 *>(vop + e));
      VOp o;
      memcpy(&o, &r, sizeof(VOp));
      double v = pqz[o.zA] * ws[o.i0] + pqz[o.zA + 3] * ws[o.i1];
      if (o.f1) v += o.f1 * (pqz[12 + 2 * o.kind] * ws[o.i2] + pqz[13 + 2 * o.kind] * ws[o.i3]);
      if (o.f2) v += o.f2 * pqz[16] * ws[o.i4];
      ws[o.out] = v;
   }
}

template <int TS>
static __device__ __forceinline__ void team_sync(unsigned mask) {
   if (TS > 1) __syncwarp(mask);
}

// ---------------------------------------------------------------------------------------
// k_prim: Fm + VRR + sum over n3 per primitive quartet
// ---------------------------------------------------------------------------------------
template <int TS>
__global__ void __launch_bounds__(256) k_prim(DevCtx ctx, BatchArgs bt, int team_doubles) {
   extern __shared__ __align__(16) double smem[];
   ClassPlan *pl = reinterpret_cast<ClassPlan *>(smem);
   {
      const int nwords = (int)(sizeof(ClassPlan) / 4);
      const int *src = reinterpret_cast<const int *>(bt.plan);
      int *dst = reinterpret_cast<int *>(smem);
      for (int w = threadIdx.x; w < nwords; w += blockDim.x) dst[w] = src[w];
   }
   __syncthreads();
   const int plan_doubles = (int)((sizeof(ClassPlan) + 15) / 16) * 2;
   const int team = threadIdx.x / TS, lane = threadIdx.x % TS, nteam = blockDim.x / TS;
   double *tws = smem + plan_doubles + (size_t)team * team_doubles;
   const int L = pl->L, V = pl->V, S = pl->S;
   double *ws = tws;                  // VRR workspace [V] and a zero slot
   double *acc = tws + V + 1;         // image-summed targets [S]
   double *pqz = acc + S;             // 17 factors of the image being processed
   double *fmx = pqz + 17;            // per-lane Fm [TS][L+1]
   const unsigned wl = (threadIdx.x & 31) / TS * TS;
   const unsigned mask = (TS >= 32) ? 0xffffffffu : (((1u << TS) - 1u) << wl);

   if (lane == 0) ws[V] = 0.0;
   for (uint32_t p = blockIdx.x * nteam + team; p < bt.nprm; p += gridDim.x * nteam) {
      PrimGeo g;
      prim_geometry(ctx, bt.shells[bt.prm_shell[p]], bt.prm[p], g);
      kill_if_screened(bt, bt.shells[bt.prm_shell[p]], g);

      for (int j = lane; j < S; j += TS) acc[j] = 0.0;
      double s00 = 0.0;
      unsigned c_cheb = 0, c_boys = 0, c_vrr = 0;
      // (ss|ss) needs no VRR: its only target is the image sum of (00|00)
      const bool need_vrr = !(pl->want00 && pl->ntg == 1);
      team_sync<TS>(mask);

      for (int n0 = 0; n0 < ctx.Ng; n0 += TS) {
         const int n3 = n0 + lane;
         bool surv = false;
         double *myfm = fmx + lane * (L + 1);
         if (n3 < ctx.Ng && !(g.upper < 0.0)) {
            const double T = image_T(ctx, g, n3);
            const int br = fm_eval(ctx, L, g.R, T, g.Kfac, myfm);
            c_cheb += (br == 1); c_boys += (br == 2);
            s00 += myfm[0];
            surv = need_vrr && (myfm[0] > 1.e-12);
         }
         unsigned bal = (TS > 1) ? ((__ballot_sync(mask, surv) & mask) >> wl) : (surv ? 1u : 0u);
         while (bal) {
            const int src = __ffs(bal) - 1;
            bal &= bal - 1;
            if (lane == src) {
               c_vrr++;
               const int n3s = n0 + src;
               const double g0 = __ldg(ctx.neighs + n3s * 3 + 0), g1 = __ldg(ctx.neighs + n3s * 3 + 1),
                            g2 = __ldg(ctx.neighs + n3s * 3 + 2);
               const double Qp0 = g.Q[0] + g0, Qp1 = g.Q[1] + g1, Qp2 = g.Q[2] + g2;
               const double W0 = wdist(g.zab, g.P[0], g.zcd, Qp0, g.inv_z);
               const double W1 = wdist(g.zab, g.P[1], g.zcd, Qp1, g.inv_z);
               const double W2 = wdist(g.zab, g.P[2], g.zcd, Qp2, g.inv_z);
               pqz[0] = g.PA[0]; pqz[1] = g.PA[1]; pqz[2] = g.PA[2];
               pqz[3] = W0 - g.P[0]; pqz[4] = W1 - g.P[1]; pqz[5] = W2 - g.P[2];
               pqz[6] = g.QC[0]; pqz[7] = g.QC[1]; pqz[8] = g.QC[2];
               pqz[9] = W0 - Qp0; pqz[10] = W1 - Qp1; pqz[11] = W2 - Qp2;
               pqz[12] = g.i2ab; pqz[13] = g.mrab; pqz[14] = g.i2cd; pqz[15] = g.mrcd; pqz[16] = g.i2z;
               const int n00 = pl->vb[0].nm;
               for (int q = 0; q < n00; q++) ws[q] = myfm[q];
            }
            team_sync<TS>(mask);
            for (int lv = 1; lv <= pl->nlev; lv++) {
               vops_level(ctx.vops + pl->vop_off, pl->vop_lev[lv - 1], pl->vop_lev[lv], lane, TS, ws, pqz);
               team_sync<TS>(mask);
            }
            for (int t = 0; t < pl->ntg; t++) {
               if (pl->want00 && pl->tg_e[t] == 0 && pl->tg_f[t] == 0) continue;
               const double *srcp = ws + pl->tg_voff[t];
               double *dst = acc + pl->tg_soff[t];
               for (int q = lane; q < pl->tg_n[t]; q += TS) dst[q] += srcp[q];
            }
            team_sync<TS>(mask);
         }
      }
      if (pl->want00) {
         if (TS > 1) {
#pragma unroll
            for (int o = TS / 2; o > 0; o >>= 1) s00 += __shfl_down_sync(mask, s00, o, TS);
         }
         if (lane == 0) acc[pl->s00] += s00;
      }
      if (ctx.cnt) {
         if (TS > 1) {
#pragma unroll
            for (int o = TS / 2; o > 0; o >>= 1) {
               c_cheb += __shfl_down_sync(mask, c_cheb, o, TS);
               c_boys += __shfl_down_sync(mask, c_boys, o, TS);
               c_vrr += __shfl_down_sync(mask, c_vrr, o, TS);
            }
         }
         if (lane == 0) {
            atomicAdd(ctx.cnt + bt.cls * 4 + 0, (unsigned long long)c_cheb);
            atomicAdd(ctx.cnt + bt.cls * 4 + 1, (unsigned long long)c_boys);
            atomicAdd(ctx.cnt + bt.cls * 4 + 2, (unsigned long long)c_vrr);
            atomicAdd(ctx.cnt + bt.cls * 4 + 3, 1ull);
         }
      }
      team_sync<TS>(mask);
      double *out = bt.AC + (size_t)p * S;
      for (int j = lane; j < S; j += TS) out[j] = acc[j];
      team_sync<TS>(mask);
   }
}

// ---------------------------------------------------------------------------------------
// k_prim2<LANE_VRR>: Fm + VRR + sum over n3, one warp per chunk of primitive quartets with
// two compaction stages. (1) all (primitive, image) pairs get the cheap truncation test
// T <= R^2 + 11R + 50 and the passing pairs are queued; (2) the queue is evaluated 32 at a time
// (G_m by the Chebyshev series or Boys) so that every lane does useful work, and the images with
// Fm[0] > 1e-12 are queued again; (3) their VRR runs one image per lane (LANE_VRR, small
// classes, lane-interleaved workspaces) or one image per warp (level-parallel), and the m = 0
// targets are summed per primitive in shared memory.
// ---------------------------------------------------------------------------------------
template <bool LANE_VRR>
__global__ void __launch_bounds__(256) k_prim2(DevCtx ctx, BatchArgs bt, int cp, int warp_doubles) {
   extern __shared__ __align__(16) double smem[];
   ClassPlan *pl = reinterpret_cast<ClassPlan *>(smem);
   {
      const int nwords = (int)(sizeof(ClassPlan) / 4);
      const int *src = reinterpret_cast<const int *>(bt.plan);
      int *dst = reinterpret_cast<int *>(smem);
      for (int w = threadIdx.x; w < nwords; w += blockDim.x) dst[w] = src[w];
   }
   __syncthreads();
   const int plan_doubles = (int)((sizeof(ClassPlan) + 15) / 16) * 2;
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
   double *wb = smem + plan_doubles + (size_t)warp * warp_doubles;
   const int L = pl->L, S = pl->S, Ng = ctx.Ng;
   const int LF = L + 1;
   // per-warp layout
   PrimGeo *geo = reinterpret_cast<PrimGeo *>(wb);                     // [cp]
   double *s00 = wb + cp * (sizeof(PrimGeo) / 8);                     // [cp]
   double *acc = s00 + cp;                                            // [cp][S]
   int *q1i = reinterpret_cast<int *>(acc + (size_t)cp * S);          // [64] pair index
   double *q1t = acc + (size_t)cp * S + 32;                           // [64] T
   int *q2i = reinterpret_cast<int *>(q1t + 64);                      // [64] pair index
   double *q2f = q1t + 64 + 32;                                       // [64][LF] Fm
   double *pqz = q2f + 64 * LF;                                       // [17][32] (lane) or [17]
   double *ws = pqz + (LANE_VRR ? 17 * 32 : 18);                      // [V][32] (lane) or [V] + zero
   const bool need_vrr = !(pl->want00 && pl->ntg == 1);
   const unsigned below = (1u << lane) - 1u;
   unsigned long long c_cheb = 0, c_boys = 0, c_vrr = 0;
   if (!LANE_VRR && lane == 0) ws[pl->V] = 0.0;

   const uint32_t nchunk = (bt.nprm + cp - 1) / cp;
   for (uint32_t ch = blockIdx.x * nwarp + warp; ch < nchunk; ch += gridDim.x * nwarp) {
      const uint32_t p0 = ch * cp;
      const int np = (int)min((uint32_t)cp, bt.nprm - p0);
      // ---- per-primitive geometry (reference src/compute_Fm.cpp:66-159, :202-210, :281-290)
      if (lane < np) {
         const uint32_t p = p0 + lane;
         PrimGeo g;
         prim_geometry(ctx, bt.shells[bt.prm_shell[p]], bt.prm[p], g);
         kill_if_screened(bt, bt.shells[bt.prm_shell[p]], g);
         geo[lane] = g;
         s00[lane] = 0.0;
      }
      for (int j = lane; j < np * S; j += 32) acc[j] = 0.0;
      __syncwarp();

      int n1 = 0, n2 = 0;
      const int npair = np * Ng;
      // stage 3: VRR of the queued images [0, cnt)
      auto run_vrr = [&](int cnt) {
         if (LANE_VRR) {
            if (lane < cnt) {
               const int pi = q2i[lane];
               const int p = pi / Ng, n3 = pi - p * Ng;
               const PrimGeo &g = geo[p];
               const double g0 = __ldg(ctx.neighs + n3 * 3 + 0), g1 = __ldg(ctx.neighs + n3 * 3 + 1),
                            g2 = __ldg(ctx.neighs + n3 * 3 + 2);
               const double Qp[3] = {g.Q[0] + g0, g.Q[1] + g1, g.Q[2] + g2};
               double *pz = pqz + lane;
               for (int q = 0; q < 3; q++) {
                  const double W = wdist(g.zab, g.P[q], g.zcd, Qp[q], g.inv_z);
                  pz[q * 32] = g.PA[q];
                  pz[(3 + q) * 32] = W - g.P[q];
                  pz[(6 + q) * 32] = g.QC[q];
                  pz[(9 + q) * 32] = W - Qp[q];
               }
               pz[12 * 32] = g.i2ab; pz[13 * 32] = g.mrab; pz[14 * 32] = g.i2cd; pz[15 * 32] = g.mrcd;
               pz[16 * 32] = g.i2z;
               double *w = ws + lane;
               const int n00 = pl->vb[0].nm;
               for (int q = 0; q < n00; q++) w[q * 32] = q2f[lane * LF + q];
               for (int bb = 1; bb < pl->nvb; bb++) {
                  const VBlock vb = pl->vb[bb];
                  for (int e = 0; e < vb.nelem; e++) vrr_elem_s<32>(vb, e, w, pz);
               }
               double *ap = acc + (size_t)p * S;
               for (int t = 0; t < pl->ntg; t++) {
                  if (pl->want00 && pl->tg_e[t] == 0 && pl->tg_f[t] == 0) continue;
                  const double *sp = w + pl->tg_voff[t] * 32;
                  double *dp = ap + pl->tg_soff[t];
                  for (int q = 0; q < pl->tg_n[t]; q++) atomicAdd(dp + q, sp[q * 32]);
               }
            }
            __syncwarp();
         } else {
            for (int s = 0; s < cnt; s++) {
               const int pi = q2i[s];
               const int p = pi / Ng, n3 = pi - p * Ng;
               const PrimGeo &g = geo[p];
               if (lane < 3) {
                  const int q = lane;
                  const double gq = __ldg(ctx.neighs + n3 * 3 + q);
                  const double Qp = g.Q[q] + gq;
                  const double W = wdist(g.zab, g.P[q], g.zcd, Qp, g.inv_z);
                  pqz[q] = g.PA[q]; pqz[3 + q] = W - g.P[q]; pqz[6 + q] = g.QC[q]; pqz[9 + q] = W - Qp;
               } else if (lane == 3) {
                  pqz[12] = g.i2ab; pqz[13] = g.mrab; pqz[14] = g.i2cd; pqz[15] = g.mrcd; pqz[16] = g.i2z;
               }
               const int n00 = pl->vb[0].nm;
               for (int q = lane; q < n00; q += 32) ws[q] = q2f[s * LF + q];
               __syncwarp();
               for (int lv = 1; lv <= pl->nlev; lv++) {
                  vops_level(ctx.vops + pl->vop_off, pl->vop_lev[lv - 1], pl->vop_lev[lv], lane, 32, ws, pqz);
                  __syncwarp();
               }
               double *ap = acc + (size_t)p * S;
               for (int t = 0; t < pl->ntg; t++) {
                  if (pl->want00 && pl->tg_e[t] == 0 && pl->tg_f[t] == 0) continue;
                  const double *sp = ws + pl->tg_voff[t];
                  double *dp = ap + pl->tg_soff[t];
                  for (int q = lane; q < pl->tg_n[t]; q += 32) dp[q] += sp[q];
               }
               __syncwarp();
            }
         }
      };
      // stage 2: G_m of the queued pairs [0, cnt), one per lane
      auto run_fm = [&](int cnt) {
         bool surv = false;
         double fm[kMaxLL + 1];
         int pi = 0;
         if (lane < cnt) {
            pi = q1i[lane];
            const double T = q1t[lane];
            const int p = pi / Ng;
            const PrimGeo &g = geo[p];
            const int br = fm_eval(ctx, L, g.R, T, g.Kfac, fm);
            c_cheb += (br == 1); c_boys += (br == 2);
            if (pl->want00) atomicAdd(s00 + p, fm[0]);
            surv = need_vrr && (fm[0] > 1.e-12);
         }
         const unsigned bal = __ballot_sync(0xffffffffu, surv);
         if (surv) {
            const int pos = n2 + __popc(bal & below);
            q2i[pos] = pi;
            for (int q = 0; q < LF; q++) q2f[pos * LF + q] = fm[q];
         }
         n2 += __popc(bal);
         __syncwarp();
         const int step = LANE_VRR ? 32 : 1;
         while (n2 >= step || (n2 > 0 && !LANE_VRR)) {
            const int cnt2 = LANE_VRR ? 32 : n2;
            c_vrr += (lane == 0) ? cnt2 : 0;
            run_vrr(cnt2);
            // shift the remainder down
            const int rem = n2 - cnt2;
            int v = 0;
            double tmp[kMaxLL + 1];
            if (lane < rem) {
               v = q2i[cnt2 + lane];
               for (int q = 0; q < LF; q++) tmp[q] = q2f[(cnt2 + lane) * LF + q];
            }
            __syncwarp();
            if (lane < rem) {
               q2i[lane] = v;
               for (int q = 0; q < LF; q++) q2f[lane * LF + q] = tmp[q];
            }
            __syncwarp();
            n2 = rem;
         }
      };
      // stage 1: truncation test over all (primitive, image) pairs
      for (int b0 = 0; b0 < npair; b0 += 32) {
         const int pi = b0 + lane;
         bool pass = false;
         double T = 0.0;
         if (pi < npair) {
            const int p = pi / Ng, n3 = pi - p * Ng;
            const PrimGeo &g = geo[p];
            T = image_T(ctx, g, n3);
            pass = !(T > g.upper);   // g.upper = trunc_upper(g.R), or -1 for a screened primitive
         }
         const unsigned bal = __ballot_sync(0xffffffffu, pass);
         if (pass) {
            const int pos = n1 + __popc(bal & below);
            q1i[pos] = pi;
            q1t[pos] = T;
         }
         n1 += __popc(bal);
         __syncwarp();
         if (n1 >= 32) {
            run_fm(32);
            const int rem = n1 - 32;
            int vi = 0; double vt = 0.0;
            if (lane < rem) { vi = q1i[32 + lane]; vt = q1t[32 + lane]; }
            __syncwarp();
            if (lane < rem) { q1i[lane] = vi; q1t[lane] = vt; }
            __syncwarp();
            n1 = rem;
         }
      }
      if (n1 > 0) { run_fm(n1); n1 = 0; }
      if (n2 > 0) {
         c_vrr += (lane == 0) ? n2 : 0;
         run_vrr(n2);
         n2 = 0;
      }
      // the (00|00) target collects every image (reference src/compute_VRR.cpp:381-389)
      if (pl->want00 && lane < np) acc[(size_t)lane * S + pl->s00] += s00[lane];
      if (lane == 0 && ctx.cnt) atomicAdd(ctx.cnt + bt.cls * 4 + 3, (unsigned long long)np);
      __syncwarp();
      double *out = bt.AC + (size_t)p0 * S;
      for (int j = lane; j < np * S; j += 32) out[j] = acc[j];
      __syncwarp();
   }
   if (ctx.cnt) {
      for (int o = 16; o > 0; o >>= 1) {
         c_cheb += __shfl_down_sync(0xffffffffu, c_cheb, o);
         c_boys += __shfl_down_sync(0xffffffffu, c_boys, o);
         c_vrr += __shfl_down_sync(0xffffffffu, c_vrr, o);
      }
      if (lane == 0) {
         atomicAdd(ctx.cnt + bt.cls * 4 + 0, c_cheb);
         atomicAdd(ctx.cnt + bt.cls * 4 + 1, c_boys);
         atomicAdd(ctx.cnt + bt.cls * 4 + 2, c_vrr);
      }
   }
}

// ---------------------------------------------------------------------------------------
// k_group: contraction + HRR + sum over image pairs + spherical transform + K update
// ---------------------------------------------------------------------------------------
// One group (all image pairs of one set quartet, all contraction rows) processed by NL
// cooperating lanes (NL = 32: one warp; NL = 1: one lane) whose workspace element x lives at
// ws[x * ST] (ST = 32 for lane-interleaved per-lane workspaces).
// Nonzero pattern of the cartesian -> spherical rows (bit k of kC2sMask[l][m]: coefficient k of
// row m), the integer solid-harmonic rows the coefficients are made from. Terms outside it are
// exact zeros, so leaving them out changes no sum; upload_constant_tables checks the pattern
// against the coefficients it uploads.
__host__ __device__ constexpr uint16_t c2s_mask(int l, int m) {
   constexpr uint16_t t[4][7] = {{0x1, 0, 0, 0, 0, 0, 0},
                                 {0x2, 0x4, 0x1, 0, 0, 0, 0},
                                 {0x02, 0x10, 0x29, 0x04, 0x09, 0, 0},
                                 {0x042, 0x010, 0x142, 0x284, 0x029, 0x084, 0x009}};
   return t[l][m];
}

// One spherical pass over centre LX: the workspace is [npre][ncart(LX)][npost] in, and
// [npre][2LX+1][npost] out. Each lane transforms whole vectors (one (pre, post) pair at a time),
// so the coefficients are uniform across the warp. Same sum order as a dense row loop.
template <int LX, int NL, int ST>
static __device__ __forceinline__ void sph_pass(const double *src, double *dst, int npre, int npost, int lane) {
   constexpr int NK = (LX + 1) * (LX + 2) / 2, NSX = 2 * LX + 1;
   const int nu = npre * npost;
   for (int u = lane; u < nu; u += NL) {
      const int pre = u / npost, post = u - pre * npost;
      const double *s = src + (pre * NK * npost + post) * ST;
      double *d = dst + (pre * NSX * npost + post) * ST;
      double x[NK];
#pragma unroll
      for (int k = 0; k < NK; k++) x[k] = s[k * npost * ST];
#pragma unroll
      for (int m = 0; m < NSX; m++) {
         double acc = 0.0;
#pragma unroll
         for (int k = 0; k < NK; k++)
            if (c2s_mask(LX, m) >> k & 1) acc += c_c2s[LX][m * NK + k] * x[k];
         d[m * npost * ST] = acc;
      }
   }
}

// q = t / n for t * n < 2^20, with M = 2^20 / n + 1 (all spherical indices here: t < 7^4, n <= 7^3)
static __device__ __forceinline__ int div_small(int t, uint32_t M) { return (int)(((uint32_t)t * M) >> 20); }

// Synchronises the NL threads that share one row's workspace: a block (NL > 32), a warp, or none.
template <int NL>
static __device__ __forceinline__ void gsync() {
   if constexpr (NL > 32) __syncthreads();
   else if constexpr (NL > 1) __syncwarp();
}

// What the rows of one set quartet share for one shell quartet: its primitive range, the
// coefficient rows of its four basis entries and the HRR displacements AB = A - B, CD = C - D.
struct ShellShared {
   uint32_t key;              // group index it was derived for (shell 0 of that group); ~0u: empty
   uint32_t prm_off, nprm;
   int k_off[4], np[4];
   double AB[3], CD[3];
};
static_assert(sizeof(ShellShared) <= kGroupShellCacheDoubles * 8, "shell cache slot too small");

static __device__ __forceinline__ void shell_shared(const DevCtx &ctx, const ShellRec &sh, ShellShared &o) {
   const BasisEnt ea = ctx.ents[sh.ent[0]], eb = ctx.ents[sh.ent[1]];
   const BasisEnt ec = ctx.ents[sh.ent[2]], ed = ctx.ents[sh.ent[3]];
   o.prm_off = sh.prm_off; o.nprm = sh.nprm;
   o.k_off[0] = ea.k_off; o.k_off[1] = eb.k_off; o.k_off[2] = ec.k_off; o.k_off[3] = ed.k_off;
   o.np[0] = ea.np; o.np[1] = eb.np; o.np[2] = ec.np; o.np[3] = ed.np;
   double A[3], B[3], C[3], D[3], CDs[3];
   shell_geom(ctx, ea, eb, ec, ed, sh.n1, sh.n2, A, B, C, D, CDs);
   for (int c = 0; c < 3; c++) { o.AB[c] = A[c] - B[c]; o.CD[c] = C[c] - D[c]; }
}

// One contraction row q (of group gi = G) processed by NL cooperating threads (a block, a warp or
// one lane; `lane` is the thread's index among them). With a cache slot (one warp's shared memory,
// key ~0u at first), shell 0's shared data is derived once and reused by the next rows of the
// same group that this warp takes.
template <int NL, int ST>
static __device__ __forceinline__ void group_body(const DevCtx &ctx, const BatchArgs &bt, const ClassPlan *pl,
                                                  const GroupRec &G, uint32_t q, double *ws, double *cart, int lane,
                                                  const uint2 *hrec, double *kpw, ShellShared *cache = nullptr,
                                                  uint32_t gi = 0) {
   const int S = pl->S, Nc = pl->Nc, Ns = pl->Ns;
   const int la = pl->la, lb = pl->lb, lc = pl->lc, ld = pl->ld;
   const int nca = ncart(la), ncb = ncart(lb), ncc = ncart(lc), ncd_ = ncart(ld);
   const int nsa = 2 * la + 1, nsb = 2 * lb + 1, nsc = 2 * lc + 1, nsd = 2 * ld + 1;
   const int nl1 = G.nl[1], nl2 = G.nl[2], nl3 = G.nl[3];
   {
      const int r = (int)(q - G.qrtt_off);
      const int ia = r / (nl1 * nl2 * nl3), ib = (r / (nl2 * nl3)) % nl1, ic = (r / nl3) % nl2, id = r % nl3;
      for (int x = lane; x < Nc; x += NL) cart[x * ST] = 0.0;
      for (uint32_t s = 0; s < G.nshell; s++) {
         ShellShared sh;
         if (cache && s == 0 && cache->key == gi) {
            sh = *cache;
         } else {
            shell_shared(ctx, bt.shells[G.shell_off + s], sh);
            if (cache && s == 0) {
               gsync<NL>();
               if (lane == 0) { *cache = sh; cache->key = gi; }
               gsync<NL>();
            }
         }
         const double *Ka = ctx.pool + sh.k_off[0] + ia * sh.np[0];
         const double *Kb = ctx.pool + sh.k_off[1] + ib * sh.np[1];
         const double *Kc = ctx.pool + sh.k_off[2] + ic * sh.np[2];
         const double *Kd = ctx.pool + sh.k_off[3] + id * sh.np[3];
         // contraction over primitives (reference src/compute_ECO.cpp:131-212)
         if constexpr (NL >= 32) {
            // the contraction coefficients of 32 primitives at a time, one per thread, then every
            // thread sums its targets over them in primitive order
            if (sh.nprm == 0)
               for (int j = lane; j < S; j += NL) ws[j] = 0.0;
            for (uint32_t p0 = 0; p0 < sh.nprm; p0 += 32) {
               const int np = (int)min(32u, sh.nprm - p0);
               if (lane < np) {
                  const uint32_t code = __ldg(bt.prm + sh.prm_off + p0 + lane);
                  kpw[lane] = __ldg(Ka + (code >> 24)) * __ldg(Kb + ((code >> 16) & 255)) *
                              __ldg(Kc + ((code >> 8) & 255)) * __ldg(Kd + (code & 255));
               }
               gsync<NL>();
               const double *acp = bt.AC + (size_t)(sh.prm_off + p0) * S;
               for (int j = lane; j < S; j += NL) {
                  double a = p0 ? ws[j] : 0.0;
                  const double *rp = acp + j;
                  int q = 0;
                  for (; q + 4 <= np; q += 4) {
                     const double v0 = __ldg(rp), v1 = __ldg(rp + S), v2 = __ldg(rp + 2 * S), v3 = __ldg(rp + 3 * S);
                     a += kpw[q] * v0;
                     a += kpw[q + 1] * v1;
                     a += kpw[q + 2] * v2;
                     a += kpw[q + 3] * v3;
                     rp += 4 * S;
                  }
                  for (; q < np; q++) { a += kpw[q] * __ldg(rp); rp += S; }
                  ws[j] = a;
               }
               gsync<NL>();
            }
         } else {
            for (int j = lane; j < S; j += NL) {
               double a = 0.0;
               for (uint32_t ip = 0; ip < sh.nprm; ip++) {
                  const uint32_t code = bt.prm[sh.prm_off + ip];
                  const double kp = __ldg(Ka + (code >> 24)) * __ldg(Kb + ((code >> 16) & 255)) *
                                    __ldg(Kc + ((code >> 8) & 255)) * __ldg(Kd + (code & 255));
                  a += kp * bt.AC[(size_t)(sh.prm_off + ip) * S + j];
               }
               ws[j * ST] = a;
            }
         }
         gsync<NL>();
         // HRR (reference src/compute_HRR.cpp:7-99), one precompiled instruction per element; the
         // elements of one level are independent, so each lane loads four before it stores any
         for (int lv = 1; lv <= pl->nhlev; lv++) {
            const HOp h0 = pl->hop[pl->hlev_off[lv - 1]], h1 = pl->hop[pl->hlev_off[lv] - 1];
            const int x0 = h0.out, x1 = h1.out + h1.nelem;
            double R0, R1, R2;
            if (h0.type == 0) { R0 = sh.CD[0]; R1 = sh.CD[1]; R2 = sh.CD[2]; }
            else { R0 = sh.AB[0]; R1 = sh.AB[1]; R2 = sh.AB[2]; }
            for (int x = x0 + lane; x < x1; x += 4 * NL) {
               uint2 ins[4];
#pragma unroll
               for (int u = 0; u < 4; u++) ins[u] = __ldg(&hrec[min(x + u * NL, x1 - 1) - S]);
               double w1[4], w2[4];
#pragma unroll
               for (int u = 0; u < 4; u++) { w1[u] = ws[(ins[u].x & 0x3fffffffu) * ST]; w2[u] = ws[ins[u].y * ST]; }
#pragma unroll
               for (int u = 0; u < 4; u++) {
                  if (x + u * NL < x1) {
                     const uint32_t dir = ins[u].x >> 30;
                     const double Rd = dir == 0 ? R0 : (dir == 1 ? R1 : R2);
                     ws[(x + u * NL) * ST] = w1[u] + Rd * w2[u];
                  }
               }
            }
            gsync<NL>();
         }
         for (int x = lane; x < Nc; x += NL) cart[x * ST] += ws[(pl->out_off + x) * ST];
         gsync<NL>();
      }
      // cartesian -> spherical, one centre at a time (a, b, c, d); the two halves of the
      // workspace take turns as the output, and l = 0 centres (a coefficient of 1) are skipped
      const double *sph = cart;
      {
         int dims[4] = {nca, ncb, ncc, ncd_};
         const int ls[4] = {la, lb, lc, ld};
         const int ns[4] = {nsa, nsb, nsc, nsd};
         for (int ctr = 0; ctr < 4; ctr++) {
            if (ls[ctr] == 0) continue;
            double *dst = (sph == ws) ? ws + Nc * ST : ws;
            int npre = 1, npost = 1;
            for (int q = 0; q < ctr; q++) npre *= dims[q];
            for (int q = ctr + 1; q < 4; q++) npost *= dims[q];
            if (ls[ctr] == 1) sph_pass<1, NL, ST>(sph, dst, npre, npost, lane);
            else if (ls[ctr] == 2) sph_pass<2, NL, ST>(sph, dst, npre, npost, lane);
            else sph_pass<3, NL, ST>(sph, dst, npre, npost, lane);
            gsync<NL>();
            dims[ctr] = ns[ctr];
            sph = dst;
         }
      }
      // K update (reference src/compute_KS.cpp:26-115)
      const QrttRec k = bt.qrtts[q];
      const double fac = c_symm[k.idx_fac] * ctx.hf_fac;
      const int nscd = nsc * nsd, nsbcd = nsb * nscd;
      const uint32_t Mbcd = (1u << 20) / nsbcd + 1, Mcd = (1u << 20) / nscd + 1, Md = (1u << 20) / nsd + 1;
      for (int t = lane; t < Ns; t += NL) {
         const int isa = div_small(t, Mbcd);
         int rem = t - isa * nsbcd;
         const int isb = div_small(rem, Mcd);
         rem -= isb * nscd;
         const int isc = div_small(rem, Md), isd = rem - isc * nsd;
         const int iac = !(k.T & 1) ? isc * k.ld[0] + isa : isa * k.ld[0] + isc;
         const int iad = !(k.T & 2) ? isd * k.ld[1] + isa : isa * k.ld[1] + isd;
         const int ibc = !(k.T & 4) ? isc * k.ld[2] + isb : isb * k.ld[2] + isc;
         const int ibd = !(k.T & 8) ? isd * k.ld[3] + isb : isb * k.ld[3] + isd;
         const size_t Iac = (size_t)k.off[0] + iac, Iad = (size_t)k.off[1] + iad;
         const size_t Ibc = (size_t)k.off[2] + ibc, Ibd = (size_t)k.off[3] + ibd;
         if (Iac >= ctx.FP_size || Iad >= ctx.FP_size || Ibc >= ctx.FP_size || Ibd >= ctx.FP_size) {
            atomicOr(ctx.err, 1);
            continue;
         }
         const double iabcd = -fac * sph[t * ST];
         for (int sp = 0; sp < ctx.nspin; sp++) {
            const double *Pm = ctx.P[sp];
            double *Km = ctx.K[sp];
            atomicAdd(Km + Ibd, iabcd * __ldg(Pm + Iac));
            atomicAdd(Km + Ibc, iabcd * __ldg(Pm + Iad));
            atomicAdd(Km + Iad, iabcd * __ldg(Pm + Ibc));
            atomicAdd(Km + Iac, iabcd * __ldg(Pm + Ibd));
         }
      }
      gsync<NL>();
   }
}

static __device__ __forceinline__ void load_plan(const ClassPlan *src_plan, double *smem) {
   const int nwords = (int)(sizeof(ClassPlan) / 4);
   const int *src = reinterpret_cast<const int *>(src_plan);
   int *dst = reinterpret_cast<int *>(smem);
   for (int w = threadIdx.x; w < nwords; w += blockDim.x) dst[w] = src[w];
}

// one warp per contraction row; the kernel waits on chains of dependent loads, so 64 registers
// (32 warps per SM, a few spills) beat 80 (24 warps)
__global__ void __launch_bounds__(256, 4) k_group(DevCtx ctx, BatchArgs bt, int warp_doubles, int use_global) {
   extern __shared__ __align__(16) double smem[];
   const ClassPlan *pl = reinterpret_cast<const ClassPlan *>(smem);
   load_plan(bt.plan, smem);
   __syncthreads();
   const int plan_doubles = (int)((sizeof(ClassPlan) + 15) / 16) * 2;
   const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nwarp = blockDim.x / 32;
   const int gwarp = blockIdx.x * nwarp + warp;
   // shared memory: plan | nwarp coefficient buffers | nwarp workspaces (unless in global memory)
   double *kpw = smem + plan_doubles + warp * kGroupKpDoubles;
   double *wbase = use_global ? (bt.gscratch + (size_t)gwarp * warp_doubles)
                              : (smem + plan_doubles + nwarp * kGroupKpDoubles + (size_t)warp * warp_doubles);
   const int Hws = max(pl->H, 2 * pl->Nc);
   const uint2 *hrec = ctx.gprog + ctx.gprog[bt.cls].x;
   ShellShared *cache = reinterpret_cast<ShellShared *>(kpw + 32);
   if (lane == 0) cache->key = ~0u;
   __syncwarp();
   // kGroupRowsPerWarp consecutive rows at a time, so that the rows of one set quartet that follow
   // each other on this warp reuse its group record and shell 0's shared data
   uint32_t gi = 0, gend = 0;
   GroupRec G = {};
   for (uint32_t q0 = gwarp * kGroupRowsPerWarp; q0 < bt.nqrtt; q0 += gridDim.x * nwarp * kGroupRowsPerWarp) {
      const uint32_t q1 = min(q0 + kGroupRowsPerWarp, bt.nqrtt);
      for (uint32_t q = q0; q < q1; q++) {
         if (q >= gend || q < G.qrtt_off) {
            gi = row_group_one(bt, q, lane);
            G = bt.groups[gi];
            gend = G.qrtt_off + (uint32_t)G.nl[0] * G.nl[1] * G.nl[2] * G.nl[3];
         }
         if (bt.gflags && !__ldg(bt.gflags + gi)) continue;   // screened on an incremental replay
         group_body<32, 1>(ctx, bt, pl, G, q, wbase, wbase + Hws, lane, hrec, kpw, cache, gi);
      }
   }
}

// one block of NT threads per contraction row, all of them on one workspace (in shared memory, or
// for the largest classes a slice of the global scratch per block): for the classes whose rows are
// long chains of HRR levels with hundreds to thousands of elements each and which have few rows,
// a warp per row leaves the GPU mostly idle and takes a level in many rounds. NT = 128 (eight
// blocks per SM at 64 registers) up to kGroupBlockWideDoubles of workspace, 256 above.
template <int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_group_block(DevCtx ctx, BatchArgs bt, int ws_doubles,
                                                                int use_global) {
   extern __shared__ __align__(16) double smem[];
   const ClassPlan *pl = reinterpret_cast<const ClassPlan *>(smem);
   load_plan(bt.plan, smem);
   __syncthreads();
   const int plan_doubles = (int)((sizeof(ClassPlan) + 15) / 16) * 2;
   double *kpw = smem + plan_doubles;
   double *ws = use_global ? bt.gscratch + (size_t)blockIdx.x * ws_doubles : kpw + kGroupKpDoubles;
   const int Hws = max(pl->H, 2 * pl->Nc);
   const uint2 *hrec = ctx.gprog + ctx.gprog[bt.cls].x;
   const int lane = threadIdx.x & 31;
   for (uint32_t q = blockIdx.x; q < bt.nqrtt; q += gridDim.x) {
      const uint32_t gi = row_group_one(bt, q, lane);   // the same in every warp of the block
      if (bt.gflags && !__ldg(bt.gflags + gi)) continue;   // screened on an incremental replay
      const GroupRec G = bt.groups[gi];
      group_body<NT, 1>(ctx, bt, pl, G, q, ws, ws + Hws, (int)threadIdx.x, hrec, kpw);
   }
}

// one lane per contraction row, for classes with a small workspace (lane-interleaved in shared memory)
__global__ void __launch_bounds__(256) k_group_lane(DevCtx ctx, BatchArgs bt, int lane_doubles) {
   extern __shared__ __align__(16) double smem[];
   const ClassPlan *pl = reinterpret_cast<const ClassPlan *>(smem);
   load_plan(bt.plan, smem);
   __syncthreads();
   const int plan_doubles = (int)((sizeof(ClassPlan) + 15) / 16) * 2;
   const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nwarp = blockDim.x / 32;
   double *wbase = smem + plan_doubles + (size_t)warp * 32 * lane_doubles + lane;
   const int Hws = max(pl->H, 2 * pl->Nc);
   const uint2 *hrec = ctx.gprog + ctx.gprog[bt.cls].x;
   const uint32_t nblk = (bt.nqrtt + 31) >> 5;
   for (uint32_t blk = blockIdx.x * nwarp + warp; blk < nblk; blk += gridDim.x * nwarp) {
      const uint32_t q0 = blk << 5, q = q0 + lane;
      const uint32_t gi = row_group_warp(bt, q0, lane);
      if (q >= bt.nqrtt || (bt.gflags && !__ldg(bt.gflags + gi))) continue;
      const GroupRec G = bt.groups[gi];
      group_body<1, 32>(ctx, bt, pl, G, q, wbase, wbase + Hws * 32, 0, hrec, nullptr);
   }
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
static int h_ncart(int l) { return (l + 1) * (l + 2) / 2; }
static int h_cidx(int x, int y, int z) { int a = y + z; return a * (a + 1) / 2 + z; }

// Cartesian index tables for l < 8: exponents, the first axis with a nonzero exponent, and the
// index of the function one lower / one higher on each axis (-1 where that does not exist).
struct CartTables {
   int8_t exp_[8][36][3], dir[8][36], dec[8][36][3], inc[8][36][3];
};

static void make_cart_tables(CartTables &t) {
   std::memset(&t, 0, sizeof(t));
   for (int l = 0; l < 8; l++) for (int i = 0; i < 36; i++) for (int q = 0; q < 3; q++) { t.dec[l][i][q] = -1; t.inc[l][i][q] = -1; }
   for (int l = 0; l < 8; l++) {
      for (int i = 0; i < h_ncart(l); i++) {
         int a = 0; while ((a + 1) * (a + 2) / 2 <= i) a++;
         int e[3]; e[0] = l - a; e[2] = i - a * (a + 1) / 2; e[1] = a - e[2];
         for (int q = 0; q < 3; q++) t.exp_[l][i][q] = (int8_t)e[q];
         t.dir[l][i] = (int8_t)(e[0] ? 0 : (e[1] ? 1 : 2));
         for (int q = 0; q < 3; q++) {
            int f[3] = {e[0], e[1], e[2]};
            if (f[q] > 0) { f[q]--; t.dec[l][i][q] = (int8_t)h_cidx(f[0], f[1], f[2]); }
            int g[3] = {e[0], e[1], e[2]};
            g[q]++;
            if (l + 1 < 8) t.inc[l][i][q] = (int8_t)h_cidx(g[0], g[1], g[2]);
         }
      }
   }
}

// The HRR instructions of all 256 classes (layout in kernels.h). Element e of a ket step (c, d)
// is (ie, k, l) = (e / (nc nd), e / nd % nc, e % nd) and reads (ie, k + 1_t, l - 1_t) and
// (ie, k, l - 1_t); element e of a bra step (a, b) is (i, j, q) and reads (i + 1_t, j - 1_t, q)
// and (i, j - 1_t, q), t the first axis on which l (or j) has a nonzero exponent (reference
// src/compute_HRR.cpp:7-99). The steps' outputs are laid out back to back from S, so element x
// of the workspace is instruction x - S.
void build_group_prog(std::vector<uint2> &out) {
   CartTables t;
   make_cart_tables(t);
   out.assign(256, make_uint2(0u, 0u));
   for (int c = 0; c < 256; c++) {
      ClassPlan p;
      out[c].x = (uint32_t)out.size();
      if (!build_class_plan(c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3, p)) continue;
      int x = p.S;
      for (int o = 0; o < p.nhop; o++) {
         const HOp &h = p.hop[o];
         if (h.out != x) { out.clear(); return; }   // steps not back to back: no program
         if (h.type == 0) {
            const int cc = h.x, d = h.y, nc = h_ncart(cc), nd = h_ncart(d), ncp = h_ncart(cc + 1), ndm = h_ncart(d - 1);
            for (int e = 0; e < h.nelem; e++) {
               const int l = e % nd, k = (e / nd) % nc, ie = e / (nd * nc);
               const int dr = t.dir[d][l], lm = t.dec[d][l][dr], kp = t.inc[cc][k][dr];
               const uint32_t in1 = (uint32_t)(h.in1 + (ie * ncp + kp) * ndm + lm);
               const uint32_t in2 = (uint32_t)(h.in2 + (ie * nc + k) * ndm + lm);
               out.push_back(make_uint2(in1 | ((uint32_t)dr << 30), in2));
            }
         } else {
            const int a = h.x, b = h.y, nb = h_ncart(b), nbm = h_ncart(b - 1);
            const int cdn = h_ncart(p.lc) * h_ncart(p.ld);
            for (int e = 0; e < h.nelem; e++) {
               const int q = e % cdn, j = (e / cdn) % nb, i = e / (cdn * nb);
               const int dr = t.dir[b][j], jm = t.dec[b][j][dr], ip = t.inc[a][i][dr];
               const uint32_t in1 = (uint32_t)(h.in1 + (ip * nbm + jm) * cdn + q);
               const uint32_t in2 = (uint32_t)(h.in2 + (i * nbm + jm) * cdn + q);
               out.push_back(make_uint2(in1 | ((uint32_t)dr << 30), in2));
            }
         }
         x += h.nelem;
      }
   }
}

cudaError_t upload_constant_tables(const double *c2s_l0to3, const double *symm5) {
   // the spherical passes leave out the terms outside the rows' nonzero pattern (c2s_mask)
   for (int l = 0; l <= 3; l++) {
      const int nk = h_ncart(l);
      for (int m = 0; m < 2 * l + 1; m++)
         for (int k = 0; k < nk; k++)
            if (((c2s_mask(l, m) >> k & 1) != 0) != (c2s_l0to3[l * 70 + m * nk + k] != 0.0)) return cudaErrorInvalidValue;
   }
   CartTables t;
   make_cart_tables(t);
   cudaError_t err;
   if ((err = cudaMemcpyToSymbol(c_cart_exp, t.exp_, sizeof(t.exp_))) != cudaSuccess) return err;
   if ((err = cudaMemcpyToSymbol(c_cart_dir, t.dir, sizeof(t.dir))) != cudaSuccess) return err;
   if ((err = cudaMemcpyToSymbol(c_cart_dec, t.dec, sizeof(t.dec))) != cudaSuccess) return err;
   if ((err = cudaMemcpyToSymbol(c_cart_inc, t.inc, sizeof(t.inc))) != cudaSuccess) return err;
   if ((err = cudaMemcpyToSymbol(c_c2s, c2s_l0to3, sizeof(double) * 4 * 70)) != cudaSuccess) return err;
   return cudaMemcpyToSymbol(c_symm, symm5, sizeof(double) * 5);
}

int plan_smem_doubles() { return (int)((sizeof(ClassPlan) + 15) / 16) * 2; }

// the opt-in shared memory per block of the first device asked (the engine's GPUs are all one
// type); a function-local static, so concurrent caller threads initialise it once
static int max_dyn_smem() {
   static const int smax = [] {
      int dev = 0, v = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
      return v > 0 ? v : 48 * 1024;
   }();
   return smax;
}

template <int TS>
static cudaError_t launch_prim_t(const DevCtx &ctx, const BatchArgs &bt, const ClassPlan &hp, cudaStream_t st) {
   const int L = hp.L;
   int team_doubles = hp.V + 1 + hp.S + 17 + TS * (L + 1);
   team_doubles = (team_doubles + 1) & ~1;
   const int budget = std::min(max_dyn_smem(), 200 * 1024);
   const size_t plan_bytes = (size_t)plan_smem_doubles() * 8;
   int teams = (int)((budget - (int)plan_bytes) / ((size_t)team_doubles * 8));
   teams = std::min(teams, 256 / TS);
   if (teams < 1) return cudaErrorInvalidConfiguration;
   const size_t smem = plan_bytes + (size_t)teams * team_doubles * 8;
   long blocks = ((long)bt.nprm + teams - 1) / teams;
   blocks = std::max(1L, std::min(blocks, 148L * 64));
   k_prim<TS><<<(unsigned)blocks, teams * TS, smem, st>>>(ctx, bt, team_doubles);
   return cudaGetLastError();
}

int prim_team_size(const ClassPlan &hp) {
   const int w = hp.V + hp.S;
   if (w <= 40) return 1;
   if (w <= 300) return 4;
   if (w <= 1200) return 8;
   return 32;
}

// k_prim2 launch shape: primitives per warp chunk and the per-warp shared-memory size. The chunk's
// image-summed targets (cp x S doubles) are the largest part of a warp's shared memory, and
// shared memory bounds the warps per SM of the large classes, so a chunk holds about 512 targets.
static void prim2_shape(const ClassPlan &hp, bool lane_vrr, int *cp, size_t *warp_doubles) {
   int c = std::max(1, std::min(32, 512 / std::max(1, hp.S)));
   const size_t geo = (sizeof(PrimGeo) / 8);
   size_t w = geo * c + c + (size_t)c * hp.S + 32 + 64 + 32 + 64 * (size_t)(hp.L + 1) +
              (lane_vrr ? 17 * 32 + 32 * (size_t)hp.V : 18 + (size_t)hp.V + 2);
   *cp = c;
   *warp_doubles = (w + 1) & ~(size_t)1;
}

static bool prim2_lane(const ClassPlan &hp) { return hp.V <= 96; }


// Primitive-kernel choice: k_prim3 (generated VRR) for the classes it covers, then k_prim2,
// then the team kernel for the largest classes.
cudaError_t launch_prim(const DevCtx &ctx, const BatchArgs &bt, const ClassPlan &hp, cudaStream_t st) {
   if (bt.nprm == 0) return cudaSuccess;
   if (bt.prim_variant == 0 || bt.fp32) {
      cudaError_t err = cudaSuccess;
      if (prim3_launch(ctx, bt, st, &err)) return err;
   }
   if (bt.fp32) return cudaErrorInvalidValue;   // FP32 segments exist only for classes with k_prim3
   {
      const bool lane = prim2_lane(hp);
      int cp = 1;
      size_t wd = 0;
      prim2_shape(hp, lane, &cp, &wd);
      const int budget = std::min(max_dyn_smem(), 200 * 1024);
      const size_t plan_bytes = (size_t)plan_smem_doubles() * 8;
      int nw = (int)((budget - (int)plan_bytes) / (wd * 8));
      nw = std::min(nw, 8);
      if (nw >= 1) {
         const size_t smem = plan_bytes + (size_t)nw * wd * 8;
         const long nchunk = ((long)bt.nprm + cp - 1) / cp;
         long blocks = std::max(1L, std::min((nchunk + nw - 1) / nw, 148L * 32));
         if (lane) {
            k_prim2<true><<<(unsigned)blocks, nw * 32, smem, st>>>(ctx, bt, cp, (int)wd);
         } else {
            k_prim2<false><<<(unsigned)blocks, nw * 32, smem, st>>>(ctx, bt, cp, (int)wd);
         }
         return cudaGetLastError();
      }
      // the largest classes fall through to the team kernel
   }
   switch (prim_team_size(hp)) {
      case 1: return launch_prim_t<1>(ctx, bt, hp, st);
      case 4: return launch_prim_t<4>(ctx, bt, hp, st);
      case 8: return launch_prim_t<8>(ctx, bt, hp, st);
      default: return launch_prim_t<32>(ctx, bt, hp, st);
   }
}

size_t group_warp_doubles(const ClassPlan &hp) {
   size_t d = (size_t)std::max(hp.H, 2 * hp.Nc) + hp.Nc;
   return (d + 1) & ~(size_t)1;
}

// returns the number of global-scratch doubles needed (0 if the shared-memory path is used)
// shared memory ahead of the group kernels' workspaces: the class plan
static size_t group_hdr_bytes() { return (size_t)plan_smem_doubles() * 8; }

// warps per block of k_group with the workspaces in shared memory (0: they do not fit)
static int group_smem_warps(size_t wd) {
   const int budget = std::min(max_dyn_smem(), 200 * 1024) - (int)group_hdr_bytes();
   return std::min(8, (int)(budget / ((wd + kGroupKpDoubles) * 8)));
}

size_t group_global_scratch(const ClassPlan &hp, int *grid, int *warps) {
   const size_t wd = group_warp_doubles(hp);
   if (group_smem_warps(wd) >= 1) return 0;
   *warps = 4;
   *grid = 148 * 2;
   return wd * (size_t)(*warps) * (*grid);
}


// Group-kernel choice: k_group3 (generated HRR, one lane per row) for the classes it covers; for
// the others on variant 0 k_group_block (one block per row) where the workspace is large and fits
// a block's shared memory, k_group_lane for small workspaces, else k_group (one warp per row),
// which variant 1 always takes.
cudaError_t launch_group(const DevCtx &ctx, const BatchArgs &bt, const ClassPlan &hp, cudaStream_t st) {
   if (bt.nqrtt == 0) return cudaSuccess;
   if (bt.group_variant == 0 || bt.fp32) {
      cudaError_t err = cudaSuccess;
      if (group3_launch(ctx, bt, st, &err)) return err;
   }
   if (bt.fp32) return cudaErrorInvalidValue;   // FP32 segments exist only for classes with k_group3
   const size_t wd = group_warp_doubles(hp);
   if (bt.group_variant == 0 && wd >= (size_t)kGroupBlockMinDoubles) {
      const bool wide = wd >= (size_t)kGroupBlockWideDoubles;
      const size_t smem = group_hdr_bytes() + (kGroupKpDoubles + wd) * 8;
      long blocks = 0;
      int use_global = 0;
      size_t dyn = smem;
      if (smem <= (size_t)std::min(max_dyn_smem(), 200 * 1024)) {
         blocks = std::max(1L, std::min((long)bt.nqrtt, 148L * 16));
      } else if (bt.gscratch) {   // workspace in the global scratch, which holds group_global_scratch's count
         int grid = 0, warps = 0;
         group_global_scratch(hp, &grid, &warps);
         blocks = std::max(1L, std::min((long)bt.nqrtt, (long)grid * warps));
         use_global = 1;
         dyn = group_hdr_bytes() + kGroupKpDoubles * 8;
      }
      if (blocks) {
         if (wide) k_group_block<256><<<(unsigned)blocks, 256, dyn, st>>>(ctx, bt, (int)wd, use_global);
         else k_group_block<128><<<(unsigned)blocks, 128, dyn, st>>>(ctx, bt, (int)wd, use_global);
         return cudaGetLastError();
      }
   }
   if (wd <= 40 && bt.group_variant == 0) {
      // small workspace: one lane per group, 32 groups per warp
      const int lane_doubles = (int)wd;
      const size_t plan_bytes = group_hdr_bytes();
      const int nw = 8;
      const size_t smem = plan_bytes + (size_t)nw * 32 * lane_doubles * 8;
      long blocks = ((long)bt.nqrtt + nw * 32 - 1) / (nw * 32);
      blocks = std::max(1L, std::min(blocks, 148L * 16));
      k_group_lane<<<(unsigned)blocks, nw * 32, smem, st>>>(ctx, bt, lane_doubles);
      return cudaGetLastError();
   }
   const size_t plan_bytes = group_hdr_bytes();
   const int nw = group_smem_warps(wd);
   if (nw >= 1) {
      const size_t smem = plan_bytes + (size_t)nw * (wd + kGroupKpDoubles) * 8;
      long blocks = ((long)bt.nqrtt + (long)nw * kGroupRowsPerWarp - 1) / ((long)nw * kGroupRowsPerWarp);
      blocks = std::max(1L, std::min(blocks, 148L * 64));
      k_group<<<(unsigned)blocks, nw * 32, smem, st>>>(ctx, bt, (int)wd, 0);
   } else {
      int grid = 0, warps = 0;
      group_global_scratch(hp, &grid, &warps);
      const size_t smem = plan_bytes + (size_t)warps * kGroupKpDoubles * 8;
      k_group<<<grid, warps * 32, smem, st>>>(ctx, bt, (int)wd, 1);
   }
   return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------
// Incremental replays. k_group_screen, one thread per group:
//  mode 0 (after a recording): the exact largest |P| over the P elements its rows' K updates read
//    (blocks ac: nsa x nsc, ad: nsa x nsd, bc: nsb x nsc, bd: nsb x nsd, with each row's offsets,
//    leading dimensions and transposition flags), stored in pmax;
//  mode 1 (P = dP): an upper bound of max|dP| over the same elements, from the maxima of 32-element
//    tiles of |dP| (k_tile_max) over the span of offsets each block's rows cover, and the group kept
//    unless that bound is zero or its bound scaled by it / pmax is below eps. The span bound never
//    underestimates, so no group that the exact test keeps is skipped.
// ---------------------------------------------------------------------------------------
constexpr int kScreenTile = 32;

__global__ void k_tile_max(const double *__restrict__ P, size_t n, float *__restrict__ tmax) {
   const size_t ntile = (n + kScreenTile - 1) / kScreenTile;
   const int lane = threadIdx.x & 31;
   for (size_t t = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) / 32; t < ntile;
        t += (size_t)gridDim.x * blockDim.x / 32) {
      const size_t i = t * kScreenTile + lane;
      double m = i < n ? fabs(__ldg(P + i)) : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0) tmax[t] = (float)(m * (1.0 + 1e-6));   // rounded up: stays an upper bound
   }
}

__global__ void k_group_screen(DevCtx ctx, BatchArgs bt, float *pmax, uint8_t *flags, double eps, int mode,
                               const float *tmax) {
   const int la = bt.cls >> 6, lb = (bt.cls >> 4) & 3, lc = (bt.cls >> 2) & 3, ld = bt.cls & 3;
   const int ns[4] = {2 * la + 1, 2 * lb + 1, 2 * lc + 1, 2 * ld + 1};
   // block u of a row: rows of centre bra[u], columns of centre ket[u] (ac, ad, bc, bd)
   const int bra[4] = {0, 0, 1, 1}, ket[4] = {2, 3, 2, 3};
   const double *Pm = ctx.P[0];
   for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < bt.ngroup; g += gridDim.x * blockDim.x) {
      const GroupRec G = bt.groups[g];
      const int nrows = G.nl[0] * G.nl[1] * G.nl[2] * G.nl[3];
      double m = 0.0;
      if (mode == 0) {
         for (int r = 0; r < nrows; r++) {
            const QrttRec k = bt.qrtts[G.qrtt_off + r];
            for (int u = 0; u < 4; u++) {
               const bool T = (k.T >> u) & 1;
               for (int i = 0; i < ns[bra[u]]; i++)
                  for (int j = 0; j < ns[ket[u]]; j++) {
                     const size_t I = (size_t)k.off[u] + (T ? i * k.ld[u] + j : j * k.ld[u] + i);
                     if (I < ctx.FP_size) m = fmax(m, fabs(__ldg(Pm + I)));
                  }
            }
         }
         pmax[g] = (float)m;
         continue;
      }
      for (int u = 0; u < 4; u++) {
         size_t lo = ~(size_t)0, hi = 0;
         for (int r = 0; r < nrows; r++) {
            const QrttRec k = bt.qrtts[G.qrtt_off + r];
            const bool T = (k.T >> u) & 1;
            const int nr = ns[bra[u]], nc = ns[ket[u]];
            const size_t a = k.off[u];
            const size_t e = a + (T ? (size_t)(nr - 1) * k.ld[u] + nc : (size_t)(nc - 1) * k.ld[u] + nr);
            lo = min(lo, a);
            hi = max(hi, e);
         }
         hi = min(hi, ctx.FP_size);
         for (size_t t = lo / kScreenTile; lo < hi && t * kScreenTile < hi; t++) m = fmax(m, (double)__ldg(tmax + t));
      }
      const double b = (double)G.bound;
      const bool skip = m == 0.0 || (isfinite(b) && b * m < eps * (double)pmax[g]);
      flags[g] = skip ? 0 : 1;
   }
}

cudaError_t launch_tile_max(const double *P, size_t n, float *tmax, cudaStream_t st) {
   const size_t ntile = (n + kScreenTile - 1) / kScreenTile;
   const long blocks = std::max(1L, std::min((long)((ntile * 32 + 255) / 256), 148L * 32));
   k_tile_max<<<(unsigned)blocks, 256, 0, st>>>(P, n, tmax);
   return cudaGetLastError();
}

size_t tile_max_count(size_t n) { return (n + kScreenTile - 1) / kScreenTile; }

// ---------------------------------------------------------------------------------------
// Merging the recorded batches of one queue class into one segment (libgint_record(h, 2)): the
// parts are copied one after another, then the indices that count within a segment are shifted
// by the part's position in the merged segment, and the per-32-row group table is rebuilt.
// ---------------------------------------------------------------------------------------
__global__ void k_rebase_part(uint32_t *prm_shell, uint32_t nprm, ShellRec *shells, uint32_t nshell, GroupRec *groups,
                              uint32_t ngroup, uint32_t prm_base, uint32_t shell_base, uint32_t group_base,
                              uint32_t qrtt_base) {
   const uint32_t n = max(nprm, max(nshell, ngroup));
   for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      if (i < nprm) prm_shell[i] += shell_base;
      if (i < nshell) { shells[i].prm_off += prm_base; shells[i].group += group_base; }
      if (i < ngroup) { groups[i].shell_off += shell_base; groups[i].qrtt_off += qrtt_base; }
   }
}

__global__ void k_row_groups(const GroupRec *groups, uint32_t ngroup, uint32_t *rowgrp) {
   for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroup; g += gridDim.x * blockDim.x) {
      const GroupRec G = groups[g];
      const uint32_t end = G.qrtt_off + (uint32_t)G.nl[0] * G.nl[1] * G.nl[2] * G.nl[3];
      for (uint32_t k = (G.qrtt_off + 31) / 32; 32 * k < end; k++) rowgrp[k] = g;
   }
}

cudaError_t launch_rebase_part(uint32_t *prm_shell, uint32_t nprm, ShellRec *shells, uint32_t nshell, GroupRec *groups,
                               uint32_t ngroup, uint32_t prm_base, uint32_t shell_base, uint32_t group_base,
                               uint32_t qrtt_base, cudaStream_t st) {
   const uint32_t n = std::max(nprm, std::max(nshell, ngroup));
   if (n == 0) return cudaSuccess;
   const long blocks = std::max(1L, std::min((long)((n + 255) / 256), 148L * 16));
   k_rebase_part<<<(unsigned)blocks, 256, 0, st>>>(prm_shell, nprm, shells, nshell, groups, ngroup, prm_base,
                                                   shell_base, group_base, qrtt_base);
   return cudaGetLastError();
}

cudaError_t launch_row_groups(const GroupRec *groups, uint32_t ngroup, uint32_t *rowgrp, cudaStream_t st) {
   if (ngroup == 0) return cudaSuccess;
   const long blocks = std::max(1L, std::min((long)((ngroup + 255) / 256), 148L * 16));
   k_row_groups<<<(unsigned)blocks, 256, 0, st>>>(groups, ngroup, rowgrp);
   return cudaGetLastError();
}

cudaError_t launch_group_screen(const DevCtx &ctx, const BatchArgs &bt, float *pmax, uint8_t *flags, double eps,
                                int mode, const float *tmax, cudaStream_t st) {
   if (bt.ngroup == 0) return cudaSuccess;
   const int threads = 128;
   const long blocks = std::max(1L, std::min(((long)bt.ngroup + threads - 1) / threads, 148L * 16));
   k_group_screen<<<(unsigned)blocks, threads, 0, st>>>(ctx, bt, pmax, flags, eps, mode, tmax);
   return cudaGetLastError();
}

// Dependent FMA chains, 8 independent chains per thread: measures the FP64 FMA pipe rate.
__global__ void k_fp64_fma(double *out, int iters, double a, double b) {
   double x[8];
#pragma unroll
   for (int i = 0; i < 8; i++) x[i] = threadIdx.x * 1e-3 + i;
   for (int it = 0; it < iters; it++) {
#pragma unroll
      for (int i = 0; i < 8; i++) x[i] = fma(x[i], a, b);
   }
   double s = 0;
#pragma unroll
   for (int i = 0; i < 8; i++) s += x[i];
   if (s == 12345.678) out[0] = s;   // keeps the chains alive
}

double measure_fp64_peak_tflops() {
   int dev = 0, sms = 0;
   cudaGetDevice(&dev);
   cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
   double *d = nullptr;
   if (cudaMalloc(&d, 8) != cudaSuccess) return 0.0;
   const int iters = 4096, threads = 512, blocks = sms * 8;
   cudaEvent_t e0, e1;
   cudaEventCreate(&e0); cudaEventCreate(&e1);
   k_fp64_fma<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);   // warm-up
   float best = 1e30f;
   for (int rep = 0; rep < 5; rep++) {
      cudaEventRecord(e0);
      k_fp64_fma<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0; cudaEventElapsedTime(&ms, e0, e1);
      best = std::min(best, ms);
   }
   cudaEventDestroy(e0); cudaEventDestroy(e1);
   cudaFree(d);
   const double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
   return flops / (best * 1e-3) / 1e12;
}

// The per-device copies of the HRR instructions (build_group_prog), made once per device by
// preload_kernels and kept until the process exits.
static const uint2 *g_group_prog[kMaxDevices] = {nullptr};

static cudaError_t group_prog_load() {
   int dev = 0;
   cudaError_t e = cudaGetDevice(&dev);
   if (e != cudaSuccess) return e;
   if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
   if (g_group_prog[dev]) return cudaSuccess;
   std::vector<uint2> prog;
   build_group_prog(prog);
   if (prog.empty()) return cudaErrorInvalidValue;
   void *p = nullptr;
   if ((e = cudaMalloc(&p, prog.size() * sizeof(uint2))) != cudaSuccess) return e;
   if ((e = cudaMemcpy(p, prog.data(), prog.size() * sizeof(uint2), cudaMemcpyHostToDevice)) != cudaSuccess) {
      cudaFree(p);
      return e;
   }
   g_group_prog[dev] = (const uint2 *)p;
   return cudaSuccess;
}

const uint2 *group_prog(int device) {
   return (device >= 0 && device < kMaxDevices) ? g_group_prog[device] : nullptr;
}

// Loads every kernel of the engine on the current device and lets each take up to the device's
// opt-in shared memory per block. The shared-memory limit is a process-wide attribute of a
// kernel: set per launch (with the launch's own size), one caller thread could lower it between
// another thread's setting and launch, which failed that launch ("invalid argument"). It is
// therefore raised once, here, before any handle launches; launches pass only their own size.
cudaError_t preload_kernels() {
   cudaError_t e;
   const int smax = max_dyn_smem();
   const void *fns[] = {(const void *)k_prim<1>, (const void *)k_prim<4>, (const void *)k_prim<8>,
                        (const void *)k_prim<32>, (const void *)k_prim2<true>, (const void *)k_prim2<false>,
                        (const void *)k_group, (const void *)k_group_lane, (const void *)k_group_block<128>,
                        (const void *)k_group_block<256>};
   for (const void *f : fns)
      if ((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smax)) != cudaSuccess) return e;
   cudaFuncAttributes a;
   if ((e = cudaFuncGetAttributes(&a, (const void *)k_fp64_fma)) != cudaSuccess) return e;
   if ((e = cudaFuncGetAttributes(&a, (const void *)k_rebase_part)) != cudaSuccess) return e;
   if ((e = cudaFuncGetAttributes(&a, (const void *)k_row_groups)) != cudaSuccess) return e;
   if ((e = prim3_preload(smax)) != cudaSuccess) return e;
   if ((e = group3_preload()) != cudaSuccess) return e;
   return group_prog_load();
}

// ---------------------------------------------------------------------------------------
// Fixed device scratch for libgint_replay_noalloc. Callers that cannot allocate device
// memory at K-build time (a framework that owns every device byte through its own pool, or
// code that must not trigger the implicit synchronisation of cudaMalloc/cudaFree) use this
// array instead of the handle's allocated AC/HRR buffers. It is a file-scope device array of
// kNoAllocScratchDoubles doubles (64 MiB) that every GPU which loads the library holds until
// the process exits. Host code cannot use the name g_noalloc_scratch as a device address; the
// address is obtained once per device with cudaGetSymbolAddress, with that device current.
// ---------------------------------------------------------------------------------------
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

cudaError_t noalloc_scratch(double **ptr) {
   static std::mutex mu;
   static double *addr[kMaxDevices] = {nullptr};
   int dev = 0;
   cudaError_t e = cudaGetDevice(&dev);
   if (e != cudaSuccess) return e;
   if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
   std::lock_guard<std::mutex> lock(mu);
   if (!addr[dev]) {
      double *p = nullptr;
      e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
      if (e != cudaSuccess) return e;
      addr[dev] = p;
   }
   *ptr = addr[dev];
   return cudaSuccess;
}

}  // namespace gint
