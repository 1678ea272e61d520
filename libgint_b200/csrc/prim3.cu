// prim3.cu -- k_prim3<la,lb,lc,ld>: Fm + VRR + sum over the third image for the classes whose
// VRR is generated as straight-line code (vrr_gen.cuh).
//
// One warp owns a chunk of CP primitive quartets (reference src/compute_Fm.cpp:20-326,
// src/compute_VRR.cpp:349-458, src/compute_ECO.cpp:216-272):
//  1. lane per primitive: the geometry (P, Q, the minimum-image shift, Kfac, R) into shared;
//  2. lane per (primitive, image) pair: the truncation test T <= R^2 + 11 R + 50; passing
//     pairs are compacted into a queue;
//  3. lane per queued pair: G_m (Chebyshev patch series or Boys); pairs with Fm[0] > 1e-12 are
//     compacted into a second queue; when la = lc = 0 every pair's Fm[0] goes to the (00|00)
//     target, screened or not, as in the reference;
//  4. lane per surviving pair: the generated VRR, entirely in registers. Both queues keep the
//     pairs in primitive order, so pairs of one primitive sit in adjacent lanes; each target is
//     summed over them by a segmented shuffle reduction and added to the primitive's row of the
//     warp's shared accumulator by the segment's first lane (no atomics).
// The chunk's image-summed targets are then stored to AC.
//
// Compiled kPrim3Parts times (PRIM3_PART = 0..7); part i instantiates the generated classes
// whose position in kVrrGenClasses is i modulo kPrim3Parts.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include "engine_types.h"
#include "kernels.h"
#include "prim3.h"
#include "prim_common.cuh"
#include "vrr_gen.cuh"

#ifndef PRIM3_PART
#define PRIM3_PART 0
#endif

namespace gint {
namespace {

constexpr unsigned kFull = 0xffffffffu;

template <int LA, int LB, int LC, int LD>
struct Prim3Shape {
   using G = VrrGen<LA, LB, LC, LD>;
   static constexpr int L = LA + LB + LC + LD, LF = L + 1, S = G::S;
   static constexpr bool NEED_VRR = G::nout > 0;
   // primitives per warp chunk: the largest power of two <= 2048 / S (at most 32), so the shared
   // accumulator stays near 16 KB per warp
   static constexpr int CP = S <= 64 ? 32 : (S <= 128 ? 16 : (S <= 256 ? 8 : (S <= 512 ? 4 : (S <= 1024 ? 2 : 1))));
   static constexpr int PG = (int)(sizeof(PrimGeo) / 8);
   // per warp, in doubles: geometry, accumulator, queue-1 T and indices, queue-2 Fm and indices
   static constexpr int WD = CP * PG + CP * S + 64 + 32 + (NEED_VRR ? 64 * LF + 32 : 0);
   // resident blocks per SM the register budget is sized for (small classes need few registers)
   static constexpr int MINB = L <= 1 ? 3 : (L <= 3 ? 2 : 1);
   static constexpr int THREADS = MINB == 3 ? 192 : 256;
};

// Segmented sum over adjacent lanes that carry the same key (keys are contiguous runs); the
// first lane of each run adds the run's sum to dst[s]. R = double, or float on the FP32 path.
template <class R>
struct SegSum {
   unsigned same;   // bit o: lane + 2^o carries this lane's key
   bool head;
   R *dst;
   __device__ __forceinline__ void operator()(int s, R v) {
#pragma unroll
      for (int o = 0; o < 5; o++) {
         const R u = __shfl_down_sync(kFull, v, 1 << o);
         if (same & (1u << o)) v += u;
      }
      if (head) dst[s] += v;
   }
};

template <class R>
static __device__ __forceinline__ SegSum<R> make_segsum(int key, int lane, R *dst) {
   SegSum<R> sg;
   sg.same = 0;
#pragma unroll
   for (int o = 0; o < 5; o++) {
      const int k2 = __shfl_down_sync(kFull, key, 1 << o);
      if (lane + (1 << o) < 32 && k2 == key) sg.same |= 1u << o;
   }
   const int kp = __shfl_up_sync(kFull, key, 1);
   sg.head = key >= 0 && (lane == 0 || kp != key);
   sg.dst = dst;
   return sg;
}

// R = double: the FP64 path; R = float: the FP32 path (G_m series, VRR, image sum and the stored
// targets in FP32; the geometry and every screening decision in FP64 as on the FP64 path).
template <int LA, int LB, int LC, int LD, class R>
__global__ void __launch_bounds__(Prim3Shape<LA, LB, LC, LD>::THREADS, Prim3Shape<LA, LB, LC, LD>::MINB)
k_prim3(DevCtx ctx, BatchArgs bt) {
   using Sh = Prim3Shape<LA, LB, LC, LD>;
   using G = typename Sh::G;
   constexpr int L = Sh::L, LF = Sh::LF, S = Sh::S, CP = Sh::CP;
   constexpr bool W00 = (LA == 0 && LC == 0);
   constexpr bool NEED_VRR = Sh::NEED_VRR;
   extern __shared__ __align__(16) double smem[];
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
   const int Ng = ctx.Ng;
   // the image vectors, shared by the block
   double *sneigh = smem;
   for (int i = threadIdx.x; i < 3 * Ng; i += blockDim.x) sneigh[i] = __ldg(ctx.neighs + i);
   __syncthreads();
   double *wbase = smem + ((3 * Ng + 1) & ~1) + (size_t)warp * Sh::WD;
   PrimGeo *geo = reinterpret_cast<PrimGeo *>(wbase);
   R *acc = reinterpret_cast<R *>(wbase + CP * Sh::PG);
   double *q1t = wbase + CP * Sh::PG + CP * S;
   int *q1i = reinterpret_cast<int *>(q1t + 64);
   R *q2f = reinterpret_cast<R *>(q1t + 64 + 32);
   int *q2i = reinterpret_cast<int *>(q1t + 64 + 32 + 64 * LF);
   // pair numbering within a chunk: pair = p * Ng + n3; each round of 32 pairs advances a lane
   // by 32 = adv_p * Ng + adv_n
   const int adv_p = 32 / Ng, adv_n = 32 - adv_p * Ng;
   const unsigned below = (1u << lane) - 1u;
   unsigned long long c_cheb = 0, c_boys = 0, c_vrr = 0;

   const uint32_t nchunk = (bt.nprm + CP - 1) / CP;
   for (uint32_t ch = blockIdx.x * nwarp + warp; ch < nchunk; ch += gridDim.x * nwarp) {
      const uint32_t p0 = ch * CP;
      const int np = (int)min((uint32_t)CP, bt.nprm - p0);
      if (lane < np) {
         PrimGeo g;
         const ShellRec sh = bt.shells[bt.prm_shell[p0 + lane]];
         prim_geometry(ctx, sh, bt.prm[p0 + lane], g);
         kill_if_screened(bt, sh, g);
         geo[lane] = g;
      }
      for (int j = lane; j < CP * S; j += 32) acc[j] = R(0);
      __syncwarp();

      int n1 = 0, n2 = 0;
      // stage 4: VRR of queued survivors [0, cnt), one per lane
      auto run_vrr = [&](int cnt) {
         const bool act = lane < cnt;
         const int pk = act ? q2i[lane] : 0;
         const int p = pk >> 8, n3 = pk & 255;
         const PrimGeo &g = geo[p];
         R z[17], F[LF];
#pragma unroll
         for (int q = 0; q < 3; q++) {
            const double Qp = g.Q[q] + sneigh[n3 * 3 + q];
            const double W = wdist(g.zab, g.P[q], g.zcd, Qp, g.inv_z);
            z[q] = (R)g.PA[q];
            z[3 + q] = (R)(W - g.P[q]);
            z[6 + q] = (R)g.QC[q];
            z[9 + q] = (R)(W - Qp);
         }
         z[12] = (R)g.i2ab; z[13] = (R)g.mrab; z[14] = (R)g.i2cd; z[15] = (R)g.mrcd; z[16] = (R)g.i2z;
#pragma unroll
         for (int m = 0; m < LF; m++) F[m] = act ? q2f[lane * LF + m] : R(0);
         SegSum<R> sg = make_segsum<R>(act ? p : -1 - lane, lane, acc + p * S);
         G::run(F, z, sg);
         c_vrr += (lane == 0) ? (unsigned)cnt : 0u;
         __syncwarp();
      };
      // stage 3: G_m of queued pairs [0, cnt), one per lane
      auto run_fm = [&](int cnt) {
         const bool act = lane < cnt;
         const int pk = act ? q1i[lane] : 0;
         const int p = pk >> 8;
         R fm[LF];
         bool surv = false;
         if (act) {
            int br;
            if constexpr (sizeof(R) == sizeof(double)) br = fm_eval_geo<L>(ctx, L, geo[p], q1t[lane], fm);
            else br = fm_eval_geo_f<L>(ctx, L, geo[p], q1t[lane], fm);
            c_cheb += (br == 1);
            c_boys += (br == 2);
            surv = NEED_VRR && (fm[0] > R(1.e-12));
         } else {
#pragma unroll
            for (int m = 0; m < LF; m++) fm[m] = R(0);
         }
         if (W00) {
            SegSum<R> sg = make_segsum<R>(act ? p : -1 - lane, lane, acc + p * S);
            sg(G::s00, fm[0]);
            __syncwarp();
         }
         if (NEED_VRR) {
            const unsigned bal = __ballot_sync(kFull, surv);
            if (surv) {
               const int pos = n2 + __popc(bal & below);
               q2i[pos] = pk;
#pragma unroll
               for (int m = 0; m < LF; m++) q2f[pos * LF + m] = fm[m];
            }
            n2 += __popc(bal);
            __syncwarp();
            if (n2 >= 32) {
               run_vrr(32);
               const int rem = n2 - 32;
               int v = 0;
               R tmp[LF];
               if (lane < rem) {
                  v = q2i[32 + lane];
#pragma unroll
                  for (int m = 0; m < LF; m++) tmp[m] = q2f[(32 + lane) * LF + m];
               }
               __syncwarp();
               if (lane < rem) {
                  q2i[lane] = v;
#pragma unroll
                  for (int m = 0; m < LF; m++) q2f[lane * LF + m] = tmp[m];
               }
               __syncwarp();
               n2 = rem;
            }
         }
      };
      // stage 2: truncation test over every (primitive, image) pair of the chunk
      const int npair = np * Ng;
      int tp = lane / Ng, tn = lane - (lane / Ng) * Ng;
      for (int b0 = 0; b0 < npair; b0 += 32) {
         bool pass = false;
         double T = 0.0;
         if (b0 + lane < npair) {
            const PrimGeo &g = geo[tp];
            const double d0 = rsub(g.D[0], sneigh[tn * 3 + 0]);
            const double d1 = rsub(g.D[1], sneigh[tn * 3 + 1]);
            const double d2 = rsub(g.D[2], sneigh[tn * 3 + 2]);
            T = rmul(g.rho, rdot3(d0, d0, d1, d1, d2, d2));
            pass = !(T > g.upper);
         }
         const unsigned bal = __ballot_sync(kFull, pass);
         if (pass) {
            const int pos = n1 + __popc(bal & below);
            q1i[pos] = (tp << 8) | tn;
            q1t[pos] = T;
         }
         n1 += __popc(bal);
         tp += adv_p;
         tn += adv_n;
         if (tn >= Ng) { tn -= Ng; tp++; }
         __syncwarp();
         if (n1 >= 32) {
            run_fm(32);
            const int rem = n1 - 32;
            int vi = 0;
            double vt = 0.0;
            if (lane < rem) { vi = q1i[32 + lane]; vt = q1t[32 + lane]; }
            __syncwarp();
            if (lane < rem) { q1i[lane] = vi; q1t[lane] = vt; }
            __syncwarp();
            n1 = rem;
         }
      }
      if (n1 > 0) run_fm(n1);
      if (NEED_VRR && n2 > 0) run_vrr(n2);
      __syncwarp();
      if (lane == 0 && ctx.cnt) atomicAdd(ctx.cnt + bt.cls * 4 + 3, (unsigned long long)np);
      R *out = reinterpret_cast<R *>(bt.AC) + (size_t)p0 * S;
      for (int j = lane; j < np * S; j += 32) out[j] = acc[j];
      __syncwarp();
   }
   if (ctx.cnt) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
         c_cheb += __shfl_down_sync(kFull, c_cheb, o);
         c_boys += __shfl_down_sync(kFull, c_boys, o);
      }
      if (lane == 0) {
         atomicAdd(ctx.cnt + bt.cls * 4 + 0, c_cheb);
         atomicAdd(ctx.cnt + bt.cls * 4 + 1, c_boys);
         atomicAdd(ctx.cnt + bt.cls * 4 + 2, c_vrr);
      }
   }
}

template <int LA, int LB, int LC, int LD, class R>
cudaError_t launch_one(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st) {
   using Sh = Prim3Shape<LA, LB, LC, LD>;
   const size_t warp_bytes = (size_t)Sh::WD * 8;
   const size_t neigh_bytes = (size_t)((3 * ctx.Ng + 1) & ~1) * 8;
   // shared memory per block sized so that MINB blocks share an SM
   const size_t budget = (220 * 1024) / Sh::MINB;
   const int maxw = Sh::THREADS / 32;
   const int nw = (int)std::max<size_t>(1, std::min<size_t>(maxw, (budget - std::min(budget, neigh_bytes)) / warp_bytes));
   const size_t smem = neigh_bytes + warp_bytes * nw;
   const long nchunk = ((long)bt.nprm + Sh::CP - 1) / Sh::CP;
   const long blocks = std::max(1L, std::min((nchunk + nw - 1) / nw, 148L * 24));
   k_prim3<LA, LB, LC, LD, R><<<(unsigned)blocks, nw * 32, smem, st>>>(ctx, bt);
   return cudaGetLastError();
}

template <int I>
struct PartTable {
   static bool launch(int cls, const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err) {
      if constexpr (I >= kVrrGenCount) {
         return false;
      } else {
         constexpr int c = kVrrGenClasses[I];
         if (cls == c) {
            if (!bt.fp32) {
               *err = launch_one<(c >> 6) & 3, (c >> 4) & 3, (c >> 2) & 3, c & 3, double>(ctx, bt, st);
            } else if constexpr (class_has_fp32((c >> 6) & 3, (c >> 4) & 3, (c >> 2) & 3, c & 3)) {
               *err = launch_one<(c >> 6) & 3, (c >> 4) & 3, (c >> 2) & 3, c & 3, float>(ctx, bt, st);
            } else {
               *err = cudaErrorInvalidValue;   // the engine queues FP32 work only for classes with a path
            }
            return true;
         }
         return PartTable<I + kPrim3Parts>::launch(cls, ctx, bt, st, err);
      }
   }
};

// loads every kernel of this part and raises its shared-memory limit to smax
template <int I>
struct PartPreload {
   static cudaError_t run(int smax) {
      if constexpr (I >= kVrrGenCount) {
         return cudaSuccess;
      } else {
         constexpr int c = kVrrGenClasses[I];
         cudaError_t e = cudaFuncSetAttribute(k_prim3<(c >> 6) & 3, (c >> 4) & 3, (c >> 2) & 3, c & 3, double>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
         if (e != cudaSuccess) return e;
         if constexpr (class_has_fp32((c >> 6) & 3, (c >> 4) & 3, (c >> 2) & 3, c & 3)) {
            e = cudaFuncSetAttribute(k_prim3<(c >> 6) & 3, (c >> 4) & 3, (c >> 2) & 3, c & 3, float>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
            if (e != cudaSuccess) return e;
         }
         return PartPreload<I + kPrim3Parts>::run(smax);
      }
   }
};

}  // namespace

#define PRIM3_CAT2(a, b) a##b
#define PRIM3_CAT(a, b) PRIM3_CAT2(a, b)
bool PRIM3_CAT(prim3_launch_part, PRIM3_PART)(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st,
                                               cudaError_t *err) {
   if (bt.nprm == 0) { *err = cudaSuccess; return true; }
   return PartTable<PRIM3_PART>::launch(bt.cls, ctx, bt, st, err);
}

cudaError_t PRIM3_CAT(prim3_preload_part, PRIM3_PART)(int smax) { return PartPreload<PRIM3_PART>::run(smax); }

#if PRIM3_PART == 0
bool prim_has_generated(int cls) {
   for (int i = 0; i < kVrrGenCount; i++)
      if (kVrrGenClasses[i] == cls) return true;
   return false;
}

cudaError_t prim3_preload(int smax) {
   cudaError_t (*parts[])(int) = {prim3_preload_part0, prim3_preload_part1, prim3_preload_part2, prim3_preload_part3,
                               prim3_preload_part4, prim3_preload_part5, prim3_preload_part6, prim3_preload_part7};
   for (auto f : parts) {
      cudaError_t e = f(smax);
      if (e != cudaSuccess) return e;
   }
   return cudaSuccess;
}

bool prim3_launch(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err) {
   static_assert(kPrim3Parts == 8, "one call per part below");
   return prim3_launch_part0(ctx, bt, st, err) || prim3_launch_part1(ctx, bt, st, err) ||
          prim3_launch_part2(ctx, bt, st, err) || prim3_launch_part3(ctx, bt, st, err) ||
          prim3_launch_part4(ctx, bt, st, err) || prim3_launch_part5(ctx, bt, st, err) ||
          prim3_launch_part6(ctx, bt, st, err) || prim3_launch_part7(ctx, bt, st, err);
}
#endif

}  // namespace gint
