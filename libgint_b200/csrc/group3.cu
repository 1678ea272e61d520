// group3.cu -- k_group3<la,lb,lc,ld>: contraction + HRR + image-pair sum + spherical transform +
// K update, one lane per contraction row, for the classes with generated HRR code (grp_gen.cuh).
//
// A group is one set quartet of one class: all its image pairs (shell quartets) and its
// nla*nlb*nlc*nld contraction rows. One lane takes one row: it contracts the image-summed targets
// of each shell over its primitives with the row's coefficients, applies that shell's HRR (its own
// AB and CD), sums the shells, transforms the sum to spherical harmonics and adds the four exchange
// updates to K with atomics (reference src/compute_ECO.cpp:12-214, src/compute_HRR.cpp:102-225,
// src/compute_SPH.cpp:58-237, src/compute_KS.cpp:8-117). All indices are compile-time
// constants and the workspace lives in registers.
//
// Compiled kGroup3Parts times (GROUP3_PART = 0..3); part i instantiates the generated classes
// whose position in kGrpGenClasses is i modulo kGroup3Parts.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include "engine_types.h"
#include "grp_gen.cuh"
#include "group3.h"
#include "kernels.h"
#include "prim_common.cuh"

#ifndef GROUP3_PART
#define GROUP3_PART 0
#endif

namespace gint {
namespace {

// symmetry factors by bucket (reference src/libGint.cpp:262-267)
__device__ __forceinline__ double symm_factor(int i) {
   return i == 0 ? 2.0 : (i == 1 ? 1.0 : (i == 2 ? 0.5 : (i == 3 ? 0.25 : 0.0)));
}

// resident 128-thread blocks per SM the register budget is sized for: the kernel waits on
// chains of dependent loads, so small classes trade registers for more warps in flight
template <int LA, int LB, int LC, int LD>
struct Group3Shape {
   static constexpr int L = LA + LB + LC + LD;
   static constexpr int MINB = L <= 1 ? 8 : (L == 2 ? 6 : 4);
};

// R = double: the FP64 path; R = float: the FP32 path (contraction, HRR and spherical transform in
// FP32 from the FP32 targets of k_prim3; the K update in FP64).
template <int LA, int LB, int LC, int LD, class R>
__global__ void __launch_bounds__(128, Group3Shape<LA, LB, LC, LD>::MINB) k_group3(DevCtx ctx, BatchArgs bt) {
   using G = GrpGen<LA, LB, LC, LD>;
   constexpr int S = G::S, Nc = G::Nc, Ns = G::Ns;
   constexpr int nsb = 2 * LB + 1, nsc = 2 * LC + 1, nsd = 2 * LD + 1;
   constexpr int nscd = nsc * nsd, nsbcd = nsb * nscd;
   const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
   const uint32_t nblk = (bt.nqrtt + 31) >> 5;
   // one lane per contraction row: a warp takes 32 consecutive rows, so the lanes of one set
   // quartet's rows read the same primitive codes and image-summed targets (broadcast loads)
   for (uint32_t blk = blockIdx.x * wpb + (threadIdx.x >> 5); blk < nblk; blk += gridDim.x * wpb) {
      const uint32_t q0 = blk << 5, q = q0 + lane;
      const uint32_t gi = row_group_warp(bt, q0, lane);
      if (q >= bt.nqrtt || (bt.gflags && !__ldg(bt.gflags + gi))) continue;   // screened (incremental)
      const GroupRec Gr = bt.groups[gi];
      const int nl1 = Gr.nl[1], nl2 = Gr.nl[2], nl3 = Gr.nl[3];
      const int r = (int)(q - Gr.qrtt_off);
      const int ia = r / (nl1 * nl2 * nl3), ib = (r / (nl2 * nl3)) % nl1, ic = (r / nl3) % nl2, id = r % nl3;
      R cart[Nc];
#pragma unroll
      for (int t = 0; t < Nc; t++) cart[t] = R(0);
      for (uint32_t s = 0; s < Gr.nshell; s++) {
         const ShellRec sh = bt.shells[Gr.shell_off + s];
         const BasisEnt ea = ctx.ents[sh.ent[0]], eb = ctx.ents[sh.ent[1]];
         const BasisEnt ec = ctx.ents[sh.ent[2]], ed = ctx.ents[sh.ent[3]];
         const double *Ka = ctx.pool + ea.k_off + ia * ea.np;
         const double *Kb = ctx.pool + eb.k_off + ib * eb.np;
         const double *Kc = ctx.pool + ec.k_off + ic * ec.np;
         const double *Kd = ctx.pool + ed.k_off + id * ed.np;
         R T[S];
#pragma unroll
         for (int j = 0; j < S; j++) T[j] = R(0);
         const R *AC = reinterpret_cast<const R *>(bt.AC);
         // contraction over the primitives (reference src/compute_ECO.cpp:131-212); four per
         // iteration so that the next ones' loads overlap this one's FMAs
#pragma unroll 4
         for (uint32_t ip = 0; ip < sh.nprm; ip++) {
            const uint32_t code = __ldg(bt.prm + sh.prm_off + ip);
            const R kp = (R)__ldg(Ka + (code >> 24)) * (R)__ldg(Kb + ((code >> 16) & 255)) *
                         (R)__ldg(Kc + ((code >> 8) & 255)) * (R)__ldg(Kd + (code & 255));
            const R *row = AC + (size_t)(sh.prm_off + ip) * S;
#pragma unroll
            for (int j = 0; j < S; j++) T[j] += kp * __ldg(row + j);
         }
         double A[3], B[3], C[3], D[3], CDs[3];
         shell_geom(ctx, ea, eb, ec, ed, sh.n1, sh.n2, A, B, C, D, CDs);
         const R AB[3] = {(R)(A[0] - B[0]), (R)(A[1] - B[1]), (R)(A[2] - B[2])};
         const R CD[3] = {(R)(C[0] - D[0]), (R)(C[1] - D[1]), (R)(C[2] - D[2])};
         G::hrr(T, AB, CD, cart);
      }
      R sph[Ns];
      G::sph(cart, sph);
      const QrttRec k = bt.qrtts[q];
      const double fac = symm_factor(k.idx_fac) * ctx.hf_fac;
#pragma unroll
      for (int t = 0; t < Ns; t++) {
         const int isa = t / nsbcd, isb = (t / nscd) % nsb, isc = (t / nsd) % nsc, isd = t % nsd;
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
         const double iabcd = -fac * (double)sph[t];
         for (int sp = 0; sp < ctx.nspin; sp++) {
            const double *Pm = ctx.P[sp];
            double *Km = ctx.K[sp];
            atomicAdd(Km + Ibd, iabcd * __ldg(Pm + Iac));
            atomicAdd(Km + Ibc, iabcd * __ldg(Pm + Iad));
            atomicAdd(Km + Iad, iabcd * __ldg(Pm + Ibc));
            atomicAdd(Km + Iac, iabcd * __ldg(Pm + Ibd));
         }
      }
   }
}

template <int LA, int LB, int LC, int LD>
cudaError_t launch_one(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st) {
   const int threads = 128;
   // one 32-row block per warp: rows cost from one primitive to thousands, so the block scheduler,
   // which starts a new block wherever one finishes, balances them better than a grid-stride loop
   const long blocks = std::max(1L, std::min(((long)bt.nqrtt + threads - 1) / threads, 1L << 30));
   if constexpr (class_has_fp32(LA, LB, LC, LD)) {
      if (bt.fp32) {
         k_group3<LA, LB, LC, LD, float><<<(unsigned)blocks, threads, 0, st>>>(ctx, bt);
         return cudaGetLastError();
      }
   } else {
      if (bt.fp32) return cudaErrorInvalidValue;   // no FP32 segments for these classes
   }
   k_group3<LA, LB, LC, LD, double><<<(unsigned)blocks, threads, 0, st>>>(ctx, bt);
   return cudaGetLastError();
}

template <int I>
struct PartTable {
   static bool launch(int cls, const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err) {
      if constexpr (I >= kGrpGenCount) {
         return false;
      } else {
         constexpr int c = kGrpGenClasses[I];
         if (cls == c) {
            *err = launch_one<(c >> 6) & 3, (c >> 4) & 3, (c >> 2) & 3, c & 3>(ctx, bt, st);
            return true;
         }
         return PartTable<I + kGroup3Parts>::launch(cls, ctx, bt, st, err);
      }
   }
};

// loads (and so registers with the runtime) every kernel of this part
template <int I>
struct PartPreload {
   static cudaError_t run() {
      if constexpr (I >= kGrpGenCount) {
         return cudaSuccess;
      } else {
         constexpr int c = kGrpGenClasses[I];
         cudaFuncAttributes a;
         cudaError_t e = cudaFuncGetAttributes(&a, k_group3<(c >> 6) & 3, (c >> 4) & 3, (c >> 2) & 3, c & 3, double>);
         if (e != cudaSuccess) return e;
         if constexpr (class_has_fp32((c >> 6) & 3, (c >> 4) & 3, (c >> 2) & 3, c & 3)) {
            e = cudaFuncGetAttributes(&a, k_group3<(c >> 6) & 3, (c >> 4) & 3, (c >> 2) & 3, c & 3, float>);
            if (e != cudaSuccess) return e;
         }
         return PartPreload<I + kGroup3Parts>::run();
      }
   }
};

}  // namespace

#define GROUP3_CAT2(a, b) a##b
#define GROUP3_CAT(a, b) GROUP3_CAT2(a, b)
bool GROUP3_CAT(group3_launch_part, GROUP3_PART)(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st,
                                                 cudaError_t *err) {
   if (bt.nqrtt == 0) { *err = cudaSuccess; return true; }
   return PartTable<GROUP3_PART>::launch(bt.cls, ctx, bt, st, err);
}

cudaError_t GROUP3_CAT(group3_preload_part, GROUP3_PART)() { return PartPreload<GROUP3_PART>::run(); }

#if GROUP3_PART == 0
cudaError_t group3_preload() {
   cudaError_t (*parts[])() = {group3_preload_part0, group3_preload_part1, group3_preload_part2,
                               group3_preload_part3};
   for (auto f : parts) {
      cudaError_t e = f();
      if (e != cudaSuccess) return e;
   }
   return cudaSuccess;
}

bool group3_launch(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err) {
   static_assert(kGroup3Parts == 4, "one call per part below");
   return group3_launch_part0(ctx, bt, st, err) || group3_launch_part1(ctx, bt, st, err) ||
          group3_launch_part2(ctx, bt, st, err) || group3_launch_part3(ctx, bt, st, err);
}
#endif

}  // namespace gint
