// kernels.h -- device context, batch arguments and launchers of the K-build kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <vector>
#include "engine_types.h"

namespace gint {

// Doubles per derivative order in the device copy of C0: 105 coefficients padded to a multiple
// of four, so that every row starts on a 32-byte boundary.
constexpr int kC0Row = 108;

// Everything the kernels read besides the batch records (device pointers).
struct DevCtx {
   const double *pool;        // exponents and normalised coefficients
   const BasisEnt *ents;
   const double *neighs;      // Ng lattice vectors
   int Ng;
   int nspin;
   double cell[18];           // h (rows = lattice vectors) and h^-1
   double R_cut;
   const double *C0;          // the caller's Chebyshev table repacked: per patch, (nder+1) rows of
   int ld_C0;                 // kC0Row doubles (105 coefficients, 3 zeros); ld_C0 = patch stride
   const float *C0f;          // the same table rounded to FP32, same layout (the FP32 path)
   const uint8_t *lut_low, *lut_high;   // 128 x 128 patch maps
   const double *bw;          // per patch: B1, W1, B2, W2
   const double *ftable;      // Boys table, 121 x 28
   const double *P[2];
   double *K[2];
   double hf_fac;
   size_t FP_size;
   int *err;
   unsigned long long *cnt;   // optional event counters per class [256][4], or null
   const VOp *vops;           // precompiled VRR instructions of every class (build_vops)
   const uint2 *gprog;        // HRR instructions of every class (group_prog), shared by all handles
};

// HRR instructions of the interpreted group kernels, one device copy per GPU (built by
// preload_kernels). Entries 0..255 hold, in .x, the index of each class's first instruction;
// instruction cls_first + (x - S) computes HRR workspace element x of that class (S <= x < H):
//    w[x] = w[in1] + R[dir] * w[in2],   stored as {in1 | dir << 30, in2}
// with R = CD on the ket levels and AB on the bra levels. Returns null before preload_kernels.
const uint2 *group_prog(int device);
void build_group_prog(std::vector<uint2> &out);

// One class-sorted segment of a batch (device pointers).
struct BatchArgs {
   const ClassPlan *plan;
   const uint32_t *prm;       // primitive quartet codes (ipa<<24|ipb<<16|ipc<<8|ipd)
   const uint32_t *prm_shell; // shell of each primitive quartet
   const ShellRec *shells;
   const GroupRec *groups;
   const QrttRec *qrtts;
   uint32_t nprm, nshell, ngroup;
   uint32_t nqrtt;            // contraction rows (the group kernels' work items), in group order
   const uint32_t *rowgrp;    // group of row 32 k, k < (nqrtt + 31) / 32
   const uint8_t *gflags;     // incremental replay: 0 = skip the group (its primitives and rows); null = all run
   double *AC;                // [nprm][S] image-summed VRR targets (floats in the first half for fp32)
   int fp32;                  // 1: the segment's shell quartets run in FP32 (Fm, VRR, contraction, HRR)
   double *gscratch;          // HRR workspace in global memory for the largest classes
   int cls;                   // la*64 + lb*16 + lc*4 + ld
   int prim_variant;          // 0: k_prim3 where the class has it (lane per image); 1: k_prim2 (warp per image)
   int group_variant;         // 0: k_group3 where the class has it (lane per row); 1: k_group (warp per row)
};

bool build_class_plan(int la, int lb, int lc, int ld, ClassPlan &p);
void build_vops(ClassPlan &p, std::vector<VOp> &out);
cudaError_t upload_constant_tables(const double *c2s_l0to3, const double *symm5);
cudaError_t launch_prim(const DevCtx &ctx, const BatchArgs &bt, const ClassPlan &hp, cudaStream_t st);
cudaError_t launch_group(const DevCtx &ctx, const BatchArgs &bt, const ClassPlan &hp, cudaStream_t st);
size_t group_global_scratch(const ClassPlan &hp, int *grid, int *warps);
// per-warp shared buffer of k_group: 32 contraction coefficients, then a slot that keeps shell 0's
// shared data (records, basis entries, displacements) for the next rows of the same set quartet
constexpr int kGroupShellCacheDoubles = 16;
constexpr int kGroupKpDoubles = 32 + kGroupShellCacheDoubles;
constexpr int kGroupRowsPerWarp = 4;      // consecutive rows a warp of k_group takes at a time
// k_group_block: 128 threads share one row's workspace, 256 from this workspace size on (on the
// 64-molecule l <= 3 workload the wider block was faster from about here on)
constexpr int kGroupBlockWideDoubles = 6000;
// k_group_block (variant 0) for the classes whose workspace holds at least this many doubles: on
// the 64-molecule l <= 3 workload it was faster than one warp per row from about here on
constexpr int kGroupBlockMinDoubles = 1536;
int prim_team_size(const ClassPlan &hp);
// Incremental replay screening (k_group_screen): mode 0 writes each group's largest |P| over the P
// blocks its rows read into pmax (the recording's P); mode 1 sets flags[g] = 0 for the groups whose
// bound * max|dP| / pmax is below eps (current P = dP; max|dP| bounded from the tile maxima tmax of
// launch_tile_max) and 1 for the others.
cudaError_t launch_group_screen(const DevCtx &ctx, const BatchArgs &bt, float *pmax, uint8_t *flags, double eps,
                                int mode, const float *tmax, cudaStream_t st);
// maxima of |P| over consecutive tiles of 32 elements (an upper bound, rounded up), tile_max_count(n)
cudaError_t launch_tile_max(const double *P, size_t n, float *tmax, cudaStream_t st);
size_t tile_max_count(size_t n);
// merging a queue class's recorded batches into one segment: shift the segment-relative indices
// of a part copied at (prm_base, shell_base, group_base, qrtt_base), and rebuild the group of
// every 32nd row of a merged segment
cudaError_t launch_rebase_part(uint32_t *prm_shell, uint32_t nprm, ShellRec *shells, uint32_t nshell, GroupRec *groups,
                               uint32_t ngroup, uint32_t prm_base, uint32_t shell_base, uint32_t group_base,
                               uint32_t qrtt_base, cudaStream_t st);
cudaError_t launch_row_groups(const GroupRec *groups, uint32_t ngroup, uint32_t *rowgrp, cudaStream_t st);
// whether k_prim3 (generated VRR) covers class cls (prim3.cu)
bool prim_has_generated(int cls);
// classes with an FP32 path (generated VRR and HRR code): la + lb + lc + ld <= 3
constexpr bool class_has_fp32(int la, int lb, int lc, int ld) { return la + lb + lc + ld <= 3; }
// Fixed device scratch (file-scope device array in kernels.cu) used by libgint_replay_noalloc:
// its device address for the current device; the first call on a device looks it up.
constexpr size_t kNoAllocScratchDoubles = (size_t)8 * 1024 * 1024;   // 64 MiB
constexpr int kMaxDevices = 64;
cudaError_t noalloc_scratch(double **ptr);
// loads every kernel on the current device (once per device, from libgint_init)
cudaError_t preload_kernels();
// sustained FP64 FMA rate of this GPU (TFLOP/s), from a dependent-FMA kernel
double measure_fp64_peak_tflops();

}  // namespace gint
