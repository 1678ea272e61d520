/*
 * libgint.h -- C-ABI of the B200 exchange-matrix (K) engine.
 *
 * Drop-in for the libGint C-ABI used by CP2K's HFX_LIBRARY libGint path: the same symbol
 * names, argument meanings and call protocol as the reference's src/extern_functions.cpp
 * (cited per entry point below), all wrapped around one opaque handle. Plain pointers and
 * sizes only. Contract summary (identical to the reference unless stated):
 *
 *   setup   libgint_create_handle, libgint_init, libgint_set_Potential_Truncated,
 *           libgint_set_hf_fac, libgint_set_max_mem, libgint_set_cell, libgint_set_neighs,
 *           libgint_set_Atom / libgint_set_Atom_L for every basis set
 *   K build libgint_set_P (zeroes K) ; per set quartet:
 *             [ libgint_add_prm* libgint_add_shell ]*   (one add_shell per image pair n1,n2)
 *             libgint_add_qrt ; libgint_add_qrtt*       (contractions in lexicographic order)
 *             libgint_add_set
 *           libgint_get_K  (K accumulated as K_bd += -f I_abcd P_ac, ... ; f = symm_fac*hf_fac)
 *
 * Differences from the reference, all additive:
 *   - errors never terminate the process; they are recorded and read with libgint_last_error;
 *   - libgint_destroy_handle releases a handle;
 *   - record/replay of the device-resident quartet list, counters and statistics are
 *     extensions declared at the end of this header.
 * Threading: one handle per host thread (each owns its streams and queues). As in the reference,
 * libgint_set_P, libgint_set_K and libgint_get_K (and their _polarized forms) are collective over
 * the calling thread's OpenMP team: the team's handles share one device P and K, and get_K copies
 * the team's whole K once (src/libGint.cpp:436-447, 555-628). Outside a parallel region a handle
 * is a team of one.
 */
#ifndef LIBGINT_B200_H
#define LIBGINT_B200_H

#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* src/extern_functions.cpp:9   new engine handle */
void *libgint_create_handle(void);
/* src/extern_functions.cpp:17  binds the handle to the current CUDA device and a stream */
void libgint_init(void *handle);
/* src/extern_functions.cpp:22  truncated Coulomb with cutoff R_cut (bohr); C0 is the
 * per-patch Chebyshev table, ld_C0 = (nder+1)*105 doubles per patch, C0_size total doubles */
void libgint_set_Potential_Truncated(void *handle, double R_cut, double *C0, int ld_C0, int C0_size);
/* src/extern_functions.cpp:27  K += -hf_fac * ... */
void libgint_set_hf_fac(void *handle, double fac);
/* src/extern_functions.cpp:34  device memory budget in MB for work buffers */
void libgint_set_max_mem(void *handle, int max_mem);
/* src/extern_functions.cpp:40  copies P (P_size doubles) to the device and zeroes K */
void libgint_set_P(void *handle, double *P, int P_size);
/* src/extern_functions.cpp:46  spin-polarised variant (P_alpha, P_beta) */
void libgint_set_P_polarized(void *handle, double *Pa, double *Pb, int P_size);
/* src/extern_functions.cpp:52  initial value of K */
void libgint_set_K(void *handle, double *K, int K_size);
/* src/extern_functions.cpp:57 */
void libgint_set_K_polarized(void *handle, double *Ka, double *Kb, int K_size);
/* src/extern_functions.cpp:62  completes all queued work and copies K to the host */
void libgint_get_K(void *handle, double *K);
/* src/extern_functions.cpp:67 */
void libgint_get_K_polarized(void *handle, double *Ka, double *Kb);
/* src/extern_functions.cpp:72  cell_h: rows are lattice vectors (bohr); cell_i its inverse */
void libgint_set_cell(void *handle, bool periodic, double *cell_h, double *cell_i);
/* src/extern_functions.cpp:77  nneighs lattice vectors (3 doubles each), nneighs <= 256 */
void libgint_set_neighs(void *handle, double *neighs, int nneighs);
/* src/extern_functions.cpp:82  set i: centre R[3], np <= 16 exponents Z */
void libgint_set_Atom(void *handle, int i, double *R, double *Z, int np);
/* src/extern_functions.cpp:114 set i: nl <= 4 contractions of angular momentum l <= 3,
 * K[nl*np]; coefficients are renormalised as in the reference */
void libgint_set_Atom_L(void *handle, int i, int l, int nl, double *K);
/* src/extern_functions.cpp:139 */
void libgint_set_AtomInfo(void *handle, int i, double *R, double *Z, int np, int lmin, int Lmax,
                          int *nl, double *K);
/* src/extern_functions.cpp:149 one surviving primitive quartet (indices within each set) */
void libgint_add_prm(void *handle, int ipa, int ipb, int ipc, int ipd);
/* src/extern_functions.cpp:154 sets i,j,k,l with images n1 (of b) and n2 (of d) */
void libgint_add_shell(void *handle, int i, int j, int k, int l, int n1, int n2);
/* src/extern_functions.cpp:159 no-op */
void libgint_add_cell(void *handle);
/* src/extern_functions.cpp:164 */
void libgint_add_qrt(void *handle, int la, int lb, int lc, int ld, int nla, int nlb, int nlc, int nld);
/* src/extern_functions.cpp:169 one contraction combination; symm_fac in {2,1,0.5,0.25,0};
 * ld_* < 256; offsets index the caller's P/K arrays; T* choose the transposed walk */
void libgint_add_qrtt(void *handle, double symm_fac, int la, int lb, int lc, int ld,
                      int inla, int inlb, int inlc, int inld,
                      int ld_ac, int ld_ad, int ld_bc, int ld_bd,
                      unsigned int offset_ac_L_set, unsigned int offset_ad_L_set,
                      unsigned int offset_bc_L_set, unsigned int offset_bd_L_set,
                      bool Tac, bool Tad, bool Tbc, bool Tbd);
/* src/extern_functions.cpp:182 closes the set quartet */
void libgint_add_set(void *handle);
/* src/extern_functions.cpp:187 launches all queued work */
void libgint_dispatch(void *handle);
/* No counterpart in the reference (a bulk form of the call stream above, for callers whose
 * per-call overhead dominates): the add_prm / add_shell / add_qrt / add_qrtt / add_set calls of n
 * set quartets in one call, with the same meaning, checks and errors as those calls made in order.
 * Per set quartet q: sets[4q..4q+3]; shell_count[q] image pairs, each with shell_images (n1, n2)
 * and prm_count primitive quartets taken in order from prm_codes
 * (ipa<<24 | ipb<<16 | ipc<<8 | ipd); qrt_count[q] l-combinations, each a record of 8 ints in qrt
 * (la, lb, lc, ld, nla, nlb, nlc, nld) followed by its nla*nlb*nlc*nld contraction rows in
 * lexicographic order: qrtt_fac, qrtt_ld (4 ints), qrtt_off (4 unsigned) and qrtt_T (bit 0 Tac,
 * 1 Tad, 2 Tbc, 3 Tbd). Returns libgint_last_error. */
int libgint_add_set_quartets(void *handle, int n, const int *sets, const int *shell_count, const int *shell_images,
                             const int *prm_count, const unsigned int *prm_codes, const int *qrt_count,
                             const int *qrt, const double *qrtt_fac, const int *qrtt_ld,
                             const unsigned int *qrtt_off, const unsigned char *qrtt_T);

/* ---- extensions (no counterpart in the reference's C-ABI) ------------------------------- */
/* No counterpart in the reference (its path is FP64 throughout). Mixed precision: shell quartets
 * whose Schwarz bound sqrt((ab|ab)(cd|cd)) max|P| (given by libgint_add_shell_bound) is below thr
 * run G_m, the VRR, the image sum, the contraction, the HRR and the spherical transform in FP32, for
 * the classes with la+lb+lc+ld <= 3; the screening decisions, every other class and the K update
 * stay FP64. thr <= 0 (the default) computes everything in FP64. Applies to the add_shell calls
 * that follow. */
void libgint_set_fp32_threshold(void *handle, double thr);
/* No counterpart in the reference: the Schwarz bound of the shell quartet of the next
 * libgint_add_shell (consumed by it; shells without one stay FP64). */
void libgint_add_shell_bound(void *handle, double bound);
/* last error code of the handle (0 = none); the text is returned by libgint_error_string */
int libgint_last_error(void *handle);
const char *libgint_error_string(void *handle);
void libgint_destroy_handle(void *handle);
/* sizes of the recursion plan of class (la,lb,lc,ld): out[0..7] = VRR workspace, contracted
 * targets, HRR workspace (doubles), cartesian and spherical block sizes, VRR blocks, HRR
 * steps, primitive team size; returns 0 for an unsupported class */
int libgint_plan_sizes(int la, int lb, int lc, int ld, int *out);
/* the HRR instructions of class (la,lb,lc,ld) as the interpreted group kernel runs them: out[2i],
 * out[2i+1] = {in1 | axis << 30, in2} computing workspace element S + i as
 * w[S+i] = w[in1] + R[axis] * w[in2] (R = C - D for the first info[3] elements, A - B after), up to
 * cap instructions; info[0..3] = S, H, offset of the final cartesian block, ket elements. Returns the
 * instruction count (-1: unsupported class). No GPU needed. */
int libgint_hrr_program(int la, int lb, int lc, int ld, unsigned int *out, int cap, int *info);
/* the precompiled VRR instructions of class (la,lb,lc,ld) as the large-class primitive kernels run
 * them, in order: 16-byte records {int16 out, i0..i4; uint8 zA, kind; int8 f1, f2}, up to cap;
 *   kind 0: w[out] = z[zA] w[i0] + z[zA+3] w[i1] + f1 (z[12] w[i2] + z[13] w[i3])
 *   kind 1: w[out] = z[zA] w[i0] + z[zA+3] w[i1] + f1 (z[14] w[i2] + z[15] w[i3]) + f2 z[16] w[i4]
 * (terms with a zero multiplier are left out; absent inputs point at a zero at w[V]); info = V, S,
 * (0|0)^(m) count at w[0..], ntg, then per target {workspace offset, target offset, length, e, f},
 * info_cap >= 4 + 5 ntg. Returns the instruction count (-1: unsupported class). No GPU needed. */
int libgint_vrr_program(int la, int lb, int lc, int ld, void *vops, int cap, int *info, int info_cap);
/* No counterpart in the reference. on = 1: keep the device batches of the following K build(s)
 * (the screened quartet list of an SCF step); on = 2: the same, and when the recording stops the
 * batches' segments of each class are merged into one (a replay then launches two kernels per
 * class instead of two per class and batch; while it merges it holds the recording twice); on = 0: stop
 * recording. libgint_replay captures the whole replay (every class segment's kernels on the worker
 * streams) into a CUDA graph once and relaunches it while the recording, P/K buffers and kernel
 * choices stay the same. */
void libgint_record(void *handle, int on);
/* recompute K from the recorded quartet list with the current P (after libgint_set_P), without
 * the add_* stream; K is then read with libgint_get_K. Returns the device time in ms. */
double libgint_replay(void *handle);
/* No counterpart in the reference. Incremental K update for SCF loops from the recorded quartet
 * list: after libgint_set_P(dP) and libgint_set_K(K_previous), adds K(dP) to K (not zeroed), skipping
 * every set quartet whose bound (libgint_add_shell_bound at recording time) scaled by
 * max|dP| / max|P_recorded| over the P blocks it reads is below eps, and those dP does not touch.
 * K_k = K_{k-1} + K(P_k - P_{k-1}) is then read with libgint_get_K. Returns the device time in ms. */
double libgint_replay_incremental(void *handle, double eps);
/* libgint_replay with the summed device time per kernel kind: kt[0] = Fm+VRR kernel,
 * kt[1] = contraction+HRR+spherical+K kernel (ms) */
double libgint_replay_profile(void *handle, double *kt);
/* libgint_replay_profile plus the per-class split: kcls[c*2 + {0,1}] (ms), c as above */
double libgint_replay_profile_classes(void *handle, double *kt, double *kcls);
/* No counterpart in the reference. Per-class kernel choice: after libgint_record and libgint_set_P,
 * libgint_autotune times, for every class of the recorded quartet list, the primitive kernel with
 * generated per-lane VRR against the per-warp interpreted one, and the group kernel with one lane
 * per contraction row (generated HRR; classes with la+lb+lc+ld <= 3) or one block per row
 * (interpreted HRR; the other classes, where the workspace fits a block's shared memory) against one
 * warp per row (interpreted HRR), and keeps the faster of each for every following launch;
 * out[2c], out[2c+1] (c = la*64+lb*16+lc*4+ld; 512 ints, may be NULL) receive the choices
 * (0 = per-lane or per-block, 1 = per-warp). libgint_set_tuning installs such a table,
 * libgint_get_tuning reads it. Returns 0 or the error code. */
int libgint_autotune(void *handle, int *out);
void libgint_set_tuning(void *handle, const int *in);
void libgint_get_tuning(void *handle, int *out);
/* algorithmic FP64 operation counts of class (la,lb,lc,ld) following the reference recursion:
 * out[0] per Chebyshev G_m evaluation, [1] per Boys evaluation, [2] VRR per image, [3] image
 * sum per image, [4] contraction per primitive and row, [5] HRR per shell and row,
 * [6] spherical transform per row, [7] K update per row */
int libgint_plan_flops(int la, int lb, int lc, int ld, double *out);
/* No counterpart in the reference. For callers that cannot allocate device memory while K is
 * built (their framework owns every device byte through its own pool, or cudaMalloc/cudaFree
 * would synchronise a pipeline they must not stall): recompute K from the recorded quartet list
 * (libgint_record) into the caller's device buffers P_dev/K_dev (K_size doubles, packed like
 * P), on `stream` (the handle's stream if NULL), with no device allocation. The intermediates
 * use a fixed 64 MiB device scratch array inside the library, held by every GPU that loads it
 * until exit; each recorded class segment must fit it (record with a small
 * libgint_set_max_mem, e.g. 150), otherwise the call fails with a clear error. K_dev is zeroed
 * first. The first call on a device looks up the scratch address (make it before any stream
 * capture); calls that overlap on the GPU share the scratch and race. Returns 0 or the error. */
int libgint_replay_noalloc(void *handle, const double *P_dev, double *K_dev, size_t K_size, void *stream);
/* per-class device event counters: out[c*4 + {0,1,2,3}] = Chebyshev G_m evaluations, Boys
 * evaluations, images through the VRR, primitive quartets; c = la*64 + lb*16 + lc*4 + ld */
void libgint_set_counters(void *handle, int on);
void libgint_get_counters(void *handle, unsigned long long *out);
/* out[0..7] = shell quartets, primitive quartets, groups, batches, kernel launches, bytes
 * copied host -> device, shell quartets and primitive quartets computed in FP32 */
void libgint_get_stats(void *handle, long long *out);
/* the tables the engine builds on the host, for inspection and tests: Boys table [121*28],
 * c2s [4][70] (per l: rows m, columns cartesian), patch maps [2*128*128], per-patch (B,W) [207*4] */
void libgint_host_tables(double *ftable, double *c2s, unsigned char *lut, double *bw);
/* FP64 FMA rate of the current GPU (TFLOP/s), measured by a dependent-FMA kernel */
double libgint_fp64_peak_tflops(void);

#ifdef __cplusplus
}
#endif
#endif
