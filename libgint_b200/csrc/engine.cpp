// engine.cpp -- host engine and C-ABI of the B200 K build.
//
// The caller streams screened quartets through the libgint_* calls exactly as for the
// reference (src/libGint.cpp:151-414). The engine keeps one host queue per angular-momentum
// class; add_set commits a set quartet as one group record (all its image pairs and
// contraction rows). When the queues reach the work-buffer budget they are flushed: packed
// class-sorted into one pinned staging buffer, copied with one cudaMemcpyAsync, and processed
// by two kernels per class on the handle's stream. Two staging/device slots alternate, so the
// GPU works on one batch while the caller fills the next. get_K drains the queue and copies K.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../../include/libgint.h"
#include "engine_types.h"
#include "kernels.h"
#include "tcg_patches.h"

namespace gint {

// ---------------------------------------------------------------------------------------
// tables built on the host
// ---------------------------------------------------------------------------------------
// Boys table F_m(T), T = 0, 0.1, ..., 12.0 and m = 0..27, the Taylor table of the
// reference's fgamma0 (src/libGint.cpp:488-497). The values must be the reference's own, not
// exact ones: its generator (src/fgamma.cpp:53-123, Bessel-function ratios by a continued
// fraction and a truncated series) is accurate to ~1e-10 for m >= 6, and the engine has to
// reproduce those values to agree with the reference's K at 1e-12. The steps below are that
// algorithm: r_{j-1} = -T / ((4j+2) - T r_j) from r_{kmax+9} = 0, then
// F_n = f/(2n+1) + sum_k f t_k (prod_{j<=k} r_{j-1}) (2k+1)/(2n+1), f = 2 sinh(T/2) e^{-T/2} / T,
// t_k = t_{k-1} (2n-2k+1)/(2n+2k+1), stopping at the first term below DBL_EPSILON.
static void boys_reference_values(int nmax, double T, double *f) {
   const int kmax = 50;
   double r[kmax + 10];
   if (T < 1.e-13) {
      for (int n = 0; n <= nmax; n++) f[n] = 1.0 / (2. * n + 1.);
      return;
   }
   r[kmax + 9] = 0.0;
   for (int j = kmax + 9; j >= 1; j--) r[j - 1] = -T / ((4. * j + 2.) - T * r[j]);
   const double factor = 2.0 * std::sinh(0.5 * T) * std::exp(-0.5 * T) / T;
   for (int n = 0; n <= nmax; n++) {
      double sumtot = factor / (2. * n + 1.);
      double term = 1.0;
      for (int k = 1; k <= kmax; k++) {
         term = term * (2. * n - 2. * k + 1.) / (2. * n + 2. * k + 1);
         double p = 1.0;
         for (int j = 1; j <= k; j++) p = p * r[j - 1];
         const double sumterm = factor * term * p * (2. * k + 1.) / (2. * n + 1.);
         if (std::fabs(sumterm) < 2.220446049250313e-16) break;
         if (k == kmax) break;
         sumtot = sumtot + sumterm;
      }
      f[n] = sumtot;
   }
}

static void make_boys_table(std::vector<double> &ft) {
   ft.assign(121 * 28, 0.0);
   for (int it = 0; it <= 120; it++) boys_reference_values(27, (double)it * 0.1, &ft[it * 28]);
}

// Cartesian -> real solid harmonic coefficients in CP2K's order and normalisation (the
// values of the reference's src/c2s.h): unnormalised solid harmonics, each row scaled to
// the norm of the monomial x^.. with unit exponents, l = 3 rows rounded to 9 decimals as in
// the CP2K table.
static void make_c2s(double out[4][70]) {
   static const int sh1[3][3] = {{0, 1, 0}, {0, 0, 1}, {1, 0, 0}};
   static const int sh2[5][6] = {{0, 1, 0, 0, 0, 0}, {0, 0, 0, 0, 1, 0}, {-1, 0, 0, -1, 0, 2},
                                 {0, 0, 1, 0, 0, 0}, {1, 0, 0, -1, 0, 0}};
   static const int sh3[7][10] = {{0, 3, 0, 0, 0, 0, -1, 0, 0, 0}, {0, 0, 0, 0, 1, 0, 0, 0, 0, 0},
                                  {0, -1, 0, 0, 0, 0, -1, 0, 4, 0}, {0, 0, -3, 0, 0, 0, 0, -3, 0, 2},
                                  {-1, 0, 0, -1, 0, 4, 0, 0, 0, 0}, {0, 0, 1, 0, 0, 0, 0, -1, 0, 0},
                                  {1, 0, 0, -3, 0, 0, 0, 0, 0, 0}};
   auto df = [](int n) { double r = 1; for (int k = n; k > 1; k -= 2) r *= k; return r; };
   auto exps = [](int l, int i, int e[3]) {
      int a = 0; while ((a + 1) * (a + 2) / 2 <= i) a++;
      e[0] = l - a; e[2] = i - a * (a + 1) / 2; e[1] = a - e[2];
   };
   std::memset(out, 0, sizeof(double) * 4 * 70);
   out[0][0] = 1.0;
   for (int l = 1; l <= 3; l++) {
      int nc = (l + 1) * (l + 2) / 2;
      for (int m = 0; m < 2 * l + 1; m++) {
         const int *row = l == 1 ? sh1[m] : (l == 2 ? sh2[m] : sh3[m]);
         double n2 = 0;
         for (int i = 0; i < nc; i++) for (int j = 0; j < nc; j++) {
            if (!row[i] || !row[j]) continue;
            int e1[3], e2[3]; exps(l, i, e1); exps(l, j, e2);
            double o = 1;
            for (int d = 0; d < 3; d++) { int s = e1[d] + e2[d]; if (s & 1) { o = 0; break; } o *= df(s - 1); }
            n2 += row[i] * row[j] * o;
         }
         double nr = std::sqrt(n2);
         for (int i = 0; i < nc; i++) {
            double v = row[i] / nr;
            if (l >= 3) v = std::round(v * 1e9) / 1e9;
            out[l][m * nc + i] = v;
         }
      }
   }
}

// Patch maps (low-R, high-R: the patch containing X = i/127 in each dimension, lo < X <= hi)
// and the per-patch bias/weight (B, W) that map a patch onto [-1, 1]: TG = (2X - B) W.
static void make_patch_tables(std::vector<uint8_t> &lut, std::vector<double> &bw) {
   lut.assign(2 * 128 * 128, 0);
   for (int i1 = 0; i1 < 128; i1++) {
      double X1 = (double)i1 / 127.0;
      for (int i2 = 0; i2 < 128; i2++) {
         double X2 = (double)i2 / 127.0;
         for (int side = 0; side < 2; side++) {
            int first = side ? TCG_NPATCH_LOW : 0, last = side ? TCG_NPATCH : TCG_NPATCH_LOW;
            int found = 0;
            for (int p = first; p < last; p++) {
               double lo1 = tcg_patch_rect[p][0] / 128.0, hi1 = tcg_patch_rect[p][1] / 128.0;
               double lo2 = tcg_patch_rect[p][2] / 128.0, hi2 = tcg_patch_rect[p][3] / 128.0;
               bool in1 = X1 <= hi1 && (X1 > lo1 || lo1 == 0.0);
               bool in2 = X2 <= hi2 && (X2 > lo2 || lo2 == 0.0);
               if (in1 && in2) { found = p; break; }
            }
            lut[side * 128 * 128 + i1 * 128 + i2] = (uint8_t)found;
         }
      }
   }
   bw.assign(TCG_NPATCH * 4, 0.0);
   for (int p = 0; p < TCG_NPATCH; p++) {
      bw[p * 4 + 0] = (tcg_patch_rect[p][0] + tcg_patch_rect[p][1]) / 128.0;
      bw[p * 4 + 1] = 128.0 / (tcg_patch_rect[p][1] - tcg_patch_rect[p][0]);
      bw[p * 4 + 2] = (tcg_patch_rect[p][2] + tcg_patch_rect[p][3]) / 128.0;
      bw[p * 4 + 3] = 128.0 / (tcg_patch_rect[p][3] - tcg_patch_rect[p][2]);
   }
}

// ---------------------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------------------
struct HostSet {
   double R[3] = {0, 0, 0};
   int np = 0;
   double Z[kMaxPrm] = {0};
   int nL = 0;
   int l[8] = {0}, nl[8] = {0};
   std::vector<double> K[8];
   bool defined = false;
};

// A group being filled by the current set quartet: the records go straight into the class
// queue and are committed (or rolled back) by add_set.
struct OpenGroup {
   int cls;
   uint32_t shell_off, qrtt_off;
   size_t prm_off;
   uint8_t nl[4];
   bool have_qrt;
   int nq;
   double bound;     // largest bound of the group's shell quartets (HUGE_VAL once one has none)
};

// Growable array in pinned host memory (pageable if no device is present), so that a batch is
// uploaded straight from the queues with cudaMemcpyAsync.
template <class T>
struct PVec {
   T *d = nullptr;
   size_t n = 0, cap = 0;
   bool pinned = false;
   PVec() = default;
   PVec(const PVec &) = delete;
   PVec &operator=(const PVec &) = delete;
   ~PVec() { release(); }
   void release() {
      if (d) { if (pinned) cudaFreeHost(d); else std::free(d); }
      d = nullptr; cap = 0; n = 0;
   }
   void reserve(size_t c) {
      if (c <= cap) return;
      size_t nc = std::max(c, cap ? cap * 2 : (size_t)16384);
      T *nd = nullptr;
      bool pin = cudaHostAlloc((void **)&nd, nc * sizeof(T), cudaHostAllocPortable) == cudaSuccess;
      if (!pin) { cudaGetLastError(); nd = (T *)std::malloc(nc * sizeof(T)); }
      if (n) std::memcpy(nd, d, n * sizeof(T));
      if (d) { if (pinned) cudaFreeHost(d); else std::free(d); }
      d = nd; cap = nc; pinned = pin;
   }
   inline void push_back(const T &x) { if (n == cap) reserve(n + 1); d[n++] = x; }
   inline void append(const T *x, size_t k) { if (n + k > cap) reserve(n + k); std::memcpy(d + n, x, k * sizeof(T)); n += k; }
   inline void fill(size_t k, const T &v) { if (n + k > cap) reserve(n + k); for (size_t i = 0; i < k; i++) d[n + i] = v; n += k; }
   inline size_t size() const { return n; }
   inline void clear() { n = 0; }
   inline void resize(size_t k) { if (k > cap) reserve(k); n = k; }
   inline T *data() { return d; }
};

struct ClassQ {
   PVec<uint32_t> prm, prm_shell;
   PVec<ShellRec> shells;
   PVec<GroupRec> groups;
   PVec<QrttRec> qrtts;
   PVec<uint32_t> rowgrp;           // group of contraction row 32 k (filled when the batch is packed)
   bool active = false;
};

struct DBuf {
   void *p = nullptr;
   size_t bytes = 0;
};

// The device P and K of a K build. As in the reference (src/libGint.cpp:436-447, 555-562,
// 613-628), the handles of one OpenMP team share them: libgint_set_P, libgint_set_K and
// libgint_get_K are collective over the calling thread's team (orphaned omp constructs bind to
// it), one thread uploads P and zeroes K for all, every handle's kernels add into the one K, and
// get_K copies the team's K once after a barrier. A handle used outside a parallel region is a
// team of one.
struct Team {
   int device = 0;
   DBuf P[2], K[2];
   int nspin = 0;
   size_t FP_size = 0;
   bool ok = false;     // P uploaded and K zeroed without an error
   Team() = default;
   Team(const Team &) = delete;
   Team &operator=(const Team &) = delete;
   ~Team();
};

struct Slot {
   DBuf rec, ac, gscr;
   cudaEvent_t ev = nullptr;        // all work of the slot's last batch
   cudaEvent_t ev_copy = nullptr;   // the uploads of the slot's last batch
   bool busy = false, copy_busy = false;
};

// Class segments of one batch are independent (K is updated with atomics), so they run on
// kWorkStreams worker streams that fork from and join back to the handle's stream; the tails of
// one class's kernels then overlap the next class's. Six workers (seven streams with the handle's,
// within the runtime's default eight device connections) replay the 32-water K build 2% faster
// than four; eight or twelve gain nothing more.
constexpr int kWorkStreams = 6;

struct Handle {
   int device = 0;
   cudaStream_t stream = nullptr;
   cudaStream_t work[kWorkStreams] = {};
   cudaEvent_t work_ev[kWorkStreams] = {};
   cudaEvent_t fork_ev = nullptr;
   cudaEvent_t noalloc_ev = nullptr;             // libgint_replay_noalloc: the caller's stream waits for the handle's
   int err = 0;
   std::string errmsg;
   // potential and tables
   double R_cut = 0;
   std::vector<double> C0;
   int ld_C0 = 0;
   bool have_pot = false, pot_dirty = true;
   double hf_fac = 1.0;
   size_t max_mem_mb = 4000;
   bool periodic = false;
   double cell[18] = {0};
   std::vector<double> neighs{0.0, 0.0, 0.0};
   int Ng = 1;
   bool neighs_dirty = true;
   // basis
   std::vector<HostSet> sets;
   std::vector<int> ent_base;
   struct SetFast { int np, nL, l0, ent; };   // hot-path copy of each set's shape
   std::vector<SetFast> fast;
   bool basis_dirty = true, ent_dirty = true;
   // device-resident data
   DBuf d_pool, d_ents, d_neighs, d_C0, d_C0f, d_lut, d_bw, d_ft, d_plans, d_err, d_vops;
   DBuf d_tmax;                     // incremental replays: tile maxima of |dP|
   std::vector<VOp> vops;           // precompiled VRR instructions of all classes
   std::shared_ptr<Team> team;      // device P and K (shared by the handles of an OpenMP team)
   int nspin = 0;
   size_t FP_size = 0;
   ClassPlan plans[256];
   // mixed precision: shell quartets whose Schwarz bound (libgint_add_shell_bound) is below the
   // threshold run in FP32 where the class has an FP32 path; 0 = everything in FP64
   double fp32_thr = 0.0;
   double next_bound = HUGE_VAL;    // bound of the next add_shell (reset by it)
   bool has_fp32[256];
   // per-class kernel choice (libgint_autotune / libgint_set_tuning): primitive and group kernel
   // variant, 0 = the generated per-lane kernels where the class has them, 1 = the per-warp ones
   uint8_t tune_prim[256], tune_group[256];
   int S_of[256];                   // plans[c].S, kept compact for the streaming path
   bool plans_ready = false;
   // streaming state
   std::vector<uint32_t> prm_tmp;
   OpenGroup open[64];
   int nopen = 0;
   // Queue classes: qc = c (FP64) or c + kFp32 (the same class in FP32), c = la*64+lb*16+lc*4+ld
   int open_of[2 * 256];
   ClassQ qs[2][2 * 256];           // queue sets, one per slot
   ClassQ *q = qs[0];               // the set being filled
   std::vector<int> active;
   size_t pend_prims = 0, pend_ac = 0, pend_rec = 0;
   Slot slots[2];
   int cur = 0;
   // record / replay of the device-resident quartet list
   struct RecSeg { int c; size_t o_prm, o_ps, o_sh, o_g, o_q, o_rg; uint32_t nprm, nshell, ngroup, nqrtt; };
   // per recorded batch: its records, its class segments, and (gbuf) each segment's per-group
   // largest |P| of the recording (float) and incremental-replay flags (byte) at g_pmax[i], g_flag[i]
   struct RecBatch { DBuf rec, gbuf; std::vector<RecSeg> segs; std::vector<size_t> g_pmax, g_flag; };
   bool recording = false;
   bool merge_rec = false;          // libgint_record(h, 2): one segment per queue class at the end
   std::vector<RecBatch> recs;
   long long rec_gen = 0;           // bumped whenever the recording changes
   // the replay captured as a CUDA graph, and what it was captured with
   struct GraphKey { DevCtx ctx; long long rec_gen; void *ac, *gscr; size_t half; double eps; };
   cudaGraphExec_t graph_exec = nullptr;
   GraphKey graph_key;
   long long graph_launches = 0;
   DBuf rec_ac, rec_gscr;
   size_t arena_off[kWorkStreams] = {};   // replay: each worker stream's AC arena in rec_ac (doubles)
   // optional device event counters [256 classes][4]
   DBuf d_cnt;
   bool counting = false;
   long long n_launch = 0;
   // statistics
   long long n_shells = 0, n_prims = 0, n_groups = 0, n_flush = 0, h2d_bytes = 0;
   long long n_shells_fp32 = 0, n_prims_fp32 = 0;
};

static void set_error(Handle *h, int code, const std::string &msg) {
   if (!h->err) { h->err = code; h->errmsg = msg; }
}

static bool ck(Handle *h, cudaError_t e, const char *what) {
   if (e == cudaSuccess) return true;
   set_error(h, 100 + (int)e, std::string(what) + ": " + cudaGetErrorString(e));
   return false;
}

static bool ensure(Handle *h, DBuf &b, size_t bytes, const char *what) {
   if (b.bytes >= bytes && b.p) return true;
   if (b.p) { cudaFree(b.p); b.p = nullptr; b.bytes = 0; }
   size_t alloc = std::max<size_t>(bytes, 256);
   if (!ck(h, cudaMalloc(&b.p, alloc), what)) return false;
   b.bytes = alloc;
   return true;
}

static void release(DBuf &b) { if (b.p) cudaFree(b.p); b.p = nullptr; b.bytes = 0; }

Team::~Team() {
   int d = -1;
   cudaGetDevice(&d);
   if (d != device) cudaSetDevice(device);
   for (int s = 0; s < 2; s++) { release(P[s]); release(K[s]); }
   if (d >= 0 && d != device) cudaSetDevice(d);
}

// whether the calling thread is inside an OpenMP parallel region (a team of more than one)
static bool in_team() {
#ifdef _OPENMP
   return omp_in_parallel() && omp_get_num_threads() > 1;
#else
   return false;
#endif
}

static inline int cls_of(int la, int lb, int lc, int ld) { return la * 64 + lb * 16 + lc * 4 + ld; }

constexpr int kFp32 = 256;          // queue-class offset of the FP32 variant of a class

// queue class of the shell quartet being added: its class, in FP32 if its bound is below the
// threshold and the class has an FP32 path (consumes the pending bound)
static inline int shell_qclass(Handle *h, int c) {
   const bool f32 = h->fp32_thr > 0.0 && h->next_bound < h->fp32_thr && h->has_fp32[c];
   return f32 ? c + kFp32 : c;
}

static inline OpenGroup *open_group(Handle *h, int c) {
   int o = h->open_of[c];
   if (o >= 0) return &h->open[o];
   if (h->nopen >= 64) return nullptr;
   o = h->nopen++;
   h->open_of[c] = o;
   OpenGroup &g = h->open[o];
   ClassQ &Q = h->q[c];
   g.cls = c;
   g.shell_off = (uint32_t)Q.shells.size();
   g.qrtt_off = (uint32_t)Q.qrtts.size();
   g.prm_off = Q.prm.size();
   g.nl[0] = g.nl[1] = g.nl[2] = g.nl[3] = 0;
   g.have_qrt = false;
   g.nq = 0;
   g.bound = 0.0;
   return &g;
}

static void ensure_ent_base(Handle *h);

// makes the handle's device current on the calling thread (a caller thread may never have
// touched CUDA, or may drive handles of several devices)
static void use_device(Handle *h) {
   int d = -1;
   if (cudaGetDevice(&d) != cudaSuccess || d != h->device) ck(h, cudaSetDevice(h->device), "cudaSetDevice");
}

// host -> device copy on the handle's stream; callers synchronise the stream before returning
// when the source may be released (the handle's streams do not order against the legacy stream)
static bool h2d(Handle *h, void *dst, const void *src, size_t bytes, const char *what) {
   return ck(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream), what);
}

static bool upload_tables(Handle *h) {
   if (h->err) return false;
   use_device(h);
   ensure_ent_base(h);
   bool uploaded = false;
   if (!h->plans_ready) {
      if (!ensure(h, h->d_plans, sizeof(ClassPlan) * 256, "plans")) return false;
      if (!h2d(h, h->d_plans.p, h->plans, sizeof(ClassPlan) * 256, "plans")) return false;
      if (!ensure(h, h->d_vops, h->vops.size() * sizeof(VOp), "VRR instructions")) return false;
      if (!h2d(h, h->d_vops.p, h->vops.data(), h->vops.size() * sizeof(VOp), "VRR instructions")) return false;
      std::vector<uint8_t> lut;
      std::vector<double> bw;
      make_patch_tables(lut, bw);
      std::vector<double> ft;
      make_boys_table(ft);
      if (!ensure(h, h->d_lut, lut.size(), "lut") || !ensure(h, h->d_bw, bw.size() * 8, "bw") ||
          !ensure(h, h->d_ft, ft.size() * 8, "ftable") || !ensure(h, h->d_err, sizeof(int) * 4, "err"))
         return false;
      if (!h2d(h, h->d_lut.p, lut.data(), lut.size(), "lut")) return false;
      if (!h2d(h, h->d_bw.p, bw.data(), bw.size() * 8, "bw")) return false;
      if (!h2d(h, h->d_ft.p, ft.data(), ft.size() * 8, "ftable")) return false;
      if (!ck(h, cudaMemsetAsync(h->d_err.p, 0, sizeof(int) * 4, h->stream), "err")) return false;
      double c2s[4][70];
      make_c2s(c2s);
      const double symm[5] = {2.0, 1.0, 0.5, 0.25, 0.0};
      if (!ck(h, upload_constant_tables(&c2s[0][0], symm), "constant tables")) return false;
      h->plans_ready = true;
      uploaded = true;
   }
   if (h->basis_dirty) {
      std::vector<double> pool;
      std::vector<BasisEnt> ents;
      for (size_t s = 0; s < h->sets.size(); s++) {
         const HostSet &hs = h->sets[s];
         int zoff = (int)pool.size();
         pool.insert(pool.end(), hs.Z, hs.Z + hs.np);
         for (int e = 0; e < hs.nL; e++) {
            BasisEnt be;
            std::memset(&be, 0, sizeof(be));
            for (int q = 0; q < 3; q++) be.R[q] = hs.R[q];
            be.z_off = zoff; be.np = hs.np; be.nl = hs.nl[e]; be.l = hs.l[e];
            be.k_off = (int)pool.size();
            pool.insert(pool.end(), hs.K[e].begin(), hs.K[e].end());
            ents.push_back(be);
         }
      }
      if (pool.empty()) pool.push_back(0.0);
      if (ents.empty()) ents.push_back(BasisEnt{});
      if (!ensure(h, h->d_pool, pool.size() * 8, "basis") || !ensure(h, h->d_ents, ents.size() * sizeof(BasisEnt), "basis"))
         return false;
      if (!h2d(h, h->d_pool.p, pool.data(), pool.size() * 8, "basis")) return false;
      if (!h2d(h, h->d_ents.p, ents.data(), ents.size() * sizeof(BasisEnt), "basis")) return false;
      h->basis_dirty = false;
      uploaded = true;
   }
   if (h->pot_dirty && h->have_pot) {
      // repack to kC0Row doubles per derivative order (32-byte aligned rows, zero padding)
      const int nord = h->ld_C0 / 105;
      std::vector<double> packed((size_t)207 * nord * kC0Row, 0.0);
      for (int p = 0; p < 207; p++)
         for (int k = 0; k < nord; k++)
            std::memcpy(&packed[((size_t)p * nord + k) * kC0Row], &h->C0[(size_t)p * h->ld_C0 + (size_t)k * 105],
                        105 * sizeof(double));
      if (!ensure(h, h->d_C0, packed.size() * 8, "C0")) return false;
      if (!h2d(h, h->d_C0.p, packed.data(), packed.size() * 8, "C0")) return false;
      // the FP32 path's copy, same layout
      std::vector<float> packed_f(packed.begin(), packed.end());
      if (!ensure(h, h->d_C0f, packed_f.size() * 4, "C0 (FP32)")) return false;
      if (!h2d(h, h->d_C0f.p, packed_f.data(), packed_f.size() * 4, "C0 (FP32)")) return false;
      if (!ck(h, cudaStreamSynchronize(h->stream), "C0 upload")) return false;
      h->pot_dirty = false;
      uploaded = true;
   }
   if (h->neighs_dirty) {
      if (!ensure(h, h->d_neighs, h->neighs.size() * 8, "neighs")) return false;
      if (!h2d(h, h->d_neighs.p, h->neighs.data(), h->neighs.size() * 8, "neighs")) return false;
      h->neighs_dirty = false;
      uploaded = true;
   }
   // the sources above are temporaries or may change: wait for the copies
   if (uploaded && !ck(h, cudaStreamSynchronize(h->stream), "table upload")) return false;
   return true;
}

static void ensure_ent_base(Handle *h) {
   if (h->ent_base.size() == h->sets.size() && !h->ent_dirty) return;
   h->ent_base.assign(h->sets.size(), 0);
   h->fast.assign(h->sets.size(), Handle::SetFast{0, 0, 0, 0});
   int n = 0;
   for (size_t s = 0; s < h->sets.size(); s++) {
      h->ent_base[s] = n;
      h->fast[s] = {h->sets[s].np, h->sets[s].nL, h->sets[s].nL ? h->sets[s].l[0] : 0, n};
      n += h->sets[s].nL;
   }
   h->ent_dirty = false;
}

// worker streams wait for everything queued so far on the handle's stream
static void fork_workers(Handle *h) {
   ck(h, cudaEventRecord(h->fork_ev, h->stream), "event record");
   for (int w = 0; w < kWorkStreams; w++) ck(h, cudaStreamWaitEvent(h->work[w], h->fork_ev, 0), "stream wait");
}

// the handle's stream waits for everything queued on the worker streams
static void join_workers(Handle *h) {
   for (int w = 0; w < kWorkStreams; w++) {
      ck(h, cudaEventRecord(h->work_ev[w], h->work[w]), "event record");
      ck(h, cudaStreamWaitEvent(h->stream, h->work_ev[w], 0), "stream wait");
   }
}

// The worker stream of the i-th segment of a batch. Segments whose group kernel uses the shared
// global HRR scratch all go to worker 0, so they never run concurrently.
static cudaStream_t worker_for(Handle *h, int i, bool uses_scratch) {
   return uses_scratch ? h->work[0] : h->work[1 + i % (kWorkStreams - 1)];
}

// The worker stream (index) that a replay gives its i-th recorded segment (of class c), as
// worker_for does, and the image-summed targets that segment needs (doubles, 32-byte multiple).
static int replay_worker(Handle *h, int c, int i) {
   int a, b;
   return group_global_scratch(h->plans[c & 255], &a, &b) != 0 ? 0 : 1 + i % (kWorkStreams - 1);
}
static size_t replay_seg_ac(Handle *h, int c, uint32_t nprm) {
   return ((size_t)nprm * h->plans[c & 255].S + 3) & ~(size_t)3;
}

static DevCtx make_ctx(Handle *h) {
   DevCtx c;
   std::memset(&c, 0, sizeof(c));
   c.pool = (const double *)h->d_pool.p;
   c.ents = (const BasisEnt *)h->d_ents.p;
   c.neighs = (const double *)h->d_neighs.p;
   c.Ng = h->Ng;
   c.nspin = h->nspin;
   std::memcpy(c.cell, h->cell, sizeof(c.cell));
   c.R_cut = h->R_cut;
   c.C0 = (const double *)h->d_C0.p;
   c.ld_C0 = (h->ld_C0 / 105) * kC0Row;
   c.C0f = (const float *)h->d_C0f.p;
   c.lut_low = (const uint8_t *)h->d_lut.p;
   c.lut_high = (const uint8_t *)h->d_lut.p + 128 * 128;
   c.bw = (const double *)h->d_bw.p;
   c.ftable = (const double *)h->d_ft.p;
   for (int s = 0; s < 2; s++) {
      c.P[s] = h->team ? (const double *)h->team->P[s].p : nullptr;
      c.K[s] = h->team ? (double *)h->team->K[s].p : nullptr;
   }
   c.hf_fac = h->hf_fac;
   c.FP_size = h->FP_size;
   c.err = (int *)h->d_err.p;
   c.cnt = h->counting ? (unsigned long long *)h->d_cnt.p : nullptr;
   c.vops = (const VOp *)h->d_vops.p;
   c.gprog = group_prog(h->device);
   return c;
}

static size_t slot_budget_bytes(Handle *h) {
   // two slots share ~90% of the caller's budget
   return std::max<size_t>((size_t)h->max_mem_mb * 1024 * 1024 * 9 / 20, 64u << 20);
}

static inline size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

static void clear_queues(Handle *h) {
   for (int c : h->active) {
      ClassQ &Q = h->q[c];
      Q.prm.clear(); Q.prm_shell.clear(); Q.shells.clear(); Q.groups.clear(); Q.qrtts.clear(); Q.rowgrp.clear();
      Q.active = false;
   }
   h->active.clear();
   h->pend_prims = h->pend_ac = h->pend_rec = 0;
}

static void flush(Handle *h) {
   if (h->active.empty()) return;
   use_device(h);
   if (h->err) { clear_queues(h); return; }   // drop queued work after an error
   if (!upload_tables(h)) { clear_queues(h); return; }
   if (h->nspin == 0 || !h->team || !h->team->K[0].p) { set_error(h, 4, "work queued before libgint_set_P"); clear_queues(h); return; }
   if (!h->have_pot) { set_error(h, 4, "work queued before libgint_set_Potential_Truncated"); clear_queues(h); return; }
   for (int c : h->active) {
      if (h->ld_C0 < (h->plans[c & 255].L + 1) * 105) {
         set_error(h, 2, "C0 holds fewer derivative orders than la+lb+lc+ld+1");
         clear_queues(h);
         return;
      }
   }
   Slot &s = h->slots[h->cur];
   if (s.busy) { ck(h, cudaEventSynchronize(s.ev), "slot wait"); s.busy = false; }
   // device layout of the batch: per class, prm | prm_shell | shells | groups | qrtts | rowgrp
   struct Seg { int c; size_t o_prm, o_ps, o_sh, o_g, o_q, o_rg; size_t ac_off; };
   std::vector<Seg> segs;
   size_t off = 0, ac = 0;
   for (int c : h->active) {
      ClassQ &Q = h->q[c];
      // the group of every 32nd contraction row (rows are stored in group order)
      const size_t nq = Q.qrtts.size(), nblk = (nq + 31) / 32;
      Q.rowgrp.resize(nblk);
      {
         const GroupRec *gr = Q.groups.data();
         const size_t ng = Q.groups.size();
         size_t gi = 0;
         for (size_t k = 0; k < nblk; k++) {
            const size_t row = 32 * k;
            while (gi + 1 < ng && gr[gi + 1].qrtt_off <= row) gi++;
            Q.rowgrp.data()[k] = (uint32_t)gi;
         }
      }
      Seg g;
      g.c = c;
      g.o_prm = off; off = al16(off + Q.prm.size() * 4);
      g.o_ps = off; off = al16(off + Q.prm_shell.size() * 4);
      g.o_sh = off; off = al16(off + Q.shells.size() * sizeof(ShellRec));
      g.o_g = off; off = al16(off + Q.groups.size() * sizeof(GroupRec));
      g.o_q = off; off = al16(off + Q.qrtts.size() * sizeof(QrttRec));
      g.o_rg = off; off = al16(off + Q.rowgrp.size() * 4);
      g.ac_off = ac;
      ac += ((size_t)Q.prm.size() * h->plans[c & 255].S + 1) & ~(size_t)1;
      segs.push_back(g);
   }
   if (!ensure(h, s.rec, std::max(off, (size_t)(64u << 20)), "record buffer")) return;
   if (!ensure(h, s.ac, std::max(ac * 8, (size_t)(64u << 20)), "AC buffer")) return;
   char *dev_rec = (char *)s.rec.p;
   Handle::RecBatch *rb = nullptr;
   if (h->recording) {
      h->recs.emplace_back();
      rb = &h->recs.back();
      if (!ensure(h, rb->rec, off, "recorded batch")) return;
      dev_rec = (char *)rb->rec.p;
   }
   for (const Seg &g : segs) {
      ClassQ &Q = h->q[g.c];
      auto up = [&](size_t o, const void *src, size_t bytes) {
         return !bytes || ck(h, cudaMemcpyAsync(dev_rec + o, src, bytes, cudaMemcpyHostToDevice, h->stream), "record upload");
      };
      if (!up(g.o_prm, Q.prm.data(), Q.prm.size() * 4) || !up(g.o_ps, Q.prm_shell.data(), Q.prm_shell.size() * 4) ||
          !up(g.o_sh, Q.shells.data(), Q.shells.size() * sizeof(ShellRec)) ||
          !up(g.o_g, Q.groups.data(), Q.groups.size() * sizeof(GroupRec)) ||
          !up(g.o_q, Q.qrtts.data(), Q.qrtts.size() * sizeof(QrttRec)) ||
          !up(g.o_rg, Q.rowgrp.data(), Q.rowgrp.size() * 4))
         return;
   }
   h->h2d_bytes += (long long)off;
   ck(h, cudaEventRecord(s.ev_copy, h->stream), "event record");
   s.copy_busy = true;
   DevCtx ctx = make_ctx(h);
   fork_workers(h);
   int nseg = 0;
   for (const Seg &g : segs) {
      ClassQ &Q = h->q[g.c];
      const ClassPlan &hp = h->plans[g.c & 255];
      BatchArgs bt;
      std::memset(&bt, 0, sizeof(bt));
      char *base = dev_rec;
      bt.cls = g.c & 255;
      bt.fp32 = g.c >= kFp32;
      bt.prim_variant = h->tune_prim[g.c & 255];
      bt.group_variant = h->tune_group[g.c & 255];
      bt.plan = (const ClassPlan *)h->d_plans.p + (g.c & 255);
      bt.prm = (const uint32_t *)(base + g.o_prm);
      bt.prm_shell = (const uint32_t *)(base + g.o_ps);
      bt.shells = (const ShellRec *)(base + g.o_sh);
      bt.groups = (const GroupRec *)(base + g.o_g);
      bt.qrtts = (const QrttRec *)(base + g.o_q);
      bt.rowgrp = (const uint32_t *)(base + g.o_rg);
      bt.nprm = (uint32_t)Q.prm.size();
      bt.nshell = (uint32_t)Q.shells.size();
      bt.ngroup = (uint32_t)Q.groups.size();
      bt.nqrtt = (uint32_t)Q.qrtts.size();
      bt.AC = (double *)s.ac.p + g.ac_off;
      int gg = 0, gw = 0;
      size_t gs = group_global_scratch(hp, &gg, &gw);
      if (gs) {
         if (!ensure(h, s.gscr, gs * 8, "HRR scratch")) return;
         bt.gscratch = (double *)s.gscr.p;
      }
      cudaStream_t ws = worker_for(h, nseg++, gs != 0);
      if (!ck(h, launch_prim(ctx, bt, hp, ws), "k_prim launch")) return;
      if (!ck(h, launch_group(ctx, bt, hp, ws), "k_group launch")) return;
      h->n_launch += 2;
      if (rb) rb->segs.push_back({g.c, g.o_prm, g.o_ps, g.o_sh, g.o_g, g.o_q, g.o_rg, bt.nprm, bt.nshell, bt.ngroup, bt.nqrtt});
      h->n_prims += bt.nprm; h->n_shells += bt.nshell; h->n_groups += bt.ngroup;
      if (bt.fp32) { h->n_prims_fp32 += bt.nprm; h->n_shells_fp32 += bt.nshell; }
   }
   join_workers(h);
   ck(h, cudaEventRecord(s.ev, h->stream), "event record");
   s.busy = true;
   h->n_flush++;
   // switch to the other queue set; its previous batch must have finished uploading
   h->active.clear();
   h->pend_prims = h->pend_ac = h->pend_rec = 0;
   h->cur ^= 1;
   h->q = h->qs[h->cur];
   Slot &o = h->slots[h->cur];
   if (o.copy_busy) { ck(h, cudaEventSynchronize(o.ev_copy), "queue wait"); o.copy_busy = false; }
   for (int c = 0; c < 2 * 256; c++) {
      ClassQ &Q = h->q[c];
      if (Q.prm.size() || Q.shells.size() || Q.qrtts.size() || Q.groups.size()) {
         Q.prm.clear(); Q.prm_shell.clear(); Q.shells.clear(); Q.groups.clear(); Q.qrtts.clear(); Q.rowgrp.clear();
      }
      Q.active = false;
   }
}

static void drain(Handle *h) {
   flush(h);
   ck(h, cudaStreamSynchronize(h->stream), "stream synchronize");
   if (h->d_err.p && !h->err) {
      int e = 0;
      if (ck(h, cudaMemcpy(&e, h->d_err.p, sizeof(int), cudaMemcpyDeviceToHost), "error flag") && e)
         set_error(h, 3, "a K update addressed P/K outside P_size");
   }
}

// libgint_set_P: collective over the calling thread's OpenMP team (see Team). Every thread
// reaches the same omp constructs whatever its own state, so that none waits at a barrier for
// another that returned early.
static void set_P_impl(Handle *h, int nspin, const double *Pa, const double *Pb, int n) {
   use_device(h);
   const bool ok = n > 0;
   if (!ok) set_error(h, 2, "P_size must be positive");
   // this handle's previous build must be complete before P/K are replaced
   for (Slot &s : h->slots) if (s.busy) { ck(h, cudaEventSynchronize(s.ev), "slot wait"); s.busy = false; }
   ck(h, cudaStreamSynchronize(h->stream), "stream synchronize");
   for (Slot &s : h->slots) s.copy_busy = false;
   std::shared_ptr<Team> *bc = nullptr;
   const bool team_call = in_team();
   // every handle of the team has finished its previous build
#pragma omp barrier
#pragma omp single copyprivate(bc)
   {
      // one thread uploads P and zeroes K for the team, reusing its team's buffers
      std::shared_ptr<Team> t = (h->team && (team_call || h->team.use_count() == 1)) ? h->team : std::make_shared<Team>();
      t->device = h->device;
      t->nspin = nspin;
      t->FP_size = ok ? (size_t)n : 0;
      t->ok = false;
      const double *src[2] = {Pa, Pb};
      bool good = ok && !h->err;
      for (int sp = 0; good && sp < nspin; sp++) {
         good = ensure(h, t->P[sp], (size_t)n * 8, "P") && ensure(h, t->K[sp], (size_t)n * 8, "K") &&
                h2d(h, t->P[sp].p, src[sp], (size_t)n * 8, "P upload") &&
                ck(h, cudaMemsetAsync(t->K[sp].p, 0, (size_t)n * 8, h->stream), "K zero");
         if (good) h->h2d_bytes += (long long)n * 8;
      }
      // P is copied at call time (the caller may reuse its array), and the other threads' kernels
      // read it once they leave this construct
      t->ok = good && ck(h, cudaStreamSynchronize(h->stream), "P upload");
      bc = new std::shared_ptr<Team>(t);
   }
   h->team = *bc;
   // every thread holds the team before the broadcast copy is released
#pragma omp barrier
#pragma omp single nowait
   delete bc;
   h->nspin = nspin;
   h->FP_size = h->team->FP_size;
   if (!h->team->ok) set_error(h, 4, "libgint_set_P: the team's P upload failed");
   upload_tables(h);
}

// libgint_get_K: every thread completes its own queued work, then one thread copies the team's K
// (collective, see Team). Threads that pass their own arrays get K in the array of the thread
// that made the copy only, as in the reference.
static void get_K_impl(Handle *h, double *Ka, double *Kb) {
   use_device(h);
   drain(h);
   const bool have = h->nspin != 0 && h->team && h->team->ok;
   if (!have) set_error(h, 4, "libgint_get_K before libgint_set_P");
   // every handle's kernels have finished adding into K
#pragma omp barrier
#pragma omp single
   {
      if (have) {
         double *dst[2] = {Ka, Kb};
         for (int sp = 0; sp < h->nspin; sp++)
            if (dst[sp]) ck(h, cudaMemcpy(dst[sp], h->team->K[sp].p, h->FP_size * 8, cudaMemcpyDeviceToHost), "K download");
      }
   }
}

// libgint_set_K / libgint_set_K_polarized: collective like set_P; one thread uploads the team's K.
static void set_K_impl(Handle *h, int nspin, const double *Ka, const double *Kb, int K_size) {
   use_device(h);
   const bool ok = h->nspin >= nspin && h->team && h->team->ok && (size_t)K_size == h->FP_size;
   if (!ok) set_error(h, 2, nspin == 1 ? "libgint_set_K: call set_P first with the same size"
                                       : "libgint_set_K_polarized: call set_P_polarized first");
   drain(h);
#pragma omp barrier
#pragma omp single
   {
      if (ok) {
         const double *src[2] = {Ka, Kb};
         for (int sp = 0; sp < nspin; sp++) h2d(h, h->team->K[sp].p, src[sp], (size_t)K_size * 8, "K upload");
         ck(h, cudaStreamSynchronize(h->stream), "K upload");
      }
   }
}

// Enqueue one replay of every recorded batch (K zeroed first) on the handle's stream: with
// kt == nullptr the segments spread over the worker streams (forked from and joined back to the
// handle's stream), otherwise they run in order on the handle's stream with an event before and
// after each kernel (kev, kcl: per-kernel timing). Each segment's image-summed targets live in
// its worker stream's arena of the replay AC buffer (prepare_replay). eps >= 0: an incremental replay (K is not zeroed; each segment's groups are screened against
// eps first, see k_group_screen, and the screened ones skipped).
static bool enqueue_replay(Handle *h, const DevCtx &ctx, std::vector<cudaEvent_t> *kev,
                           std::vector<int> *kcl, long long *nlaunch, double eps = -1.0) {
   if (eps < 0.0) {
      for (int sp = 0; sp < h->nspin; sp++)
         if (!ck(h, cudaMemsetAsync(h->team->K[sp].p, 0, h->FP_size * 8, h->stream), "K zero")) return false;
   } else {
      // tile maxima of |dP| for the groups' screening (before the fork: every worker needs them)
      if (!ck(h, launch_tile_max(ctx.P[0], h->FP_size, (float *)h->d_tmax.p, h->stream), "tile max launch")) return false;
      *nlaunch += 1;
   }
   auto kmark = [&]() {
      if (!kev) return;
      cudaEvent_t e; cudaEventCreate(&e); cudaEventRecord(e, h->stream); kev->push_back(e);
   };
   const bool spread = kev == nullptr;
   if (spread) fork_workers(h);
   int nseg = 0;
   for (size_t bi = 0; bi < h->recs.size(); bi++) {
      auto &rb = h->recs[bi];
      char *base = (char *)rb.rec.p;
      for (size_t si = 0; si < rb.segs.size(); si++) {
         const auto &g = rb.segs[si];
         BatchArgs bt;
         std::memset(&bt, 0, sizeof(bt));
         bt.cls = g.c & 255;
         bt.fp32 = g.c >= kFp32;
         bt.prim_variant = h->tune_prim[g.c & 255];
         bt.group_variant = h->tune_group[g.c & 255];
         bt.plan = (const ClassPlan *)h->d_plans.p + (g.c & 255);
         bt.prm = (const uint32_t *)(base + g.o_prm);
         bt.prm_shell = (const uint32_t *)(base + g.o_ps);
         bt.shells = (const ShellRec *)(base + g.o_sh);
         bt.groups = (const GroupRec *)(base + g.o_g);
         bt.qrtts = (const QrttRec *)(base + g.o_q);
         bt.rowgrp = (const uint32_t *)(base + g.o_rg);
         bt.nprm = g.nprm; bt.nshell = g.nshell; bt.ngroup = g.ngroup; bt.nqrtt = g.nqrtt;
         // the segment's targets live in its worker stream's arena: the segments of one stream run
         // one after another, and no other stream touches that arena
         const int w = replay_worker(h, g.c, nseg++);
         bt.AC = (double *)h->rec_ac.p + h->arena_off[w];
         bt.gscratch = (double *)h->rec_gscr.p;
         const ClassPlan &hp = h->plans[g.c & 255];
         cudaStream_t st = spread ? h->work[w] : h->stream;
         if (eps >= 0.0) {
            char *gb = (char *)rb.gbuf.p;
            uint8_t *flags = (uint8_t *)(gb + rb.g_flag[si]);
            if (!ck(h, launch_group_screen(ctx, bt, (float *)(gb + rb.g_pmax[si]), flags, eps, 1,
                                           (const float *)h->d_tmax.p, st), "screen launch"))
               return false;
            bt.gflags = flags;
            *nlaunch += 1;
         }
         kmark();
         if (kcl) kcl->push_back(g.c & 255);
         if (!ck(h, launch_prim(ctx, bt, hp, st), "k_prim launch")) return false;
         kmark();
         if (!ck(h, launch_group(ctx, bt, hp, st), "k_group launch")) return false;
         kmark();
         *nlaunch += 2;
      }
   }
   if (spread) join_workers(h);
   return !h->err;
}

static void drop_graph(Handle *h) {
   if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
   h->graph_exec = nullptr;
}

// Re-run every recorded batch with the current P (K is zeroed first). Returns the elapsed
// milliseconds measured with CUDA events on the handle's stream. The spread replay is captured
// once into a CUDA graph (the whole K build: every class segment's two kernels on the worker
// streams, with their batch-to-batch dependencies) and relaunched as one graph while the recording
// and the device pointers it was captured with stay the same.
// Checks that a replay can run and sizes its buffers; *half = the replay AC buffer's size (doubles).
static bool prepare_replay(Handle *h, size_t *half) {
   if (h->err) return false;
   use_device(h);
   if (h->recs.empty()) { set_error(h, 4, "libgint_replay: nothing recorded"); return false; }
   if (!h->team || !h->team->ok) { set_error(h, 4, "libgint_replay: call libgint_set_P first"); return false; }
   if (!upload_tables(h)) return false;
   // The replay runs the recorded segments in order on the worker streams (replay_worker); the
   // segments of one stream run one after another, so each stream needs one AC arena as large as
   // the largest segment it runs, and the streams' arenas are disjoint.
   size_t arena[kWorkStreams] = {}, gs = 0;
   int i = 0;
   for (auto &rb : h->recs)
      for (auto &g : rb.segs) {
         const int w = replay_worker(h, g.c, i++);
         arena[w] = std::max(arena[w], replay_seg_ac(h, g.c, g.nprm));
         int a, b;
         gs = std::max(gs, group_global_scratch(h->plans[g.c & 255], &a, &b));
      }
   size_t ac = 0;
   for (int w = 0; w < kWorkStreams; w++) { h->arena_off[w] = ac; ac += arena[w]; }
   if (!ensure(h, h->rec_ac, std::max<size_t>(ac * 8, 256), "replay AC")) return false;
   if (gs && !ensure(h, h->rec_gscr, gs * 8, "replay HRR scratch")) return false;
   *half = ac;
   return true;
}

static double replay_impl(Handle *h, double *kt, double *kcls = nullptr, double eps = -1.0) {
   size_t ac = 0;
   if (!prepare_replay(h, &ac)) return -1.0;
   if (eps >= 0.0) {
      for (auto &rb : h->recs)
         if (!rb.gbuf.p) { set_error(h, 4, "libgint_replay_incremental: the recording has no group screening data"); return -1.0; }
      if (!ensure(h, h->d_tmax, std::max<size_t>(tile_max_count(h->FP_size) * 4, 256), "tile maxima")) return -1.0;
   }
   DevCtx ctx = make_ctx(h);
   cudaEvent_t e0, e1;
   cudaEventCreate(&e0); cudaEventCreate(&e1);
   if (kt) {
      // per-kernel timing: the launches in order on one stream, one event pair per kernel
      std::vector<cudaEvent_t> kev;
      std::vector<int> kcl;
      ck(h, cudaEventRecord(e0, h->stream), "event");
      enqueue_replay(h, ctx, &kev, &kcl, &h->n_launch, eps);
      ck(h, cudaEventRecord(e1, h->stream), "event");
      ck(h, cudaEventSynchronize(e1), "replay");
      kt[0] = kt[1] = 0.0;
      if (kcls) std::memset(kcls, 0, sizeof(double) * 512);
      for (size_t i = 0; i + 2 < kev.size(); i += 3) {
         float a = 0, b = 0;
         cudaEventElapsedTime(&a, kev[i], kev[i + 1]);
         cudaEventElapsedTime(&b, kev[i + 1], kev[i + 2]);
         kt[0] += a; kt[1] += b;
         if (kcls) { kcls[kcl[i / 3] * 2] += a; kcls[kcl[i / 3] * 2 + 1] += b; }
      }
      for (auto e : kev) cudaEventDestroy(e);
   } else {
      Handle::GraphKey key;
      std::memset(&key, 0, sizeof(key));
      std::memcpy(&key.ctx, &ctx, sizeof(ctx));
      key.rec_gen = h->rec_gen;
      key.ac = h->rec_ac.p; key.gscr = h->rec_gscr.p; key.half = ac; key.eps = eps;
      if (!h->graph_exec || std::memcmp(&key, &h->graph_key, sizeof(key)) != 0) {
         drop_graph(h);
         cudaGraph_t graph = nullptr;
         long long n = 0;
         bool ok = ck(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
         if (ok) {
            ok = enqueue_replay(h, ctx, nullptr, nullptr, &n, eps);
            const cudaError_t ec = cudaStreamEndCapture(h->stream, &graph);
            ok = ok && ck(h, ec, "graph capture");
         }
         if (ok && !ck(h, cudaGraphInstantiate(&h->graph_exec, graph, 0), "graph instantiate")) h->graph_exec = nullptr;
         if (graph) cudaGraphDestroy(graph);
         if (!h->graph_exec) { cudaEventDestroy(e0); cudaEventDestroy(e1); return -1.0; }
         h->graph_key = key;
         h->graph_launches = n;
      }
      ck(h, cudaEventRecord(e0, h->stream), "event");
      ck(h, cudaGraphLaunch(h->graph_exec, h->stream), "graph launch");
      h->n_launch += h->graph_launches;
      ck(h, cudaEventRecord(e1, h->stream), "event");
      ck(h, cudaEventSynchronize(e1), "replay");
   }
   float ms = -1.f;
   cudaEventElapsedTime(&ms, e0, e1);
   cudaEventDestroy(e0); cudaEventDestroy(e1);
   return h->err ? -1.0 : (double)ms;
}

// After a recording: per recorded segment, each group's largest |P| over the blocks its rows read,
// with the recording's P (for the screening of incremental replays, libgint_replay_incremental).
// libgint_record(h, 2) at the end of the recording: the segments of each queue class in all the
// recorded batches become one segment of one batch, so that a replay launches two kernels per class
// instead of two per class and batch. The parts are copied device to device in batch order (so
// every row, shell and primitive keeps its relative order) and their segment-relative indices are
// shifted (launch_rebase_part); the per-32-row group table is rebuilt. While it copies, the
// recording is held twice.
static bool merge_recording(Handle *h) {
   if (h->err || h->recs.size() < 2) return !h->err;
   std::vector<int> order;
   std::vector<std::vector<std::pair<size_t, size_t>>> parts(2 * 256);
   for (size_t bi = 0; bi < h->recs.size(); bi++)
      for (size_t si = 0; si < h->recs[bi].segs.size(); si++) {
         const int c = h->recs[bi].segs[si].c;
         if (parts[c].empty()) order.push_back(c);
         parts[c].push_back({bi, si});
      }
   Handle::RecBatch m;
   size_t off = 0;
   for (int c : order) {
      Handle::RecSeg g;
      std::memset(&g, 0, sizeof(g));
      g.c = c;
      for (auto &pr : parts[c]) {
         const auto &s = h->recs[pr.first].segs[pr.second];
         g.nprm += s.nprm; g.nshell += s.nshell; g.ngroup += s.ngroup; g.nqrtt += s.nqrtt;
      }
      g.o_prm = off; off = al16(off + (size_t)g.nprm * 4);
      g.o_ps = off; off = al16(off + (size_t)g.nprm * 4);
      g.o_sh = off; off = al16(off + (size_t)g.nshell * sizeof(ShellRec));
      g.o_g = off; off = al16(off + (size_t)g.ngroup * sizeof(GroupRec));
      g.o_q = off; off = al16(off + (size_t)g.nqrtt * sizeof(QrttRec));
      g.o_rg = off; off = al16(off + ((size_t)g.nqrtt + 31) / 32 * 4);
      m.segs.push_back(g);
   }
   if (!ensure(h, m.rec, std::max<size_t>(off, 256), "merged recording")) return false;
   char *dst = (char *)m.rec.p;
   for (size_t k = 0; k < order.size(); k++) {
      const Handle::RecSeg &g = m.segs[k];
      uint32_t pb = 0, sb = 0, gb = 0, qb = 0;
      for (auto &pr : parts[g.c]) {
         const auto &s = h->recs[pr.first].segs[pr.second];
         const char *src = (const char *)h->recs[pr.first].rec.p;
         auto cp = [&](size_t to, size_t from, size_t bytes) {
            return !bytes || ck(h, cudaMemcpyAsync(dst + to, src + from, bytes, cudaMemcpyDeviceToDevice, h->stream),
                                "merged recording copy");
         };
         if (!cp(g.o_prm + (size_t)pb * 4, s.o_prm, (size_t)s.nprm * 4) ||
             !cp(g.o_ps + (size_t)pb * 4, s.o_ps, (size_t)s.nprm * 4) ||
             !cp(g.o_sh + (size_t)sb * sizeof(ShellRec), s.o_sh, (size_t)s.nshell * sizeof(ShellRec)) ||
             !cp(g.o_g + (size_t)gb * sizeof(GroupRec), s.o_g, (size_t)s.ngroup * sizeof(GroupRec)) ||
             !cp(g.o_q + (size_t)qb * sizeof(QrttRec), s.o_q, (size_t)s.nqrtt * sizeof(QrttRec))) {
            cudaStreamSynchronize(h->stream);   // the copies already queued read the old batches
            release(m.rec);
            return false;
         }
         if ((pb || sb || gb || qb) &&
             !ck(h, launch_rebase_part((uint32_t *)(dst + g.o_ps) + pb, s.nprm, (ShellRec *)(dst + g.o_sh) + sb,
                                       s.nshell, (GroupRec *)(dst + g.o_g) + gb, s.ngroup, pb, sb, gb, qb, h->stream),
                 "merged recording rebase")) {
            cudaStreamSynchronize(h->stream);
            release(m.rec);
            return false;
         }
         pb += s.nprm; sb += s.nshell; gb += s.ngroup; qb += s.nqrtt;
      }
      if (!ck(h, launch_row_groups((const GroupRec *)(dst + g.o_g), g.ngroup, (uint32_t *)(dst + g.o_rg), h->stream),
              "merged recording row table")) {
         cudaStreamSynchronize(h->stream);
         release(m.rec);
         return false;
      }
   }
   if (!ck(h, cudaStreamSynchronize(h->stream), "merged recording")) { release(m.rec); return false; }
   for (auto &rb : h->recs) { release(rb.rec); release(rb.gbuf); }
   h->recs.clear();
   h->recs.push_back(m);
   return true;
}

static void record_group_pmax(Handle *h) {
   if (h->err || h->recs.empty() || !h->team || !h->team->ok) return;
   use_device(h);
   DevCtx ctx = make_ctx(h);
   for (auto &rb : h->recs) {
      if (rb.gbuf.p) continue;
      size_t off = 0;
      rb.g_pmax.clear(); rb.g_flag.clear();
      for (auto &g : rb.segs) {
         rb.g_pmax.push_back(off); off = al16(off + (size_t)g.ngroup * 4);
         rb.g_flag.push_back(off); off = al16(off + (size_t)g.ngroup);
      }
      if (!ensure(h, rb.gbuf, std::max<size_t>(off, 256), "recorded screening data")) return;
      char *base = (char *)rb.rec.p;
      for (size_t si = 0; si < rb.segs.size(); si++) {
         const auto &g = rb.segs[si];
         BatchArgs bt;
         std::memset(&bt, 0, sizeof(bt));
         bt.cls = g.c & 255;
         bt.groups = (const GroupRec *)(base + g.o_g);
         bt.qrtts = (const QrttRec *)(base + g.o_q);
         bt.ngroup = g.ngroup; bt.nqrtt = g.nqrtt;
         if (!ck(h, launch_group_screen(ctx, bt, (float *)((char *)rb.gbuf.p + rb.g_pmax[si]), nullptr, 0.0, 0, nullptr,
                                        h->stream),
                 "screen launch"))
            return;
      }
   }
   ck(h, cudaStreamSynchronize(h->stream), "recorded screening data");
}

// The autotuner: for every class of the recording, the primitive kernels (generated per-lane VRR,
// variant 0, against the per-warp interpreted VRR, variant 1) and the group kernels (one lane per
// contraction row with generated HRR, variant 0, against one warp per row with the interpreted HRR,
// variant 1) are timed on the class's recorded segments, serialised on the handle's stream with
// CUDA events, and the faster of each is kept. FP32 segments have only variant 0. K is zeroed
// afterwards (the timing runs add into it).
static int autotune_impl(Handle *h, int *out) {
   size_t ac = 0;
   if (!prepare_replay(h, &ac)) return h->err ? h->err : 4;
   drop_graph(h);
   DevCtx ctx = make_ctx(h);
   double t[256][2][2] = {};
   bool seen[256] = {}, alt_p[256] = {}, alt_g[256] = {};
   cudaEvent_t ev[5];
   for (auto &e : ev) cudaEventCreate(&e);
   int nseg = 0;
   for (size_t bi = 0; bi < h->recs.size() && !h->err; bi++) {
      auto &rb = h->recs[bi];
      char *base = (char *)rb.rec.p;
      for (auto &g : rb.segs) {
         const int wk = replay_worker(h, g.c, nseg++);   // the arena the replay gives this segment
         if (g.c >= kFp32) continue;
         const int c = g.c;
         const ClassPlan &hp = h->plans[c];
         BatchArgs bt;
         std::memset(&bt, 0, sizeof(bt));
         bt.cls = c;
         bt.plan = (const ClassPlan *)h->d_plans.p + c;
         bt.prm = (const uint32_t *)(base + g.o_prm);
         bt.prm_shell = (const uint32_t *)(base + g.o_ps);
         bt.shells = (const ShellRec *)(base + g.o_sh);
         bt.groups = (const GroupRec *)(base + g.o_g);
         bt.qrtts = (const QrttRec *)(base + g.o_q);
         bt.rowgrp = (const uint32_t *)(base + g.o_rg);
         bt.nprm = g.nprm; bt.nshell = g.nshell; bt.ngroup = g.ngroup; bt.nqrtt = g.nqrtt;
         bt.AC = (double *)h->rec_ac.p + h->arena_off[wk];
         bt.gscratch = (double *)h->rec_gscr.p;
         seen[c] = true;
         alt_p[c] = prim_has_generated(c);
         alt_g[c] = true;   // variant 0: k_group3, or k_group_block where it applies; variant 1: k_group
         ck(h, cudaEventRecord(ev[0], h->stream), "event");
         bt.prim_variant = 1;
         ck(h, launch_prim(ctx, bt, hp, h->stream), "k_prim launch");
         ck(h, cudaEventRecord(ev[1], h->stream), "event");
         bt.prim_variant = 0;
         ck(h, launch_prim(ctx, bt, hp, h->stream), "k_prim launch");
         ck(h, cudaEventRecord(ev[2], h->stream), "event");
         bt.group_variant = 1;
         ck(h, launch_group(ctx, bt, hp, h->stream), "k_group launch");
         ck(h, cudaEventRecord(ev[3], h->stream), "event");
         bt.group_variant = 0;
         ck(h, launch_group(ctx, bt, hp, h->stream), "k_group launch");
         ck(h, cudaEventRecord(ev[4], h->stream), "event");
         if (!ck(h, cudaEventSynchronize(ev[4]), "autotune")) break;
         float ms[4];
         for (int k = 0; k < 4; k++) cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]);
         t[c][0][1] += ms[0]; t[c][0][0] += ms[1]; t[c][1][1] += ms[2]; t[c][1][0] += ms[3];
      }
   }
   for (auto &e : ev) cudaEventDestroy(e);
   for (int sp = 0; sp < h->nspin; sp++) ck(h, cudaMemsetAsync(h->team->K[sp].p, 0, h->FP_size * 8, h->stream), "K zero");
   ck(h, cudaStreamSynchronize(h->stream), "autotune");
   if (h->err) return h->err;
   for (int c = 0; c < 256; c++) {
      if (!seen[c]) continue;
      h->tune_prim[c] = (alt_p[c] && t[c][0][1] < t[c][0][0]) ? 1 : 0;
      h->tune_group[c] = (alt_g[c] && t[c][1][1] < t[c][1][0]) ? 1 : 0;
   }
   if (out)
      for (int c = 0; c < 256; c++) { out[2 * c] = h->tune_prim[c]; out[2 * c + 1] = h->tune_group[c]; }
   return 0;
}

}  // namespace gint

using namespace gint;

// ---------------------------------------------------------------------------------------
// C-ABI (reference src/extern_functions.cpp:9-190)
// ---------------------------------------------------------------------------------------
extern "C" {

void *libgint_create_handle(void) {
   Handle *h = new Handle();
   h->prm_tmp.reserve(65536);
   for (int c = 0; c < 2 * 256; c++) h->open_of[c] = -1;
   for (int c = 0; c < 256; c++) {
      build_class_plan(c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3, h->plans[c]);
      build_vops(h->plans[c], h->vops);
      h->S_of[c] = h->plans[c].S;
      h->has_fp32[c] = class_has_fp32(c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3);
      h->tune_prim[c] = h->tune_group[c] = 0;
   }
   return h;
}

void libgint_init(void *hh) {
   Handle *h = (Handle *)hh;
   ck(h, cudaGetDevice(&h->device), "cudaGetDevice");
   // every kernel loaded once per device before any handle launches (see preload_kernels)
   static std::once_flag loaded[kMaxDevices];
   if (h->device >= 0 && h->device < kMaxDevices) {
      cudaError_t pe = cudaSuccess;
      std::call_once(loaded[h->device], [&]() { pe = preload_kernels(); });
      ck(h, pe, "kernel preload");
      if (!h->err && !group_prog(h->device)) set_error(h, 4, "kernel preload: no HRR instructions on this device");
   }
   if (!h->stream) ck(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
   for (int w = 0; w < kWorkStreams; w++) {
      if (!h->work[w]) ck(h, cudaStreamCreateWithFlags(&h->work[w], cudaStreamNonBlocking), "stream");
      if (!h->work_ev[w]) ck(h, cudaEventCreateWithFlags(&h->work_ev[w], cudaEventDisableTiming), "event");
   }
   if (!h->fork_ev) ck(h, cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming), "event");
   if (!h->noalloc_ev) ck(h, cudaEventCreateWithFlags(&h->noalloc_ev, cudaEventDisableTiming), "event");
   for (Slot &s : h->slots) {
      if (!s.ev) ck(h, cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming), "event");
      if (!s.ev_copy) ck(h, cudaEventCreateWithFlags(&s.ev_copy, cudaEventDisableTiming), "event");
   }
}

void libgint_set_Potential_Truncated(void *hh, double R_cut, double *C0, int ld_C0, int C0_size) {
   Handle *h = (Handle *)hh;
   if (!C0 || ld_C0 < 105 || ld_C0 % 105 != 0 || C0_size < 207 * ld_C0) {
      set_error(h, 2, "libgint_set_Potential_Truncated: C0 must hold 207 patches of ld_C0 = (nder+1)*105 doubles");
      return;
   }
   h->R_cut = R_cut;
   h->ld_C0 = ld_C0;
   h->C0.assign(C0, C0 + C0_size);
   h->have_pot = true;
   h->pot_dirty = true;
}

void libgint_set_hf_fac(void *hh, double fac) { ((Handle *)hh)->hf_fac = fac; }

void libgint_set_max_mem(void *hh, int max_mem) {
   Handle *h = (Handle *)hh;
   if (max_mem > 0) h->max_mem_mb = (size_t)max_mem;
}

void libgint_set_P(void *hh, double *P, int P_size) { set_P_impl((Handle *)hh, 1, P, nullptr, P_size); }

void libgint_set_P_polarized(void *hh, double *Pa, double *Pb, int P_size) { set_P_impl((Handle *)hh, 2, Pa, Pb, P_size); }

void libgint_set_K(void *hh, double *K, int K_size) { set_K_impl((Handle *)hh, 1, K, nullptr, K_size); }

void libgint_set_K_polarized(void *hh, double *Ka, double *Kb, int K_size) { set_K_impl((Handle *)hh, 2, Ka, Kb, K_size); }

void libgint_get_K(void *hh, double *K) { get_K_impl((Handle *)hh, K, nullptr); }

void libgint_get_K_polarized(void *hh, double *Ka, double *Kb) { get_K_impl((Handle *)hh, Ka, Kb); }

void libgint_set_cell(void *hh, bool periodic, double *cell_h, double *cell_i) {
   Handle *h = (Handle *)hh;
   h->periodic = periodic;   // stored; the wrap always uses the cell, as in the reference
   for (int i = 0; i < 9; i++) { h->cell[i] = cell_h[i]; h->cell[9 + i] = cell_i[i]; }
}

void libgint_set_neighs(void *hh, double *neighs, int nneighs) {
   Handle *h = (Handle *)hh;
   if (nneighs < 1 || nneighs > kMaxCell) { set_error(h, 2, "libgint_set_neighs: 1 <= nneighs <= 256"); return; }
   h->neighs.assign(neighs, neighs + 3 * (size_t)nneighs);
   h->Ng = nneighs;
   h->neighs_dirty = true;
}

void libgint_set_Atom(void *hh, int i, double *R, double *Z, int np) {
   Handle *h = (Handle *)hh;
   if (i < 0 || np < 1 || np > kMaxPrm) { set_error(h, 2, "libgint_set_Atom: 1 <= np <= 16"); return; }
   if ((size_t)i >= h->sets.size()) h->sets.resize(i + 1);
   HostSet &s = h->sets[i];
   s = HostSet();
   for (int q = 0; q < 3; q++) s.R[q] = R[q];
   s.np = np;
   for (int p = 0; p < np; p++) s.Z[p] = Z[p];
   s.defined = true;
   h->basis_dirty = true;
   h->ent_dirty = true;
}

void libgint_set_Atom_L(void *hh, int i, int l, int nl, double *K) {
   Handle *h = (Handle *)hh;
   if (i < 0 || (size_t)i >= h->sets.size() || !h->sets[i].defined) { set_error(h, 2, "libgint_set_Atom_L: set not defined"); return; }
   if (l < 0 || l > kMaxL || nl < 1 || nl > kMaxNl) { set_error(h, 2, "libgint_set_Atom_L: l <= 3 and 1 <= nl <= 4"); return; }
   HostSet &s = h->sets[i];
   if (s.nL >= 8) { set_error(h, 2, "libgint_set_Atom_L: too many l entries in one set"); return; }
   const int np = s.np;
   std::vector<double> Kn((size_t)nl * np);
   for (int c = 0; c < nl; c++) {
      // renormalisation of the reference (src/extern_functions.cpp:95-136)
      const double *Kr = K + (size_t)c * np;
      double ans = 0.0;
      for (int a = 0; a < np; a++) for (int b = 0; b < np; b++) ans += Kr[a] * Kr[b] / std::pow(s.Z[a] + s.Z[b], 1.5 + l);
      ans *= std::pow(M_PI, 1.5) / std::pow(2.0, l);
      double nrm = std::sqrt(ans);
      for (int p = 0; p < np; p++) Kn[(size_t)c * np + p] = Kr[p] / nrm;
   }
   s.l[s.nL] = l; s.nl[s.nL] = nl; s.K[s.nL] = Kn; s.nL++;
   h->basis_dirty = true;
   h->ent_dirty = true;
}

void libgint_set_AtomInfo(void *hh, int i, double *R, double *Z, int np, int lmin, int Lmax, int *nl, double *K) {
   libgint_set_Atom(hh, i, R, Z, np);
   int k_offset = 0;
   for (int l = lmin; l < Lmax; l++) {
      libgint_set_Atom_L(hh, i, l, nl[l - lmin], &K[k_offset]);
      k_offset += nl[l - lmin] * np;
   }
}

void libgint_add_prm(void *hh, int ipa, int ipb, int ipc, int ipd) {
   Handle *h = (Handle *)hh;
   h->prm_tmp.push_back(((uint32_t)ipa << 24) | ((uint32_t)ipb << 16) | ((uint32_t)ipc << 8) | (uint32_t)ipd);
}

static void add_shell_general(Handle *h, const int idx[4], int n1, int n2);

void libgint_add_shell(void *hh, int i, int j, int k, int l, int n1, int n2) {
   Handle *h = (Handle *)hh;
   const size_t np = h->prm_tmp.size();
   const double bound = h->next_bound;
   h->next_bound = HUGE_VAL;        // a bound applies to one add_shell
   if (np == 0) return;
   const int ns = (int)h->sets.size();
   if ((unsigned)i >= (unsigned)ns || (unsigned)j >= (unsigned)ns || (unsigned)k >= (unsigned)ns ||
       (unsigned)l >= (unsigned)ns || (unsigned)n1 >= (unsigned)h->Ng || (unsigned)n2 >= (unsigned)h->Ng) {
      set_error(h, 2, "libgint_add_shell: set or image index out of range");
      h->prm_tmp.clear();
      return;
   }
   ensure_ent_base(h);
   const Handle::SetFast fa = h->fast[i], fb = h->fast[j], fc = h->fast[k], fd = h->fast[l];
   // every primitive index must lie inside its set (the kernels index exponents with them)
   unsigned ma = 0, mb = 0, mc = 0, md = 0;
   const uint32_t *pc = h->prm_tmp.data();
   for (size_t p = 0; p < np; p++) {
      const uint32_t c = pc[p];
      ma = std::max(ma, c >> 24); mb = std::max(mb, (c >> 16) & 255u);
      mc = std::max(mc, (c >> 8) & 255u); md = std::max(md, c & 255u);
   }
   if ((int)ma >= fa.np || (int)mb >= fb.np || (int)mc >= fc.np || (int)md >= fd.np) {
      set_error(h, 2, "libgint_add_prm: primitive index out of range");
      h->prm_tmp.clear();
      return;
   }
   if (fa.nL == 1 && fb.nL == 1 && fc.nL == 1 && fd.nL == 1) {
      h->next_bound = bound;
      const int cl = shell_qclass(h, cls_of(fa.l0, fb.l0, fc.l0, fd.l0));
      h->next_bound = HUGE_VAL;
      OpenGroup *og = open_group(h, cl);
      if (!og) { set_error(h, 2, "libgint_add_shell: too many l-combinations in one set quartet"); h->prm_tmp.clear(); return; }
      og->bound = std::max(og->bound, bound);
      ClassQ &Q = h->q[cl];
      ShellRec sr;
      sr.ent[0] = (uint32_t)fa.ent; sr.ent[1] = (uint32_t)fb.ent; sr.ent[2] = (uint32_t)fc.ent; sr.ent[3] = (uint32_t)fd.ent;
      sr.prm_off = (uint32_t)Q.prm.size();
      sr.nprm = (uint32_t)np;
      sr.n1 = (uint16_t)n1; sr.n2 = (uint16_t)n2;
      sr.group = 0;
      const uint32_t sid = (uint32_t)Q.shells.size();
      Q.prm.append(pc, np);
      Q.prm_shell.fill(np, sid);
      Q.shells.push_back(sr);
      h->prm_tmp.clear();
      return;
   }
   const int idx[4] = {i, j, k, l};
   h->next_bound = bound;
   add_shell_general(h, idx, n1, n2);
   h->next_bound = HUGE_VAL;
}

static void add_shell_general(Handle *h, const int idx[4], int n1, int n2) {
   const HostSet *S4[4] = {&h->sets[idx[0]], &h->sets[idx[1]], &h->sets[idx[2]], &h->sets[idx[3]]};
   const uint32_t np = (uint32_t)h->prm_tmp.size();
   for (int a = 0; a < S4[0]->nL; a++) for (int b = 0; b < S4[1]->nL; b++)
   for (int c = 0; c < S4[2]->nL; c++) for (int d = 0; d < S4[3]->nL; d++) {
      const int cl = shell_qclass(h, cls_of(S4[0]->l[a], S4[1]->l[b], S4[2]->l[c], S4[3]->l[d]));
      OpenGroup *og = open_group(h, cl);
      if (!og) { set_error(h, 2, "libgint_add_shell: too many l-combinations in one set quartet"); break; }
      og->bound = std::max(og->bound, h->next_bound);
      ClassQ &Q = h->q[cl];
      ShellRec sr;
      const int li[4] = {a, b, c, d};
      for (int q = 0; q < 4; q++) sr.ent[q] = (uint32_t)(h->ent_base[idx[q]] + li[q]);
      sr.prm_off = (uint32_t)Q.prm.size();
      sr.nprm = np;
      sr.n1 = (uint16_t)n1; sr.n2 = (uint16_t)n2;
      sr.group = 0;
      const uint32_t sid = (uint32_t)Q.shells.size();
      Q.prm.append(h->prm_tmp.data(), np);
      Q.prm_shell.fill(np, sid);
      Q.shells.push_back(sr);
   }
   h->prm_tmp.clear();
}

void libgint_add_cell(void *hh) { (void)hh; }

void libgint_add_qrt(void *hh, int la, int lb, int lc, int ld, int nla, int nlb, int nlc, int nld) {
   Handle *h = (Handle *)hh;
   if (la < 0 || lb < 0 || lc < 0 || ld < 0 || la > kMaxL || lb > kMaxL || lc > kMaxL || ld > kMaxL ||
       nla < 1 || nlb < 1 || nlc < 1 || nld < 1 || nla > kMaxNl || nlb > kMaxNl || nlc > kMaxNl || nld > kMaxNl) {
      set_error(h, 2, "libgint_add_qrt: l <= 3 and 1 <= nl <= 4");
      return;
   }
   // the class's FP64 group, and its FP32 group if FP32 shell quartets were added
   const int c = cls_of(la, lb, lc, ld);
   OpenGroup *og = open_group(h, c);
   if (!og) { set_error(h, 2, "libgint_add_qrt: too many l-combinations in one set quartet"); return; }
   if (og->have_qrt) { set_error(h, 2, "libgint_add_qrt: the same l-combination twice in one set quartet"); return; }
   OpenGroup *o32 = h->open_of[c + kFp32] >= 0 ? &h->open[h->open_of[c + kFp32]] : nullptr;
   for (OpenGroup *g : {og, o32}) {
      if (!g) continue;
      g->nl[0] = (uint8_t)nla; g->nl[1] = (uint8_t)nlb; g->nl[2] = (uint8_t)nlc; g->nl[3] = (uint8_t)nld;
      g->have_qrt = true;
   }
}

void libgint_add_qrtt(void *hh, double symm_fac, int la, int lb, int lc, int ld, int inla, int inlb, int inlc, int inld,
                      int ld_ac, int ld_ad, int ld_bc, int ld_bd, unsigned int off_ac, unsigned int off_ad,
                      unsigned int off_bc, unsigned int off_bd, bool Tac, bool Tad, bool Tbc, bool Tbd) {
   Handle *h = (Handle *)hh;
   (void)inla; (void)inlb; (void)inlc; (void)inld;
   if (ld_ac < 0 || ld_ad < 0 || ld_bc < 0 || ld_bd < 0 || ld_ac > 255 || ld_ad > 255 || ld_bc > 255 || ld_bd > 255) {
      set_error(h, 2, "libgint_add_qrtt: leading dimensions must be < 256");
      return;
   }
   // symmetry factor encoding of the reference (src/libGint.cpp:262-267)
   unsigned idx_fac = 0;
   if (symm_fac < 0.1) idx_fac = 4;
   else if (symm_fac < 0.3) idx_fac = 3;
   else if (symm_fac < 0.75) idx_fac = 2;
   else if (symm_fac < 1.5) idx_fac = 1;
   if (la < 0 || lb < 0 || lc < 0 || ld < 0 || la > kMaxL || lb > kMaxL || lc > kMaxL || ld > kMaxL) {
      set_error(h, 2, "libgint_add_qrtt: l <= 3");
      return;
   }
   const int cl = cls_of(la, lb, lc, ld);
   OpenGroup *og = open_group(h, cl);
   if (!og) { set_error(h, 2, "libgint_add_qrtt: too many l-combinations in one set quartet"); return; }
   OpenGroup *o32 = h->open_of[cl + kFp32] >= 0 ? &h->open[h->open_of[cl + kFp32]] : nullptr;
   QrttRec r;
   r.off[0] = off_ac; r.off[1] = off_ad; r.off[2] = off_bc; r.off[3] = off_bd;
   r.ld[0] = (uint8_t)ld_ac; r.ld[1] = (uint8_t)ld_ad; r.ld[2] = (uint8_t)ld_bc; r.ld[3] = (uint8_t)ld_bd;
   r.T = (uint8_t)((Tac ? 1 : 0) | (Tad ? 2 : 0) | (Tbc ? 4 : 0) | (Tbd ? 8 : 0));
   r.idx_fac = (uint8_t)idx_fac;
   r.pad[0] = r.pad[1] = 0;
   h->q[cl].qrtts.push_back(r);
   og->nq++;
   if (o32) { h->q[cl + kFp32].qrtts.push_back(r); o32->nq++; }   // the FP32 group updates the same rows
}

}  // extern "C"

namespace gint {

// Primitive-target products per contraction row above which a group is split (see commit_group).
constexpr size_t kChunkWork = 4096;

// Commits the group of one set quartet and queue class: its shell quartets [shell0, end of the
// shell queue), primitives [prm0, end) and contraction rows [qrtt0, qrtt0 + nrows). The group
// kernels give each contraction row to one lane (or warp), which contracts every primitive of every
// shell of the group, so one heavy group keeps one lane busy long after the rest of the GPU has
// finished (a (pp|ps) group of 8-primitive sets holds up to 8192 primitive quartets per image
// pair). A group with more than kChunkWork primitive-target products per row is therefore
// committed as several groups over consecutive chunks of its primitives: each chunk gets shell
// records of its own that cover sub-ranges of the shells' primitive lists (the original records
// stay for the primitive kernel) and its own copy of the rows. Contraction, HRR, spherical
// transform and K update are linear, so the chunks' K updates add up to the group's.
static void commit_group(Handle *h, ClassQ &Q, int qcls, uint32_t shell0, uint32_t qrtt0, size_t prm0,
                         const uint8_t nl[4], int nrows, double bound) {
   const uint32_t nshell = (uint32_t)Q.shells.size() - shell0;
   const size_t nprm = Q.prm.size() - prm0;
   const size_t S = (size_t)h->S_of[qcls & 255];
   const size_t cap = std::max<size_t>(32, kChunkWork / std::max<size_t>(S, 1));
   size_t recs = nprm * 8 + (size_t)nshell * sizeof(ShellRec);
   // every record of the set quartet's shells names its group (the primitive kernel reads the
   // first group's flag on an incremental replay)
   const uint32_t first_group = (uint32_t)Q.groups.size();
   for (uint32_t si = shell0; si < shell0 + nshell; si++) Q.shells.data()[si].group = first_group;
   auto push_group = [&](uint32_t sh_off, uint32_t nsh, uint32_t q_off) {
      GroupRec g;
      g.shell_off = sh_off; g.nshell = nsh; g.qrtt_off = q_off;
      for (int q = 0; q < 4; q++) g.nl[q] = nl[q];
      g.bound = bound < 3.0e38 ? (float)bound : INFINITY;
      for (uint32_t si = sh_off; si < sh_off + nsh; si++) Q.shells.data()[si].group = (uint32_t)Q.groups.size();
      Q.groups.push_back(g);
      recs += sizeof(GroupRec) + (size_t)nrows * sizeof(QrttRec);
   };
   if (nprm <= cap) {
      push_group(shell0, nshell, qrtt0);
   } else {
      QrttRec rows[kMaxNl * kMaxNl * kMaxNl * kMaxNl];
      std::memcpy(rows, Q.qrtts.data() + qrtt0, sizeof(QrttRec) * (size_t)nrows);
      uint32_t chunk_shell0 = (uint32_t)Q.shells.size(), q_off = qrtt0;
      size_t in_chunk = 0;
      for (uint32_t si = shell0; si < shell0 + nshell; si++) {
         const ShellRec sr = Q.shells.data()[si];
         for (uint32_t p = 0; p < sr.nprm;) {
            const uint32_t take = (uint32_t)std::min<size_t>(sr.nprm - p, cap - in_chunk);
            ShellRec c = sr;
            c.prm_off = sr.prm_off + p;
            c.nprm = take;
            Q.shells.push_back(c);
            recs += sizeof(ShellRec);
            p += take;
            in_chunk += take;
            if (in_chunk == cap) {
               push_group(chunk_shell0, (uint32_t)Q.shells.size() - chunk_shell0, q_off);
               chunk_shell0 = (uint32_t)Q.shells.size();
               in_chunk = 0;
               q_off = (uint32_t)Q.qrtts.size();
               Q.qrtts.append(rows, (size_t)nrows);
            }
         }
      }
      if (in_chunk > 0) push_group(chunk_shell0, (uint32_t)Q.shells.size() - chunk_shell0, q_off);
      else Q.qrtts.resize(q_off);   // the last copy of the rows has no chunk
   }
   if (!Q.active) { Q.active = true; h->active.push_back(qcls); }
   h->pend_prims += nprm;
   h->pend_ac += nprm * S;
   h->pend_rec += recs;
}

}  // namespace gint

extern "C" {

void libgint_add_set(void *hh) {
   Handle *h = (Handle *)hh;
   for (int o = 0; o < h->nopen; o++) {
      OpenGroup &og = h->open[o];
      h->open_of[og.cls] = -1;
      ClassQ &Q = h->q[og.cls];
      const uint32_t nshell = (uint32_t)Q.shells.size() - og.shell_off;
      const int nrows = og.nl[0] * og.nl[1] * og.nl[2] * og.nl[3];
      if (nshell == 0 || !og.have_qrt || og.nq != nrows) {
         // nothing to compute for this class, or an inconsistent stream: roll the group back
         if (nshell && (!og.have_qrt || og.nq != nrows))
            set_error(h, 2, "libgint_add_set: add_qrtt count differs from nla*nlb*nlc*nld");
         Q.prm.resize(og.prm_off);
         Q.prm_shell.resize(og.prm_off);
         Q.shells.resize(og.shell_off);
         Q.qrtts.resize(og.qrtt_off);
         continue;
      }
      commit_group(h, Q, og.cls, og.shell_off, og.qrtt_off, og.prm_off, og.nl, nrows, og.bound);
   }
   h->nopen = 0;
   const size_t budget = slot_budget_bytes(h);
   if (h->pend_ac * 8 > budget * 7 / 10 || h->pend_rec > budget * 3 / 10) flush(h);
}

// The add_prm / add_shell / add_qrt / add_qrtt / add_set stream of n set quartets in one call,
// processed exactly as those calls made in order (same checks, same errors). Per set quartet q:
// sets[4q..4q+3]; shell_count[q] image pairs, each with shell_images (n1, n2) and prm_count
// primitive quartets taken in order from prm_codes (ipa<<24 | ipb<<16 | ipc<<8 | ipd);
// qrt_count[q] l-combinations, each a qrt record (la, lb, lc, ld, nla, nlb, nlc, nld) followed by
// its nla*nlb*nlc*nld contraction rows in lexicographic order: qrtt_fac, qrtt_ld (4), qrtt_off (4)
// and qrtt_T (bit0 Tac, bit1 Tad, bit2 Tbc, bit3 Tbd).
int libgint_add_set_quartets(void *hh, int n, const int *sets, const int *shell_count, const int *shell_images,
                             const int *prm_count, const unsigned int *prm_codes, const int *qrt_count,
                             const int *qrt, const double *qrtt_fac, const int *qrtt_ld,
                             const unsigned int *qrtt_off, const unsigned char *qrtt_T) {
   Handle *h = (Handle *)hh;
   ensure_ent_base(h);
   const int nsets = (int)h->sets.size();
   size_t ish = 0, ip = 0, iqrt = 0, ir = 0;
   for (int q = 0; q < n; q++) {
      const int *s4 = sets + 4 * (size_t)q;
      // Fast path: one l-combination on four single-l sets, every index in range and nothing
      // pending from earlier per-item calls. Everything is checked before anything is appended,
      // so the result is the per-item path's; any other set quartet takes the per-item path below.
      if (qrt_count[q] == 1 && h->nopen == 0 && h->prm_tmp.empty()) {
         const int *r = qrt + 8 * iqrt;
         bool ok = true;
         for (int k = 0; k < 4; k++) ok = ok && (unsigned)s4[k] < (unsigned)nsets && h->fast[s4[k]].nL == 1 &&
                                           h->fast[s4[k]].l0 == r[k] && r[4 + k] >= 1 && r[4 + k] <= kMaxNl;
         const int nrow = ok ? r[4] * r[5] * r[6] * r[7] : 0;
         size_t jp = ip;
         if (ok) {
            const Handle::SetFast fa = h->fast[s4[0]], fb = h->fast[s4[1]], fc = h->fast[s4[2]], fd = h->fast[s4[3]];
            for (int k = 0; k < shell_count[q] && ok; k++) {
               const size_t sh = ish + k;
               ok = (unsigned)shell_images[2 * sh] < (unsigned)h->Ng && (unsigned)shell_images[2 * sh + 1] < (unsigned)h->Ng;
               for (int t = 0; t < prm_count[sh] && ok; t++) {
                  const uint32_t c = prm_codes[jp + t];
                  ok = (int)(c >> 24) < fa.np && (int)((c >> 16) & 255u) < fb.np && (int)((c >> 8) & 255u) < fc.np &&
                       (int)(c & 255u) < fd.np;
               }
               jp += (size_t)std::max(prm_count[sh], 0);
            }
            for (int t = 0; t < nrow && ok; t++)
               for (int u = 0; u < 4; u++) ok = ok && qrtt_ld[4 * (ir + t) + u] >= 0 && qrtt_ld[4 * (ir + t) + u] <= 255;
         }
         if (ok) {
            const Handle::SetFast fa = h->fast[s4[0]], fb = h->fast[s4[1]], fc = h->fast[s4[2]], fd = h->fast[s4[3]];
            const int cl = cls_of(fa.l0, fb.l0, fc.l0, fd.l0);
            ClassQ &Q = h->q[cl];
            const uint32_t shell0 = (uint32_t)Q.shells.size(), qrtt0 = (uint32_t)Q.qrtts.size();
            const size_t prm0 = Q.prm.size();
            for (int k = 0; k < shell_count[q]; k++, ish++) {
               const int np = prm_count[ish];
               if (np > 0) {
                  ShellRec sr;
                  sr.ent[0] = (uint32_t)fa.ent; sr.ent[1] = (uint32_t)fb.ent; sr.ent[2] = (uint32_t)fc.ent; sr.ent[3] = (uint32_t)fd.ent;
                  sr.prm_off = (uint32_t)Q.prm.size();
                  sr.nprm = (uint32_t)np;
                  sr.n1 = (uint16_t)shell_images[2 * ish]; sr.n2 = (uint16_t)shell_images[2 * ish + 1];
                  sr.group = 0;
                  const uint32_t sid = (uint32_t)Q.shells.size();
                  Q.prm.append(prm_codes + ip, (size_t)np);
                  Q.prm_shell.fill((size_t)np, sid);
                  Q.shells.push_back(sr);
               }
               ip += (size_t)std::max(np, 0);
            }
            for (int t = 0; t < nrow; t++, ir++) {
               const double f = qrtt_fac[ir];
               QrttRec rr;
               for (int u = 0; u < 4; u++) { rr.off[u] = qrtt_off[4 * ir + u]; rr.ld[u] = (uint8_t)qrtt_ld[4 * ir + u]; }
               rr.T = (uint8_t)(qrtt_T[ir] & 15);
               rr.idx_fac = (uint8_t)(f < 0.1 ? 4 : (f < 0.3 ? 3 : (f < 0.75 ? 2 : (f < 1.5 ? 1 : 0))));
               rr.pad[0] = rr.pad[1] = 0;
               Q.qrtts.push_back(rr);
            }
            iqrt++;
            const uint32_t nshell = (uint32_t)Q.shells.size() - shell0;
            if (nshell > 0) {
               uint8_t nl4[4];
               for (int u = 0; u < 4; u++) nl4[u] = (uint8_t)r[4 + u];
               commit_group(h, Q, cl, shell0, qrtt0, prm0, nl4, nrow, HUGE_VAL);
            } else {
               Q.qrtts.resize(qrtt0);   // nothing to compute: the group rolls back, as in add_set
            }
            const size_t budget = slot_budget_bytes(h);
            if (h->pend_ac * 8 > budget * 7 / 10 || h->pend_rec > budget * 3 / 10) flush(h);
            continue;
         }
      }
      for (int k = 0; k < shell_count[q]; k++, ish++) {
         const int np = prm_count[ish];
         h->prm_tmp.assign(prm_codes + ip, prm_codes + ip + np);
         ip += (size_t)np;
         libgint_add_shell(h, s4[0], s4[1], s4[2], s4[3], shell_images[2 * ish], shell_images[2 * ish + 1]);
      }
      for (int t = 0; t < qrt_count[q]; t++, iqrt++) {
         const int *r = qrt + 8 * iqrt;
         libgint_add_qrt(h, r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]);
         const int na = std::max(r[4], 0), nb = std::max(r[5], 0), nc = std::max(r[6], 0), nd = std::max(r[7], 0);
         for (int ia = 0; ia < na; ia++) for (int ib = 0; ib < nb; ib++)
         for (int ic = 0; ic < nc; ic++) for (int id = 0; id < nd; id++, ir++) {
            const int *l4 = qrtt_ld + 4 * ir;
            const unsigned int *o4 = qrtt_off + 4 * ir;
            const unsigned char T = qrtt_T[ir];
            libgint_add_qrtt(h, qrtt_fac[ir], r[0], r[1], r[2], r[3], ia, ib, ic, id, l4[0], l4[1], l4[2], l4[3],
                             o4[0], o4[1], o4[2], o4[3], (T & 1) != 0, (T & 2) != 0, (T & 4) != 0, (T & 8) != 0);
         }
      }
      libgint_add_set(h);
   }
   return h->err;
}

void libgint_dispatch(void *hh) { flush((Handle *)hh); }

// Mixed precision (no counterpart in the reference): shell quartets whose Schwarz bound
// sqrt((ab|ab)(cd|cd)) max|P| is below thr run G_m, VRR, contraction, HRR and the spherical
// transform in FP32 (classes with la+lb+lc+ld <= 3; the others, the screening decisions and the K
// update stay FP64). thr <= 0 turns it off (the default). Applies to the add_shell calls that follow.
void libgint_set_fp32_threshold(void *hh, double thr) { ((Handle *)hh)->fp32_thr = thr > 0.0 ? thr : 0.0; }

// The Schwarz bound of the next add_shell's shell quartet (used by the mixed-precision threshold).
void libgint_add_shell_bound(void *hh, double bound) { ((Handle *)hh)->next_bound = bound; }

int libgint_last_error(void *hh) { return ((Handle *)hh)->err; }

// The tables the engine builds on the host (for tests): Boys table (121*28), c2s for l<=3
// (4*70, row-major [m][cartesian] per l), patch maps (2*128*128 bytes), per-patch (B,W) (207*4).
void libgint_host_tables(double *ftable, double *c2s, unsigned char *lut, double *bw) {
   std::vector<double> ft;
   make_boys_table(ft);
   std::memcpy(ftable, ft.data(), ft.size() * 8);
   double c[4][70];
   make_c2s(c);
   std::memcpy(c2s, c, sizeof(c));
   std::vector<uint8_t> l;
   std::vector<double> b;
   make_patch_tables(l, b);
   std::memcpy(lut, l.data(), l.size());
   std::memcpy(bw, b.data(), b.size() * 8);
}

// Record the device batches of the following K build(s) so that libgint_replay can recompute
// K for a new P without the add_* stream (on = 1 starts a new recording, 2 one whose batches are
// merged into one segment per class when it stops, 0 stops).
void libgint_record(void *hh, int on) {
   Handle *h = (Handle *)hh;
   if (on) {
      drain(h);
      drop_graph(h);
      for (auto &rb : h->recs) { release(rb.rec); release(rb.gbuf); }
      h->recs.clear();
   } else {
      flush(h);
      // the streaming slots' buffers are not needed to replay; release them, so that a recording's
      // replays hold the recorded batches and the replay buffers only (a streamed build allocates
      // them again)
      if (!h->err && ck(h, cudaStreamSynchronize(h->stream), "record")) {
         for (Slot &sl : h->slots) {
            if (sl.busy) { ck(h, cudaEventSynchronize(sl.ev), "slot wait"); sl.busy = false; }
            sl.copy_busy = false;
            release(sl.rec); release(sl.ac); release(sl.gscr);
         }
      }
      if (h->merge_rec) merge_recording(h);
      record_group_pmax(h);
   }
   h->recording = on != 0;
   if (on) h->merge_rec = on == 2;
   h->rec_gen++;
}

double libgint_replay(void *hh) { return replay_impl((Handle *)hh, nullptr); }

// Incremental K update from the recorded quartet list (no counterpart in the reference): with the
// current P = dP (libgint_set_P) and K = the previous K (libgint_set_K), adds K(dP) to K without
// zeroing it, skipping every set quartet whose recorded bound scaled by max|dP| / max|P_recorded|
// over the P blocks it reads is below eps (and the ones dP does not touch). The SCF loop's
// K_k = K_{k-1} + K(P_k - P_{k-1}). Returns the device time in ms, like libgint_replay.
double libgint_replay_incremental(void *hh, double eps) {
   return replay_impl((Handle *)hh, nullptr, nullptr, eps < 0.0 ? 0.0 : eps);
}

// The per-class kernel choice (no counterpart in the reference): libgint_autotune times both
// primitive kernels and both group kernels of every class on the recorded quartet list (after
// libgint_record and libgint_set_P) and keeps the faster ones for every following launch;
// out[2c], out[2c+1] (if out is given) receive class c's choices. libgint_set_tuning installs a
// table of the same layout (e.g. one measured earlier); libgint_get_tuning reads the current one.
int libgint_autotune(void *hh, int *out) { return autotune_impl((Handle *)hh, out); }

void libgint_set_tuning(void *hh, const int *in) {
   Handle *h = (Handle *)hh;
   drop_graph(h);
   for (int c = 0; c < 256; c++) {
      h->tune_prim[c] = in[2 * c] ? 1 : 0;
      h->tune_group[c] = in[2 * c + 1] ? 1 : 0;
   }
}

void libgint_get_tuning(void *hh, int *out) {
   Handle *h = (Handle *)hh;
   for (int c = 0; c < 256; c++) { out[2 * c] = h->tune_prim[c]; out[2 * c + 1] = h->tune_group[c]; }
}

// Recompute K from the recorded quartet list into caller-owned device buffers, without any
// device allocation: the primitive-quartet intermediates and the HRR workspace live in the
// library's fixed device scratch (64 MiB) instead of buffers allocated by the handle. For
// callers that cannot call cudaMalloc while building K. Every recorded class segment must fit
// the scratch (record with a small libgint_set_max_mem, e.g. 150 MB, to keep batches small).
// K_dev (K_size doubles, the P_size of the recorded build) is zeroed and then accumulated on
// `stream` (the handle's stream if null), after the work already queued on the handle's stream
// (the uploads of the recording); the call returns after launching. One density per call: a
// spin-polarised caller makes one call per spin. Calls that overlap on the GPU share the scratch
// and race. The first call on a device looks up the scratch address; make it before any stream
// capture. Returns 0, or the handle's error code.
int libgint_replay_noalloc(void *hh, const double *P_dev, double *K_dev, size_t K_size, void *stream) {
   Handle *h = (Handle *)hh;
   if (h->err) return h->err;
   if (h->recs.empty() || !h->plans_ready || h->basis_dirty || h->pot_dirty || h->neighs_dirty || !h->d_err.p) {
      set_error(h, 4, "libgint_replay_noalloc: record a K build (libgint_record) first");
      return h->err;
   }
   if (!P_dev || !K_dev || K_size == 0) {
      set_error(h, 2, "libgint_replay_noalloc: P_dev, K_dev and K_size must be given");
      return h->err;
   }
   if (K_size != h->FP_size) {
      set_error(h, 2, "libgint_replay_noalloc: K_size must be the P_size of the recorded K build");
      return h->err;
   }
   // the handle's device holds the recording, the plans and the scratch this call uses
   use_device(h);
   if (h->err) return h->err;
   double *scr = nullptr;
   if (!ck(h, noalloc_scratch(&scr), "libgint_replay_noalloc: scratch lookup")) return h->err;
   // every class segment must fit: image-summed targets [nprm][S], then the HRR workspace
   for (auto &rb : h->recs) {
      for (auto &g : rb.segs) {
         const ClassPlan &hp = h->plans[g.c & 255];
         int a = 0, b = 0;
         const size_t ac = ((size_t)g.nprm * hp.S + 31) & ~(size_t)31;
         const size_t need = ac + group_global_scratch(hp, &a, &b);
         if (need > kNoAllocScratchDoubles) {
            char msg[256];
            std::snprintf(msg, sizeof(msg), "libgint_replay_noalloc: a recorded batch of class (%d%d|%d%d) needs %zu "
                          "doubles of scratch, the maximum is %zu; record with a smaller libgint_set_max_mem",
                          (g.c >> 6) & 3, (g.c >> 4) & 3, (g.c >> 2) & 3, g.c & 3, need, kNoAllocScratchDoubles);
            set_error(h, 5, msg);
            return h->err;
         }
      }
   }
   cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
   // the recorded batches' uploads (queued on the handle's stream by the recording build) come first
   if (st != h->stream) {
      if (!ck(h, cudaEventRecord(h->noalloc_ev, h->stream), "libgint_replay_noalloc: event record") ||
          !ck(h, cudaStreamWaitEvent(st, h->noalloc_ev, 0), "libgint_replay_noalloc: stream wait"))
         return h->err;
   }
   DevCtx ctx = make_ctx(h);
   ctx.nspin = 1;
   ctx.P[0] = P_dev; ctx.P[1] = nullptr;
   ctx.K[0] = K_dev; ctx.K[1] = nullptr;
   ctx.FP_size = K_size;
   ctx.cnt = nullptr;
   if (!ck(h, cudaMemsetAsync(K_dev, 0, K_size * 8, st), "libgint_replay_noalloc: K zero")) return h->err;
   for (auto &rb : h->recs) {
      char *base = (char *)rb.rec.p;
      for (auto &g : rb.segs) {
         const ClassPlan &hp = h->plans[g.c & 255];
         BatchArgs bt;
         std::memset(&bt, 0, sizeof(bt));
         bt.cls = g.c & 255;
         bt.fp32 = g.c >= kFp32;
         bt.prim_variant = h->tune_prim[g.c & 255];
         bt.group_variant = h->tune_group[g.c & 255];
         bt.plan = (const ClassPlan *)h->d_plans.p + (g.c & 255);
         bt.prm = (const uint32_t *)(base + g.o_prm);
         bt.prm_shell = (const uint32_t *)(base + g.o_ps);
         bt.shells = (const ShellRec *)(base + g.o_sh);
         bt.groups = (const GroupRec *)(base + g.o_g);
         bt.qrtts = (const QrttRec *)(base + g.o_q);
         bt.rowgrp = (const uint32_t *)(base + g.o_rg);
         bt.nprm = g.nprm; bt.nshell = g.nshell; bt.ngroup = g.ngroup; bt.nqrtt = g.nqrtt;
         bt.AC = scr;                                                   // segments run in stream order
         bt.gscratch = scr + (((size_t)g.nprm * hp.S + 31) & ~(size_t)31);
         if (!ck(h, launch_prim(ctx, bt, hp, st), "libgint_replay_noalloc: k_prim launch")) return h->err;
         if (!ck(h, launch_group(ctx, bt, hp, st), "libgint_replay_noalloc: k_group launch")) return h->err;
      }
   }
   return 0;
}

// the same with the summed device time of each kernel kind: kt[0] = k_prim, kt[1] = k_group
double libgint_replay_profile(void *hh, double *kt) { return replay_impl((Handle *)hh, kt); }

// the same with the per-class split: kcls[c*2 + {0,1}] = ms of the two kernels of class c
double libgint_replay_profile_classes(void *hh, double *kt, double *kcls) { return replay_impl((Handle *)hh, kt, kcls); }

// Device event counters per class: [c*4+0] Chebyshev G_m evaluations, [1] Boys evaluations,
// [2] images through the VRR, [3] primitive quartets (c = la*64+lb*16+lc*4+ld).
void libgint_set_counters(void *hh, int on) {
   Handle *h = (Handle *)hh;
   drain(h);
   if (on) {
      if (!ensure(h, h->d_cnt, 256 * 4 * sizeof(unsigned long long), "counters")) return;
      ck(h, cudaMemset(h->d_cnt.p, 0, 256 * 4 * sizeof(unsigned long long)), "counters");
   }
   h->counting = on != 0;
}

void libgint_get_counters(void *hh, unsigned long long *out) {
   Handle *h = (Handle *)hh;
   drain(h);
   if (!h->d_cnt.p) { std::memset(out, 0, 256 * 4 * sizeof(unsigned long long)); return; }
   ck(h, cudaMemcpy(out, h->d_cnt.p, 256 * 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost), "counters");
}

// host-side totals: shells, primitive quartets, groups, flushes, kernel launches
void libgint_get_stats(void *hh, long long *out) {
   Handle *h = (Handle *)hh;
   out[0] = h->n_shells; out[1] = h->n_prims; out[2] = h->n_groups; out[3] = h->n_flush; out[4] = h->n_launch;
   out[5] = h->h2d_bytes; out[6] = h->n_shells_fp32; out[7] = h->n_prims_fp32;
}

double libgint_fp64_peak_tflops(void) { return measure_fp64_peak_tflops(); }

// Sizes of the recursion plan of one class (VRR workspace, contracted targets, HRR workspace,
// cartesian and spherical block sizes), for inspection and tests.
// Algorithmic FP64 operation counts of one class, following the reference recursion:
// out[0] per Chebyshev G_m evaluation, [1] per Boys evaluation, [2] VRR per image,
// [3] image sum per image (targets), [4] contraction per primitive and contraction row,
// [5] HRR per shell and contraction row, [6] spherical transform per row, [7] K update per row.
int libgint_plan_flops(int la, int lb, int lc, int ld, double *out) {
   ClassPlan p;
   if (!build_class_plan(la, lb, lc, ld, p)) return 0;
   auto nc = [](int l) { return (l + 1) * (l + 2) / 2; };
   const int L = p.L;
   out[0] = 2.0 * (L + 1) * 105 + 2.0 * (L + 1) * 14 + 4.0 * 13;
   out[1] = 25.0 + 3.0 * L;
   double v = 0;
   for (int b = 1; b < p.nvb; b++) {
      const VBlock &vb = p.vb[b];
      double ct;
      if (vb.c == 0) ct = (vb.a == 1) ? 3 : 7;            // VRR1 / VRR2
      else if (vb.a == 0) ct = (vb.c == 1) ? 3 : 7;       // VRR3 / VRR4
      else ct = (vb.c == 1) ? 6 : 10;                     // VRR6 / VRR5
      v += ct * vb.nelem;
   }
   out[2] = v;
   out[3] = p.S;
   out[4] = 2.0 * p.S + 3.0;
   double hrr = 0;
   for (int o = 0; o < p.nhop; o++) hrr += 2.0 * p.hop[o].nelem;
   out[5] = hrr;
   const int dims[4] = {nc(la), nc(lb), nc(lc), nc(ld)}, ls[4] = {la, lb, lc, ld};
   int cur[4] = {dims[0], dims[1], dims[2], dims[3]};
   double sph = 0;
   for (int c = 0; c < 4; c++) {
      int o[4] = {cur[0], cur[1], cur[2], cur[3]}; o[c] = 2 * ls[c] + 1;
      sph += 2.0 * o[0] * o[1] * o[2] * o[3] * dims[c];
      cur[c] = 2 * ls[c] + 1;
   }
   out[6] = sph;
   out[7] = 9.0 * p.Ns;
   return 1;
}

int libgint_plan_sizes(int la, int lb, int lc, int ld, int *out) {
   ClassPlan p;
   if (!build_class_plan(la, lb, lc, ld, p)) return 0;
   out[0] = p.V; out[1] = p.S; out[2] = p.H; out[3] = p.Nc; out[4] = p.Ns; out[5] = p.nvb; out[6] = p.nhop;
   out[7] = prim_team_size(p);
   return 1;
}

// The HRR instructions the interpreted group kernel runs for one class (host copy of the per-GPU
// table, build_group_prog): out[2i], out[2i+1] = {in1 | axis << 30, in2} of workspace element
// S + i, up to cap instructions; info[0..3] = S, H, the offset of the final cartesian block, the
// number of ket elements (the first ones; they use CD, the rest AB). Returns the number of
// instructions, -1 for an unsupported class. Needs no GPU.
int libgint_hrr_program(int la, int lb, int lc, int ld, unsigned int *out, int cap, int *info) {
   ClassPlan p;
   if (la < 0 || lb < 0 || lc < 0 || ld < 0 || la > kMaxL || lb > kMaxL || lc > kMaxL || ld > kMaxL ||
       !build_class_plan(la, lb, lc, ld, p))
      return -1;
   static std::vector<uint2> prog;
   static std::once_flag built;
   std::call_once(built, [] { build_group_prog(prog); });
   if (prog.empty()) return -1;
   const int c = la * 64 + lb * 16 + lc * 4 + ld;
   const uint32_t first = prog[c].x, end = c + 1 < 256 ? prog[c + 1].x : (uint32_t)prog.size();
   const int n = (int)(end - first);
   for (int i = 0; i < n && i < cap; i++) { out[2 * i] = prog[first + i].x; out[2 * i + 1] = prog[first + i].y; }
   int ket = 0;
   for (int o = 0; o < p.nhop; o++) if (p.hop[o].type == 0) ket += p.hop[o].nelem;
   if (info) { info[0] = p.S; info[1] = p.H; info[2] = p.out_off; info[3] = ket; }
   return n;
}

// The precompiled VRR instructions of one class (build_vops), as k_prim2 and k_prim run them
// level after level: 16-byte VOp records (engine_types.h) into vops, up to cap of them. info gets
// V, S, the number of (0|0)^(m) values at the start of the workspace, the number of targets ntg,
// then per target its workspace offset, target offset, length and (e, f) shells; info_cap >= 4 +
// 5 ntg. Returns the instruction count, -1 for an unsupported class. Needs no GPU.
int libgint_vrr_program(int la, int lb, int lc, int ld, void *vops, int cap, int *info, int info_cap) {
   ClassPlan p;
   if (la < 0 || lb < 0 || lc < 0 || ld < 0 || la > kMaxL || lb > kMaxL || lc > kMaxL || ld > kMaxL ||
       !build_class_plan(la, lb, lc, ld, p))
      return -1;
   std::vector<VOp> v;
   build_vops(p, v);
   if (vops) std::memcpy(vops, v.data(), sizeof(VOp) * std::min<size_t>(v.size(), (size_t)std::max(cap, 0)));
   if (info && info_cap >= 4 + 5 * p.ntg) {
      info[0] = p.V; info[1] = p.S; info[2] = p.vb[0].nm; info[3] = p.ntg;
      for (int t = 0; t < p.ntg; t++) {
         int *q = info + 4 + 5 * t;
         q[0] = p.tg_voff[t]; q[1] = p.tg_soff[t]; q[2] = p.tg_n[t]; q[3] = p.tg_e[t]; q[4] = p.tg_f[t];
      }
   }
   return (int)v.size();
}

const char *libgint_error_string(void *hh) { return ((Handle *)hh)->errmsg.c_str(); }

void libgint_destroy_handle(void *hh) {
   Handle *h = (Handle *)hh;
   if (!h) return;
   if (h->stream) { use_device(h); cudaStreamSynchronize(h->stream); }
   drop_graph(h);
   for (Slot &s : h->slots) {
      release(s.rec); release(s.ac); release(s.gscr);
      if (s.ev) cudaEventDestroy(s.ev);
      if (s.ev_copy) cudaEventDestroy(s.ev_copy);
   }
   for (auto &rb : h->recs) { release(rb.rec); release(rb.gbuf); }
   release(h->rec_ac); release(h->rec_gscr); release(h->d_cnt);
   DBuf *bufs[] = {&h->d_pool, &h->d_ents, &h->d_neighs, &h->d_C0, &h->d_C0f, &h->d_lut, &h->d_bw, &h->d_ft, &h->d_vops, &h->d_tmax,
                   &h->d_plans, &h->d_err};
   for (DBuf *b : bufs) release(*b);
   h->team.reset();
   for (int w = 0; w < kWorkStreams; w++) {
      if (h->work[w]) cudaStreamDestroy(h->work[w]);
      if (h->work_ev[w]) cudaEventDestroy(h->work_ev[w]);
   }
   if (h->fork_ev) cudaEventDestroy(h->fork_ev);
   if (h->noalloc_ev) cudaEventDestroy(h->noalloc_ev);
   if (h->stream) cudaStreamDestroy(h->stream);
   delete h;
}

}  // extern "C"
