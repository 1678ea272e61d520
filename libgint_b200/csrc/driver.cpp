// driver.cpp -- workload generator, C0 table fitter and C-ABI replayer.
//
// This library stands in for the caller of the libGint C-ABI (CP2K's HFX module): it builds
// seeded synthetic water systems, screens set quartets and primitive quartets, records the
// resulting add_* call stream as a compact trace, and replays that trace through any shared
// library that exports the libgint_* entry points (this engine, the CPU oracle, or the
// reference build). Every library therefore sees an identical quartet list.
//
// It also fits the truncated-Coulomb coefficient table C0 (the data the caller passes to
// libgint_set_Potential_Truncated). CP2K's own fit is not available here, so the table is
// produced from the definition of the operator:
//   G_m(T,R) = (-d/dT)^m G_0(T,R),
//   G_0(T,R) = sqrt(pi)/(4 sqrt(T)) [2 erf(sqrt T) + erf(R - sqrt T) - erf(R + sqrt T)],
// evaluated as G_m = F_m(T) - H_m(T,R) with the Boys function F_m and
//   H_m = (-1)^m / (2 4^m m!) Int_{-1}^{1} (1-u^2)^m H_{2m}(R + sqrt(T) u) exp(-(R + sqrt(T) u)^2) du
// (H_n = Hermite polynomial), then projected on the degree-13 triangular Chebyshev basis of
// each patch (patch geometry in tcg_patches.h).
#include <algorithm>
#include <array>
#include <atomic>
#include <functional>
#include <mutex>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <omp.h>
#include <string>
#include <thread>
#include <vector>

#include "tcg_patches.h"

namespace {

constexpr double kAngToBohr = 1.8897261254578281;

// ---------------------------------------------------------------------------------------
// deterministic random numbers (splitmix64 seeding + xoshiro256**)
// ---------------------------------------------------------------------------------------
struct Rng {
   uint64_t s[4];
   explicit Rng(uint64_t seed) {
      uint64_t z = seed;
      for (int i = 0; i < 4; i++) {
         z += 0x9e3779b97f4a7c15ULL;
         uint64_t x = z;
         x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
         x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
         s[i] = x ^ (x >> 31);
      }
   }
   static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
   uint64_t next() {
      uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
      s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
      return r;
   }
   double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
   double uniform(double a, double b) { return a + (b - a) * uniform(); }
   double normal() {
      double u1 = uniform(), u2 = uniform();
      if (u1 < 1e-300) u1 = 1e-300;
      return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
   }
};

// ---------------------------------------------------------------------------------------
// Boys function and the truncated-Coulomb auxiliary function (reference values for the fit)
// ---------------------------------------------------------------------------------------
void boys_all(int nmax, double T, double *F) {
   if (T < 50.0) {
      // F_m(T) = exp(-T) sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)); all terms positive
      double e = std::exp(-T);
      for (int m = 0; m <= nmax; m++) {
         double term = 1.0 / (2 * m + 1), sum = term;
         for (int k = 1; k < 2000; k++) {
            term *= 2.0 * T / (2 * m + 2 * k + 1);
            sum += term;
            if (term < 1e-18 * sum) break;
         }
         F[m] = e * sum;
      }
   } else {
      double s = std::sqrt(T), e = std::exp(-T);
      F[0] = 0.5 * std::sqrt(M_PI) * std::erf(s) / s;
      for (int m = 0; m < nmax; m++) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
   }
}

struct GaussLegendre {
   std::vector<double> x, w;
   explicit GaussLegendre(int n) : x(n), w(n) {
      for (int i = 0; i < n; i++) {
         double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0.0;
         for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; k++) { double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
         }
         double p0 = 1.0, p1 = z;
         for (int k = 2; k <= n; k++) { double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
         dp = n * (z * p1 - p0) / (z * z - 1.0);
         x[i] = z; w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
      }
   }
};

// G_m(T,R) for m = 0..nder
void tcg_exact(int nder, double T, double R, double *G, const GaussLegendre &gl) {
   double F[40];
   boys_all(nder, T, F);
   double Hm[40] = {0};
   const double Y = 13.0;
   double s = std::sqrt(T);
   double ulo, uhi;
   if (s > 0.0) { ulo = std::max(-1.0, (-Y - R) / s); uhi = std::min(1.0, (Y - R) / s); }
   else { ulo = -1.0; uhi = (std::fabs(R) < Y) ? 1.0 : -1.0; }
   if (uhi > ulo) {
      double half = 0.5 * (uhi - ulo), mid = 0.5 * (uhi + ulo);
      double I[40] = {0};
      for (size_t q = 0; q < gl.x.size(); q++) {
         double u = mid + half * gl.x[q], wq = half * gl.w[q];
         double y = R + s * u;
         double h0 = std::exp(-y * y), h1 = 2.0 * y * h0;
         double hv[2 * 40 + 2];
         hv[0] = h0; hv[1] = h1;
         for (int n = 1; n < 2 * nder; n++) hv[n + 1] = 2.0 * y * hv[n] - 2.0 * n * hv[n - 1];
         double om = 1.0, one_u2 = 1.0 - u * u;
         for (int m = 0; m <= nder; m++) { I[m] += wq * om * hv[2 * m]; om *= one_u2; }
      }
      double fact = 1.0, p4 = 1.0;
      for (int m = 0; m <= nder; m++) {
         if (m > 0) { fact *= m; p4 *= 4.0; }
         double sg = (m & 1) ? -1.0 : 1.0;
         Hm[m] = sg * I[m] / (2.0 * p4 * fact);
      }
   }
   for (int m = 0; m <= nder; m++) G[m] = F[m] - Hm[m];
}

// ---------------------------------------------------------------------------------------
// workload
// ---------------------------------------------------------------------------------------
struct SetDef {
   int kind;          // 0 = O, 1 = H
   int l, np, nl;
   std::vector<double> Z;      // exponents (descending)
   std::vector<double> Kraw;   // nl*np raw coefficients (as passed to set_Atom_L)
   std::vector<double> Knorm;  // renormalised the way the library does it
};

struct Set {
   int atom;
   int def;           // index into defs
   double R[3];       // bohr
   int bf_off;        // first basis function
};

struct SetQ {
   int i, j, k, l;
   float fac;
   uint32_t shell_begin, shell_end;
};
struct Shell {
   uint16_t n1, n2;
   uint32_t prm_begin, prm_end;
   float bound;       // the screening estimate sqrt((ab|ab)(cd|cd)) max|P| of the shell quartet
};

}  // namespace

extern "C" {

struct gd_config {
   int n_mol;
   double box_ang;
   int periodic;
   int n_img_1d;        // images per dimension (1, 3, 5, ...); Ng = n_img_1d^3
   int basis;           // 2: l<=2 sets with one contraction; 3: adds d,d,f sets, general contraction
   int n_occ;
   double rc_ang;
   double eps_schwarz;
   uint64_t seed;
   int full_enum;       // 1: all (i,j,k,l) with factor 0.25 instead of the unique quartets
   int max_prm;         // max primitives per set for the l<=3 basis (<=16)
   int max_ncontr;      // max contractions per set for the l<=3 basis (<=4)
   int setq_stride;     // > 1: keep the candidate set quartets (i,j,k,l) whose hash is setq_phase
   int setq_phase;      //      modulo setq_stride (a uniform sample of a workload too large to run whole)
   int threads;         // enumeration threads (0: all hardware threads); the result does not depend on it
   int max_images;      // > 0: keep the max_images lattice vectors nearest the origin (origin first)
};

struct gd_info {
   int n_bf, n_sets, n_atoms, Ng;
   long n_setq, n_shells, n_prims, n_qrtt;
   double rc_bohr;
   int nder, ld_C0, C0_size;
   double max_abs_P;
   long flat_size;
};

struct gd_workload {
   gd_config cfg;
   std::vector<SetDef> defs;
   std::vector<Set> sets;
   int n_bf = 0;
   double cell_h[9] = {0}, cell_i[9] = {0};
   std::vector<double> neighs;
   int Ng = 1;
   std::vector<double> P;          // dense, column-major n x n
   std::vector<double> Pflat;      // packed set-pair blocks (the layout passed to set_P)
   std::vector<uint32_t> blkoff;   // offset of block (X,Y), X >= Y, in the packed layout
   size_t flat_size = 0;
   std::vector<SetQ> setq;
   std::vector<Shell> shells;
   std::vector<uint32_t> prims;
   long n_qrtt = 0;
   std::vector<double> C0;
   int nder = 12;
   double rc_bohr = 0;
};

// ----- C0 table ------------------------------------------------------------------------
// Fit of G_k(T,R), k = 0..nder, on the 207 patches. Layout (per the reference's reader,
// src/t_c_g0_n.cpp:29-51 and :161-178): C0[patch*ld + k*105 + jl], jl running over
// (j = 0..13 outer, l = 0..13-j inner) with coefficient of T~_l(x1) T~_j(x2),
// T~_0 = 1, T~_n = sqrt(2) T_n.
int gd_tcg_table(int nder, double *out) {
   const int N = 24;   // Gauss-Chebyshev nodes per dimension
   const int ld = (nder + 1) * 105;
   GaussLegendre gl(160);
   std::vector<double> xn(N);
   for (int a = 0; a < N; a++) xn[a] = std::cos(M_PI * (a + 0.5) / N);
   std::vector<double> Tt(N * 14);
   for (int a = 0; a < N; a++) {
      double x = xn[a], t0 = 1.0, t1 = x;
      Tt[a * 14 + 0] = 1.0;
      Tt[a * 14 + 1] = std::sqrt(2.0) * t1;
      for (int n = 2; n < 14; n++) { double t2 = 2 * x * t1 - t0; t0 = t1; t1 = t2; Tt[a * 14 + n] = std::sqrt(2.0) * t2; }
   }
   std::vector<double> fv((size_t)N * N * (nder + 1));
   for (int p = 0; p < TCG_NPATCH; p++) {
      const double lo1 = tcg_patch_rect[p][0] / 128.0, hi1 = tcg_patch_rect[p][1] / 128.0;
      const double lo2 = tcg_patch_rect[p][2] / 128.0, hi2 = tcg_patch_rect[p][3] / 128.0;
      const bool low = p < TCG_NPATCH_LOW;
      for (int a = 0; a < N; a++) for (int b = 0; b < N; b++) {
         double X1 = 0.5 * (lo1 + hi1) + 0.5 * (hi1 - lo1) * xn[a];
         double X2 = 0.5 * (lo2 + hi2) + 0.5 * (hi2 - lo2) * xn[b];
         double R, T;
         if (low) { R = 11.0 * X2; double up = R * R + 11.0 * R + 50.0; T = X1 * up; }
         else { R = 11.0 / X2; double lw = R * R - 11.0 * R, up = R * R + 11.0 * R + 50.0; T = lw + X1 * (up - lw); }
         double G[40];
         tcg_exact(nder, T, R, G, gl);
         for (int k = 0; k <= nder; k++) fv[((size_t)k * N + a) * N + b] = G[k];
      }
      for (int k = 0; k <= nder; k++) {
         int jl = 0;
         for (int j = 0; j < 14; j++) for (int l = 0; l < 14 - j; l++) {
            double c = 0.0;
            for (int a = 0; a < N; a++) {
               double ta = Tt[a * 14 + l];
               double acc = 0.0;
               for (int b = 0; b < N; b++) acc += fv[((size_t)k * N + a) * N + b] * Tt[b * 14 + j];
               c += ta * acc;
            }
            out[(size_t)p * ld + k * 105 + jl] = c / (double)(N * N);
            jl++;
         }
      }
   }
   return ld;
}

// exact G_m(T,R), m = 0..nder (for tests)
void gd_tcg_exact(int nder, double T, double R, double *G) {
   static GaussLegendre gl(160);
   tcg_exact(nder, T, R, G, gl);
}

void gd_boys(int nmax, double T, double *F) { boys_all(nmax, T, F); }

// ----- workload construction -----------------------------------------------------------
static double norm_psi(const double *K, const double *z, int np, int l) {
   // same convention as the library's renormalisation (src/extern_functions.cpp:95-110)
   double ans = 0.0;
   for (int i = 0; i < np; i++) for (int j = 0; j < np; j++) ans += K[i] * K[j] / std::pow(z[i] + z[j], 1.5 + l);
   ans *= std::pow(M_PI, 1.5) / std::pow(2.0, l);
   return std::sqrt(ans);
}

static void make_def(SetDef &d, int kind, int l, int np, int nl, Rng &rng, bool general) {
   d.kind = kind; d.l = l; d.np = np; d.nl = nl;
   d.Z.resize(np);
   for (int i = 0; i < np; i++) d.Z[i] = std::exp(std::log(0.1) + rng.uniform() * (std::log(5e3) - std::log(0.1)));
   std::sort(d.Z.begin(), d.Z.end(), [](double a, double b) { return a > b; });
   d.Kraw.resize((size_t)nl * np);
   for (int c = 0; c < nl; c++) for (int i = 0; i < np; i++)
      d.Kraw[(size_t)c * np + i] = general ? rng.normal() : rng.uniform(0.1, 1.0);
   d.Knorm.resize(d.Kraw.size());
   for (int c = 0; c < nl; c++) {
      double n = norm_psi(&d.Kraw[(size_t)c * np], d.Z.data(), np, l);
      for (int i = 0; i < np; i++) d.Knorm[(size_t)c * np + i] = d.Kraw[(size_t)c * np + i] / n;
   }
}

static double min_image_dist2(const double *a, const double *b, double L, bool periodic) {
   double d2 = 0;
   for (int q = 0; q < 3; q++) {
      double d = a[q] - b[q];
      if (periodic) d -= L * std::round(d / L);
      d2 += d * d;
   }
   return d2;
}

gd_workload *gd_create(const gd_config *cfg) {
   gd_workload *w = new gd_workload();
   w->cfg = *cfg;
   Rng rng(cfg->seed);
   const bool periodic = cfg->periodic != 0;
   // ---- basis definitions (one per element kind, shared by all molecules)
   std::vector<int> O_sets, H_sets;
   auto add_def = [&](int kind, int l, int np, int nl, bool general) {
      SetDef d; make_def(d, kind, l, np, nl, rng, general);
      w->defs.push_back(d);
      return (int)w->defs.size() - 1;
   };
   if (cfg->basis == 2) {
      O_sets = {add_def(0, 0, 6, 1, false), add_def(0, 0, 1, 1, false), add_def(0, 1, 3, 1, false),
                add_def(0, 1, 1, 1, false), add_def(0, 2, 1, 1, false)};
      H_sets = {add_def(1, 0, 3, 1, false), add_def(1, 0, 1, 1, false), add_def(1, 1, 1, 1, false)};
   } else {
      int mp = cfg->max_prm > 0 ? cfg->max_prm : 16, mc = cfg->max_ncontr > 0 ? cfg->max_ncontr : 4;
      auto np_ = [&](int want) { return std::min(want, mp); };
      auto nc_ = [&](int want, int np) { return std::min(std::min(want, mc), np); };
      O_sets = {add_def(0, 0, np_(16), nc_(4, np_(16)), true), add_def(0, 0, 1, 1, true),
                add_def(0, 1, np_(8), nc_(3, np_(8)), true), add_def(0, 1, 1, 1, true),
                add_def(0, 2, np_(4), nc_(2, np_(4)), true), add_def(0, 2, 1, 1, true),
                add_def(0, 2, 1, 1, true), add_def(0, 3, 1, 1, true)};
      H_sets = {add_def(1, 0, np_(6), nc_(2, np_(6)), true), add_def(1, 0, 1, 1, true),
                add_def(1, 1, 1, 1, true)};
   }
   // ---- molecules
   const double L = cfg->box_ang;
   std::vector<std::array<double, 3>> Opos;
   std::vector<double> atoms;   // 3 per atom, angstrom
   std::vector<int> akind;
   for (int m = 0; m < cfg->n_mol; m++) {
      double o[3];
      for (int tries = 0; tries < 1000000; tries++) {
         for (int q = 0; q < 3; q++) o[q] = rng.uniform(0.0, L);
         bool ok = true;
         for (auto &p : Opos) if (min_image_dist2(o, p.data(), L, periodic) < 2.8 * 2.8) { ok = false; break; }
         if (ok) break;
      }
      Opos.push_back({o[0], o[1], o[2]});
      // random rotation from a unit quaternion
      double q0 = rng.normal(), q1 = rng.normal(), q2 = rng.normal(), q3 = rng.normal();
      double qn = std::sqrt(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
      q0 /= qn; q1 /= qn; q2 /= qn; q3 /= qn;
      double Rm[3][3] = {{1 - 2 * (q2 * q2 + q3 * q3), 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)},
                         {2 * (q1 * q2 + q0 * q3), 1 - 2 * (q1 * q1 + q3 * q3), 2 * (q2 * q3 - q0 * q1)},
                         {2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 1 - 2 * (q1 * q1 + q2 * q2)}};
      const double half = 0.5 * 104.5 * M_PI / 180.0;
      double hloc[2][3] = {{0.96 * std::sin(half), 0.0, 0.96 * std::cos(half)},
                           {-0.96 * std::sin(half), 0.0, 0.96 * std::cos(half)}};
      atoms.insert(atoms.end(), {o[0], o[1], o[2]}); akind.push_back(0);
      for (int h = 0; h < 2; h++) {
         double v[3];
         for (int r = 0; r < 3; r++) v[r] = o[r] + Rm[r][0] * hloc[h][0] + Rm[r][1] * hloc[h][1] + Rm[r][2] * hloc[h][2];
         atoms.insert(atoms.end(), {v[0], v[1], v[2]}); akind.push_back(1);
      }
   }
   // ---- sets and basis-function offsets
   int bf = 0;
   for (size_t a = 0; a < akind.size(); a++) {
      const std::vector<int> &ds = akind[a] == 0 ? O_sets : H_sets;
      for (int d : ds) {
         Set s; s.atom = (int)a; s.def = d;
         for (int q = 0; q < 3; q++) s.R[q] = atoms[a * 3 + q] * kAngToBohr;
         s.bf_off = bf;
         bf += (2 * w->defs[d].l + 1) * w->defs[d].nl;
         w->sets.push_back(s);
      }
   }
   w->n_bf = bf;
   // ---- cell and images (bohr). Rows of h are the lattice vectors.
   const double Lb = L * kAngToBohr;
   if (periodic) {
      for (int q = 0; q < 3; q++) { w->cell_h[q * 3 + q] = Lb; w->cell_i[q * 3 + q] = 1.0 / Lb; }
      int k = cfg->n_img_1d / 2;
      w->neighs = {0.0, 0.0, 0.0};
      std::vector<std::array<int, 3>> cells;
      for (int x = -k; x <= k; x++) for (int y = -k; y <= k; y++) for (int z = -k; z <= k; z++) {
         if (x == 0 && y == 0 && z == 0) continue;
         cells.push_back({x, y, z});
      }
      if (cfg->max_images > 0 && (int)cells.size() + 1 > cfg->max_images) {
         // the nearest cells (a ball of images), ties kept in enumeration order
         std::stable_sort(cells.begin(), cells.end(), [](const std::array<int, 3> &a, const std::array<int, 3> &b) {
            return a[0] * a[0] + a[1] * a[1] + a[2] * a[2] < b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
         });
         cells.resize(cfg->max_images - 1);
      }
      for (const auto &c : cells) w->neighs.insert(w->neighs.end(), {c[0] * Lb, c[1] * Lb, c[2] * Lb});
   } else {
      // a cell far larger than the system makes the minimum-image wrap the identity
      for (int q = 0; q < 3; q++) { w->cell_h[q * 3 + q] = 1024.0; w->cell_i[q * 3 + q] = 1.0 / 1024.0; }
      w->neighs = {0.0, 0.0, 0.0};
   }
   w->Ng = (int)w->neighs.size() / 3;
   // ---- density P = 2 C C^T, C orthonormal (modified Gram-Schmidt of N(0,1))
   const int n = w->n_bf, no = std::min(cfg->n_occ, n);
   std::vector<double> C((size_t)n * no);
   for (auto &x : C) x = rng.normal();
   for (int c = 0; c < no; c++) {
      double *v = &C[(size_t)c * n];
      for (int p = 0; p < c; p++) {
         const double *u = &C[(size_t)p * n];
         double d = 0; for (int i = 0; i < n; i++) d += u[i] * v[i];
         for (int i = 0; i < n; i++) v[i] -= d * u[i];
      }
      double nn = 0; for (int i = 0; i < n; i++) nn += v[i] * v[i];
      nn = std::sqrt(nn); for (int i = 0; i < n; i++) v[i] /= nn;
   }
   w->P.assign((size_t)n * n, 0.0);
   {
      // columns of P in parallel; each column sums the orbitals in the same order as a serial loop
      const int nth = cfg->threads > 0 ? cfg->threads : std::max(1, (int)std::thread::hardware_concurrency());
      std::atomic<int> next{0};
      std::vector<std::thread> th;
      for (int t = 0; t < nth; t++)
         th.emplace_back([&]() {
            for (int col; (col = next.fetch_add(1)) < n;) {
               double *Pc = &w->P[(size_t)col * n];
               for (int c = 0; c < no; c++) {
                  const double *v = &C[(size_t)c * n];
                  const double vc = 2.0 * v[col];
                  for (int r = 0; r < n; r++) Pc[r] += vc * v[r];
               }
            }
         });
      for (auto &x : th) x.join();
   }
   // ---- packed block layout: blocks (X,Y) with X >= Y, column-major, ld = functions of X
   const int S = (int)w->sets.size();
   auto nbf_of = [&](int x) { const SetDef &d = w->defs[w->sets[x].def]; return (2 * d.l + 1) * d.nl; };
   w->blkoff.assign((size_t)S * S, 0u);
   {
      size_t off = 0;
      for (int x = 0; x < S; x++) for (int y = 0; y <= x; y++) {
         w->blkoff[(size_t)x * S + y] = (uint32_t)off;
         off += (size_t)nbf_of(x) * nbf_of(y);
      }
      w->flat_size = off;
      w->Pflat.assign(off, 0.0);
      for (int x = 0; x < S; x++) for (int y = 0; y <= x; y++) {
         int nx = nbf_of(x), ny = nbf_of(y), bx = w->sets[x].bf_off, by = w->sets[y].bf_off;
         double *blk = &w->Pflat[w->blkoff[(size_t)x * S + y]];
         for (int c = 0; c < ny; c++) for (int r = 0; r < nx; r++) blk[(size_t)c * nx + r] = w->P[(size_t)(by + c) * n + bx + r];
      }
   }
   // ---- screening data
   std::vector<double> Pblk((size_t)S * S, 0.0);
   for (int a = 0; a < S; a++) for (int b = 0; b < S; b++) {
      const SetDef &da = w->defs[w->sets[a].def], &db = w->defs[w->sets[b].def];
      int na = (2 * da.l + 1) * da.nl, nb = (2 * db.l + 1) * db.nl;
      double m = 0;
      for (int i = 0; i < na; i++) for (int j = 0; j < nb; j++)
         m = std::max(m, std::fabs(w->P[(size_t)(w->sets[b].bf_off + j) * n + w->sets[a].bf_off + i]));
      Pblk[(size_t)a * S + b] = m;
   }
   w->rc_bohr = cfg->rc_ang * kAngToBohr;
   const double eps = cfg->eps_schwarz;
   // per-set coefficient magnitude per primitive (max over contractions)
   std::vector<std::vector<double>> cmax(S);
   for (int a = 0; a < S; a++) {
      const SetDef &d = w->defs[w->sets[a].def];
      cmax[a].assign(d.np, 0.0);
      for (int c = 0; c < d.nl; c++) for (int i = 0; i < d.np; i++)
         cmax[a][i] = std::max(cmax[a][i], std::fabs(d.Knorm[(size_t)c * d.np + i]));
   }
   // pair lists: for (a,b,n1) the primitive pair estimates q_ij ~ sqrt((ab|ab))
   struct Pair { int n1; double Q; double ctr[3]; double rad; std::vector<float> q; };
   auto pair_of = [&](int a, int b, int n1, Pair &pr) {
      const Set &sa = w->sets[a], &sb = w->sets[b];
      const SetDef &da = w->defs[sa.def], &db = w->defs[sb.def];
      double Bp[3], AB2 = 0;
      for (int q = 0; q < 3; q++) {
         double d = sb.R[q] - sa.R[q];
         if (periodic) d -= Lb * std::round(d / Lb);
         Bp[q] = sa.R[q] + d + w->neighs[n1 * 3 + q];
         AB2 += (sa.R[q] - Bp[q]) * (sa.R[q] - Bp[q]);
      }
      pr.n1 = n1; pr.Q = 0; pr.q.assign((size_t)da.np * db.np, 0.f);
      double zmin = 1e300;
      for (int i = 0; i < da.np; i++) for (int j = 0; j < db.np; j++) {
         double za = da.Z[i], zb = db.Z[j], zz = za + zb, mu = za * zb / zz;
         double v = cmax[a][i] * cmax[b][j] * std::exp(-mu * AB2) *
                    std::sqrt(2.0 * std::pow(M_PI, 2.5) / (zz * zz * std::sqrt(2.0 * zz)));
         pr.q[(size_t)i * db.np + j] = (float)v;
         pr.Q += v;
         if (v * 1e6 > eps) zmin = std::min(zmin, zz);
      }
      for (int q = 0; q < 3; q++) pr.ctr[q] = 0.5 * (sa.R[q] + Bp[q]);
      pr.rad = 0.5 * std::sqrt(AB2) + (zmin < 1e299 ? std::sqrt(27.6 / zmin) : 0.0);
   };
   std::vector<std::vector<Pair>> pairs((size_t)S * S);
   const int nth = cfg->threads > 0 ? cfg->threads : std::max(1, (int)std::thread::hardware_concurrency());
   // rows a of the pair table (and below, the first set i of the quartets) are handed out to the
   // threads one at a time; every row is written by one thread, so the result is the serial one
   auto parallel_rows = [&](const std::function<void(int)> &fn) {
      std::atomic<int> next{0};
      std::vector<std::thread> th;
      for (int t = 0; t < nth; t++)
         th.emplace_back([&]() { for (int r; (r = next.fetch_add(1)) < S;) fn(r); });
      for (auto &x : th) x.join();
   };
   parallel_rows([&](int a) {
      for (int b = 0; b < S; b++) {
         if (!cfg->full_enum && b > a) continue;
         for (int n1 = 0; n1 < w->Ng; n1++) {
            Pair pr; pair_of(a, b, n1, pr);
            if (pr.Q * 10.0 < eps) continue;   // negligible pair even against |P| ~ 10
            pairs[(size_t)a * S + b].push_back(std::move(pr));
         }
      }
   });
   // ---- quartet enumeration: each first set i is enumerated by one thread into its own lists,
   // which are then joined in the order of i
   auto pidx = [&](int a, int b) { return (long)a * S + b; };
   const double rc = w->rc_bohr;
   struct Part { std::vector<SetQ> setq; std::vector<Shell> shells; std::vector<uint32_t> prims; long n_qrtt = 0; };
   std::vector<Part> parts(S);
   const uint64_t stride = cfg->setq_stride > 1 ? (uint64_t)cfg->setq_stride : 1;
   const uint64_t phase = cfg->setq_stride > 1 ? (uint64_t)cfg->setq_phase % stride : 0;
   // Set quartets in canonical order: (i,j) >= (k,l) with i >= j, k >= l. With setq_stride > 1 only
   // every stride-th ket pair index of each row is visited, from an offset that a hash of the bra
   // pair picks (a sample of 1/stride of the set quartets whose cost does not grow with the
   // workload's full size).
   parallel_rows([&](int i) {
   Part &out = parts[i];
   auto visit = [&](int j, int k, int l, const std::vector<Pair> &PL) {
      const auto &QL = pairs[(size_t)pidx(k, l)];
      if (QL.empty()) return;
      double pmax = std::max(std::max(Pblk[(size_t)i * S + k], Pblk[(size_t)i * S + l]),
                             std::max(Pblk[(size_t)j * S + k], Pblk[(size_t)j * S + l]));
      const SetDef &da = w->defs[w->sets[i].def], &db = w->defs[w->sets[j].def];
      const SetDef &dc = w->defs[w->sets[k].def], &dd = w->defs[w->sets[l].def];
      SetQ sq; sq.i = i; sq.j = j; sq.k = k; sq.l = l;
      if (cfg->full_enum) sq.fac = 0.25f;
      else {
         double f = 2.0;
         if (i == j) f *= 0.5;
         if (k == l) f *= 0.5;
         if (i == k && j == l) f *= 0.5;
         sq.fac = (float)f;
      }
      sq.shell_begin = (uint32_t)out.shells.size();
      for (const Pair &pa : PL) for (const Pair &pc : QL) {
         if (pa.Q * pc.Q * pmax < eps) continue;
         // truncated-Coulomb range: the nearest image of the ket distribution must be in reach
         double d2 = 0;
         for (int q = 0; q < 3; q++) {
            double d = pa.ctr[q] - pc.ctr[q];
            if (periodic) d -= Lb * std::round(d / Lb);
            d2 += d * d;
         }
         double lim = rc + pa.rad + pc.rad;
         bool reach = d2 <= lim * lim;
         if (!reach) continue;
         Shell sh; sh.n1 = (uint16_t)pa.n1; sh.n2 = (uint16_t)pc.n1;
         sh.bound = (float)(pa.Q * pc.Q * pmax);
         sh.prm_begin = (uint32_t)out.prims.size();
         for (int ia = 0; ia < da.np; ia++) for (int ib = 0; ib < db.np; ib++) {
            double qab = pa.q[(size_t)ia * db.np + ib];
            if (qab * pc.Q * pmax < eps) continue;
            for (int ic = 0; ic < dc.np; ic++) for (int id = 0; id < dd.np; id++) {
               double qcd = pc.q[(size_t)ic * dd.np + id];
               if (qab * qcd * pmax < eps) continue;
               out.prims.push_back(((uint32_t)ia << 24) | ((uint32_t)ib << 16) | ((uint32_t)ic << 8) | (uint32_t)id);
            }
         }
         sh.prm_end = (uint32_t)out.prims.size();
         if (sh.prm_end > sh.prm_begin) out.shells.push_back(sh);
      }
      sq.shell_end = (uint32_t)out.shells.size();
      if (sq.shell_end > sq.shell_begin) {
         out.setq.push_back(sq);
         out.n_qrtt += (long)da.nl * db.nl * dc.nl * dd.nl;
      }
   };
   for (int j = 0; j < S; j++) {
      if (!cfg->full_enum && j > i) continue;
      const auto &PL = pairs[(size_t)pidx(i, j)];
      if (PL.empty()) continue;
      if (cfg->full_enum) {
         for (int k = 0; k < S; k++) for (int l = 0; l < S; l++) visit(j, k, l, PL);
         continue;
      }
      const uint64_t pij = (uint64_t)i * (i + 1) / 2 + j;   // ket pairs (k,l) <= (i,j): indices 0..pij
      uint64_t kl = 0;
      if (stride > 1) {
         uint64_t x = pij + 0x9e3779b97f4a7c15ULL;   // splitmix64 of the bra pair index
         x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
         x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
         x ^= x >> 31;
         kl = (x + phase) % stride;
      }
      int k = 0;
      for (; kl <= pij; kl += stride) {
         while ((uint64_t)(k + 1) * (k + 2) / 2 <= kl) k++;
         visit(j, k, (int)(kl - (uint64_t)k * (k + 1) / 2), PL);
      }
   }
   });
   {
      size_t nsq = 0, nsh = 0, npr = 0;
      for (const Part &pt : parts) { nsq += pt.setq.size(); nsh += pt.shells.size(); npr += pt.prims.size(); }
      if (npr > 0xffffffffull || nsh > 0xffffffffull) {
         fprintf(stderr, "gd_create: %zu primitive quartets exceed the 32-bit trace indices; use setq_stride\n", npr);
         delete w;
         return nullptr;
      }
      w->setq.reserve(nsq); w->shells.reserve(nsh); w->prims.reserve(npr);
      for (Part &pt : parts) {
         const uint32_t sh0 = (uint32_t)w->shells.size(), pr0 = (uint32_t)w->prims.size();
         for (SetQ q : pt.setq) { q.shell_begin += sh0; q.shell_end += sh0; w->setq.push_back(q); }
         for (Shell h : pt.shells) { h.prm_begin += pr0; h.prm_end += pr0; w->shells.push_back(h); }
         w->prims.insert(w->prims.end(), pt.prims.begin(), pt.prims.end());
         w->n_qrtt += pt.n_qrtt;
         std::vector<SetQ>().swap(pt.setq); std::vector<Shell>().swap(pt.shells); std::vector<uint32_t>().swap(pt.prims);
      }
   }
   // ---- C0
   w->nder = 12;
   const int ld = (w->nder + 1) * 105;
   {
      // the fit depends only on nder: made once per process and copied into every workload
      static std::mutex mu;
      static std::vector<double> fitted;
      static int fitted_nder = -1;
      std::lock_guard<std::mutex> lock(mu);
      if (fitted_nder != w->nder) {
         fitted.assign((size_t)TCG_NPATCH * ld, 0.0);
         gd_tcg_table(w->nder, fitted.data());
         fitted_nder = w->nder;
      }
      w->C0 = fitted;
   }
   return w;
}

void gd_free(gd_workload *w) { delete w; }

void gd_get_info(const gd_workload *w, gd_info *inf) {
   inf->n_bf = w->n_bf; inf->n_sets = (int)w->sets.size(); inf->n_atoms = w->cfg.n_mol * 3;
   inf->Ng = w->Ng; inf->n_setq = (long)w->setq.size(); inf->n_shells = (long)w->shells.size();
   inf->n_prims = (long)w->prims.size(); inf->n_qrtt = w->n_qrtt; inf->rc_bohr = w->rc_bohr;
   inf->nder = w->nder; inf->ld_C0 = (w->nder + 1) * 105; inf->C0_size = (int)w->C0.size();
   double m = 0; for (double x : w->P) m = std::max(m, std::fabs(x));
   inf->max_abs_P = m;
   inf->flat_size = (long)w->flat_size;
}

void gd_get_P(const gd_workload *w, double *P) { std::memcpy(P, w->P.data(), sizeof(double) * w->P.size()); }
void gd_get_Pflat(const gd_workload *w, double *P) { std::memcpy(P, w->Pflat.data(), sizeof(double) * w->Pflat.size()); }

// Unpack a K (or P) in the packed block layout into the symmetric dense matrix of the full
// exchange operator, K = (U + U^T)/2 where U are the accumulated updates; the updates of the
// pair (X,Y) and (Y,X) were folded into the block (max, min).
void gd_unpack_K(const gd_workload *w, const double *Kflat, double *Kdense) {
   const int S = (int)w->sets.size(), n = w->n_bf;
   std::fill(Kdense, Kdense + (size_t)n * n, 0.0);
   for (int x = 0; x < S; x++) for (int y = 0; y <= x; y++) {
      const SetDef &dx = w->defs[w->sets[x].def], &dy = w->defs[w->sets[y].def];
      int nx = (2 * dx.l + 1) * dx.nl, ny = (2 * dy.l + 1) * dy.nl;
      int bx = w->sets[x].bf_off, by = w->sets[y].bf_off;
      const double *blk = &Kflat[w->blkoff[(size_t)x * S + y]];
      for (int c = 0; c < ny; c++) for (int r = 0; r < nx; r++) {
         double v = 0.5 * blk[(size_t)c * nx + r];
         Kdense[(size_t)(by + c) * n + bx + r] += v;   // (row bx+r, col by+c)
         Kdense[(size_t)(bx + r) * n + by + c] += v;   // transpose
      }
   }
}
void gd_get_C0(const gd_workload *w, double *C0) { std::memcpy(C0, w->C0.data(), sizeof(double) * w->C0.size()); }

// basis-function layout of each set: {bf_off, l, nl, atom}
void gd_get_sets(const gd_workload *w, int *out) {
   for (size_t s = 0; s < w->sets.size(); s++) {
      const SetDef &d = w->defs[w->sets[s].def];
      out[s * 4 + 0] = w->sets[s].bf_off; out[s * 4 + 1] = d.l; out[s * 4 + 2] = d.nl; out[s * 4 + 3] = w->sets[s].atom;
   }
}

// normalised coefficients of set s (nl*np) and its exponents; returns np
int gd_get_coeffs(const gd_workload *w, int s, double *K, double *Z, int *nl) {
   const SetDef &d = w->defs[w->sets[s].def];
   std::memcpy(K, d.Knorm.data(), sizeof(double) * d.Knorm.size());
   std::memcpy(Z, d.Z.data(), sizeof(double) * d.Z.size());
   *nl = d.nl;
   return d.np;
}

// shells of set quartet q: {n1, n2, n_prims} each; returns the count
long gd_get_shells(const gd_workload *w, long q, long *out) {
   const SetQ &s = w->setq[q];
   long n = 0;
   for (uint32_t h = s.shell_begin; h < s.shell_end; h++, n++) {
      out[n * 3 + 0] = w->shells[h].n1; out[n * 3 + 1] = w->shells[h].n2;
      out[n * 3 + 2] = w->shells[h].prm_end - w->shells[h].prm_begin;
   }
   return n;
}

// primitive-quartet codes (ipa<<24 | ipb<<16 | ipc<<8 | ipd) of shell quartet h (index in the
// workload's shell list, set quartet q's shells are [sum of earlier n_shells, + n_shells)); returns
// the count
long gd_get_shell_prims(const gd_workload *w, long h, uint32_t *out) {
   const Shell &sh = w->shells[h];
   std::memcpy(out, &w->prims[sh.prm_begin], sizeof(uint32_t) * (sh.prm_end - sh.prm_begin));
   return (long)(sh.prm_end - sh.prm_begin);
}

// a dense symmetric n_bf x n_bf matrix (column-major) in the packed set-pair block layout of P/K
void gd_pack(const gd_workload *w, const double *dense, double *flat) {
   const int S = (int)w->sets.size(), n = w->n_bf;
   auto nbf_of = [&](int x) { const SetDef &d = w->defs[w->sets[x].def]; return (2 * d.l + 1) * d.nl; };
   for (int x = 0; x < S; x++) for (int y = 0; y <= x; y++) {
      const int nx = nbf_of(x), ny = nbf_of(y), bx = w->sets[x].bf_off, by = w->sets[y].bf_off;
      double *blk = flat + w->blkoff[(size_t)x * S + y];
      for (int c = 0; c < ny; c++) for (int r = 0; r < nx; r++) blk[(size_t)c * nx + r] = dense[(size_t)(by + c) * n + bx + r];
   }
}

// the screening estimate of every shell quartet, in the workload's shell order
void gd_get_shell_bounds(const gd_workload *w, float *out) {
   for (size_t h = 0; h < w->shells.size(); h++) out[h] = w->shells[h].bound;
}

// per set quartet {i,j,k,l,n_shells,n_prims} (for cost/class statistics)
void gd_get_setq(const gd_workload *w, long *out) {
   for (size_t q = 0; q < w->setq.size(); q++) {
      const SetQ &s = w->setq[q];
      long np = 0;
      for (uint32_t h = s.shell_begin; h < s.shell_end; h++) np += w->shells[h].prm_end - w->shells[h].prm_begin;
      out[q * 6 + 0] = s.i; out[q * 6 + 1] = s.j; out[q * 6 + 2] = s.k; out[q * 6 + 3] = s.l;
      out[q * 6 + 4] = s.shell_end - s.shell_begin; out[q * 6 + 5] = np;
   }
}

// ----- replay --------------------------------------------------------------------------
typedef void *(*fn_create)();
typedef void (*fn_h)(void *);
typedef void (*fn_pot)(void *, double, double *, int, int);
typedef void (*fn_d)(void *, double);
typedef void (*fn_i)(void *, int);
typedef void (*fn_P)(void *, double *, int);
typedef void (*fn_getK)(void *, double *);
typedef void (*fn_cell)(void *, bool, double *, double *);
typedef void (*fn_neighs)(void *, double *, int);
typedef void (*fn_atom)(void *, int, double *, double *, int);
typedef void (*fn_atomL)(void *, int, int, int, double *);
typedef void (*fn_prm)(void *, int, int, int, int);
typedef void (*fn_shell)(void *, int, int, int, int, int, int);
typedef void (*fn_qrt)(void *, int, int, int, int, int, int, int, int);
typedef void (*fn_qrtt)(void *, double, int, int, int, int, int, int, int, int, int, int, int, int,
                        unsigned, unsigned, unsigned, unsigned, bool, bool, bool, bool);

typedef int (*fn_bulk)(void *, int, const int *, const int *, const int *, const int *, const unsigned *, const int *,
                       const int *, const double *, const int *, const unsigned *, const unsigned char *);

struct gd_api {
   void *dl;
   fn_create create; fn_h init; fn_pot pot; fn_d hf; fn_i maxmem; fn_P setP; fn_getK getK;
   fn_cell cell; fn_neighs neighs; fn_atom atom; fn_atomL atomL; fn_prm prm; fn_shell shell;
   fn_qrt qrt; fn_qrtt qrtt; fn_h addset; fn_h dispatch; fn_h destroy;
   fn_bulk bulk;   // libgint_add_set_quartets, if the library has it
   fn_d fp32thr;   // libgint_set_fp32_threshold, if the library has it
   fn_d bound;     // libgint_add_shell_bound, if the library has it
};

gd_api *gd_api_open(const char *path) {
   void *dl = dlopen(path, RTLD_NOW | RTLD_LOCAL);
   if (!dl) { fprintf(stderr, "gd_api_open: %s\n", dlerror()); return nullptr; }
   gd_api *a = new gd_api();
   a->dl = dl;
#define SYM(f, T, name) a->f = (T)dlsym(dl, name); if (!a->f) { fprintf(stderr, "missing %s\n", name); delete a; return nullptr; }
   SYM(create, fn_create, "libgint_create_handle");
   SYM(init, fn_h, "libgint_init");
   SYM(pot, fn_pot, "libgint_set_Potential_Truncated");
   SYM(hf, fn_d, "libgint_set_hf_fac");
   SYM(maxmem, fn_i, "libgint_set_max_mem");
   SYM(setP, fn_P, "libgint_set_P");
   SYM(getK, fn_getK, "libgint_get_K");
   SYM(cell, fn_cell, "libgint_set_cell");
   SYM(neighs, fn_neighs, "libgint_set_neighs");
   SYM(atom, fn_atom, "libgint_set_Atom");
   SYM(atomL, fn_atomL, "libgint_set_Atom_L");
   SYM(prm, fn_prm, "libgint_add_prm");
   SYM(shell, fn_shell, "libgint_add_shell");
   SYM(qrt, fn_qrt, "libgint_add_qrt");
   SYM(qrtt, fn_qrtt, "libgint_add_qrtt");
   SYM(addset, fn_h, "libgint_add_set");
   SYM(dispatch, fn_h, "libgint_dispatch");
#undef SYM
   a->destroy = (fn_h)dlsym(dl, "libgint_destroy_handle");
   a->bulk = (fn_bulk)dlsym(dl, "libgint_add_set_quartets");
   a->fp32thr = (fn_d)dlsym(dl, "libgint_set_fp32_threshold");
   a->bound = (fn_d)dlsym(dl, "libgint_add_shell_bound");
   return a;
}

void *gd_api_symbol(gd_api *a, const char *name) { return dlsym(a->dl, name); }

// Set up a handle for this workload (basis, potential, cell): everything before set_P.
void *gd_setup(const gd_workload *w, gd_api *a, int max_mem_mb) {
   void *h = a->create();
   a->init(h);
   gd_workload *wm = const_cast<gd_workload *>(w);
   a->pot(h, w->rc_bohr, wm->C0.data(), (w->nder + 1) * 105, (int)w->C0.size());
   a->hf(h, 1.0);
   a->maxmem(h, max_mem_mb);
   a->cell(h, w->cfg.periodic != 0, wm->cell_h, wm->cell_i);
   a->neighs(h, wm->neighs.data(), w->Ng);
   for (size_t s = 0; s < w->sets.size(); s++) {
      const SetDef &d = w->defs[w->sets[s].def];
      a->atom(h, (int)s, wm->sets[s].R, const_cast<double *>(d.Z.data()), d.np);
      a->atomL(h, (int)s, d.l, d.nl, const_cast<double *>(d.Kraw.data()));
   }
   return h;
}

// One K build: set_P, the add_* stream of set quartets [q0, q1), get_K. Returns wall ms.
// times[0] = set_P, [1] = stream, [2] = get_K (ms). P == nullptr uses the workload's P.
static double build_K_impl(const gd_workload *w, gd_api *a, void *h, const double *P, double *K,
                           long q0, long q1, const long *idx, double *times, bool bulk = false);
static int g_reverse_prims = 0;
static int g_bulk = 0;        // stream through libgint_add_set_quartets when the library has it
void gd_set_bulk(int on) { g_bulk = on; }
// mixed precision: every K build sets this threshold (libgint_set_fp32_threshold, 0 = FP64) where
// the library has it; each shell quartet's bound goes before its add_shell (libgint_add_shell_bound)
// wherever the library takes one (it also drives incremental replays' screening)
static double g_fp32_thr = 0.0;
void gd_set_fp32_threshold(double thr) { g_fp32_thr = thr; }
static long g_only_shell = -1;   // replay only this shell (index within its set quartet), -1: all
void gd_set_only_shell(long k) { g_only_shell = k; }
// replay the primitive quartets of every shell in reverse order (a reordering of the same sums)
void gd_set_reverse_prims(int on) { g_reverse_prims = on; }

double gd_build_K(const gd_workload *w, gd_api *a, void *h, const double *P, double *K,
                  long q0, long q1, double *times) {
   return build_K_impl(w, a, h, P, K, q0, q1, nullptr, times, g_bulk != 0);
}

// the same for an explicit list of set quartets idx[0..n)
double gd_build_K_subset(const gd_workload *w, gd_api *a, void *h, const double *P, double *K,
                         const long *idx, long n, double *times) {
   return build_K_impl(w, a, h, P, K, 0, n, idx, times, g_bulk != 0);
}

// the add_* arguments of one set quartet's contraction rows, in the packed block layout of P/K:
// the pair (x,y) lands in block (max, min); T selects the transposed walk when x < y; ld =
// functions of the block's row set (< 256)
static inline __attribute__((always_inline)) void qrtt_addr(const gd_workload *w, int S, int sx, int sy, int inx,
                                                             int iny, unsigned &off, int &ld, bool &T) {
   const SetDef &dx = w->defs[w->sets[sx].def], &dy = w->defs[w->sets[sy].def];
   int nsx = 2 * dx.l + 1, nsy = 2 * dy.l + 1;
   if (sx >= sy) {
      T = false; ld = nsx * dx.nl;
      off = w->blkoff[(size_t)sx * S + sy] + (unsigned)(iny * nsy * ld + inx * nsx);
   } else {
      T = true; ld = nsy * dy.nl;
      off = w->blkoff[(size_t)sy * S + sx] + (unsigned)(inx * nsx * ld + iny * nsy);
   }
}

// The same stream through libgint_add_set_quartets, in chunks of set quartets: the chunk's
// shells, primitive codes and contraction rows are counted first, then written by index into
// arrays that keep their capacity from chunk to chunk.
static void stream_bulk(const gd_workload *w, gd_api *a, void *h, long q0, long q1, const long *idx) {
   const long CH = 4096;
   const int S = (int)w->sets.size();
   std::vector<int> sets, shc, shi, pc, qc, qr, ld;
   std::vector<unsigned> codes, off;
   std::vector<double> fac;
   std::vector<unsigned char> T;
   for (long c0 = q0; c0 < q1; c0 += CH) {
      const long c1 = std::min(q1, c0 + CH), nq = c1 - c0;
      size_t nsh = 0, npr = 0, nrow = 0;
      for (long iq0 = c0; iq0 < c1; iq0++) {
         const SetQ &q = w->setq[idx ? idx[iq0] : iq0];
         for (uint32_t hs = q.shell_begin; hs < q.shell_end; hs++) {
            if (g_only_shell >= 0 && (long)(hs - q.shell_begin) != g_only_shell) continue;
            nsh++;
            npr += w->shells[hs].prm_end - w->shells[hs].prm_begin;
         }
         nrow += (size_t)w->defs[w->sets[q.i].def].nl * w->defs[w->sets[q.j].def].nl *
                 w->defs[w->sets[q.k].def].nl * w->defs[w->sets[q.l].def].nl;
      }
      sets.resize(4 * nq); shc.resize(nq); qc.resize(nq); qr.resize(8 * nq);
      shi.resize(2 * nsh); pc.resize(nsh); codes.resize(npr);
      fac.resize(nrow); ld.resize(4 * nrow); off.resize(4 * nrow); T.resize(nrow);
      size_t ish = 0, ip = 0, ir = 0;
      for (long iq0 = c0; iq0 < c1; iq0++) {
         const long k = iq0 - c0;
         const SetQ &q = w->setq[idx ? idx[iq0] : iq0];
         const SetDef *d4[4] = {&w->defs[w->sets[q.i].def], &w->defs[w->sets[q.j].def], &w->defs[w->sets[q.k].def],
                                &w->defs[w->sets[q.l].def]};
         int *s4 = &sets[4 * k];
         s4[0] = q.i; s4[1] = q.j; s4[2] = q.k; s4[3] = q.l;
         int ns = 0;
         for (uint32_t hs = q.shell_begin; hs < q.shell_end; hs++) {
            if (g_only_shell >= 0 && (long)(hs - q.shell_begin) != g_only_shell) continue;
            const Shell &sh = w->shells[hs];
            shi[2 * ish] = sh.n1; shi[2 * ish + 1] = sh.n2;
            const int np = (int)(sh.prm_end - sh.prm_begin);
            pc[ish++] = np;
            for (int pp = 0; pp < np; pp++)
               codes[ip++] = w->prims[g_reverse_prims ? sh.prm_end - 1 - pp : sh.prm_begin + pp];
            ns++;
         }
         shc[k] = ns;
         qc[k] = 1;
         int *r = &qr[8 * k];
         r[0] = d4[0]->l; r[1] = d4[1]->l; r[2] = d4[2]->l; r[3] = d4[3]->l;
         r[4] = d4[0]->nl; r[5] = d4[1]->nl; r[6] = d4[2]->nl; r[7] = d4[3]->nl;
         for (int ia = 0; ia < d4[0]->nl; ia++) for (int ib = 0; ib < d4[1]->nl; ib++)
         for (int ic = 0; ic < d4[2]->nl; ic++) for (int id = 0; id < d4[3]->nl; id++, ir++) {
            bool t4[4];
            qrtt_addr(w, S, q.i, q.k, ia, ic, off[4 * ir + 0], ld[4 * ir + 0], t4[0]);
            qrtt_addr(w, S, q.i, q.l, ia, id, off[4 * ir + 1], ld[4 * ir + 1], t4[1]);
            qrtt_addr(w, S, q.j, q.k, ib, ic, off[4 * ir + 2], ld[4 * ir + 2], t4[2]);
            qrtt_addr(w, S, q.j, q.l, ib, id, off[4 * ir + 3], ld[4 * ir + 3], t4[3]);
            fac[ir] = (double)q.fac;
            T[ir] = (unsigned char)((t4[0] ? 1 : 0) | (t4[1] ? 2 : 0) | (t4[2] ? 4 : 0) | (t4[3] ? 8 : 0));
         }
      }
      a->bulk(h, (int)nq, sets.data(), shc.data(), shi.data(), pc.data(), codes.data(), qc.data(), qr.data(),
              fac.data(), ld.data(), off.data(), T.data());
   }
}

// The per-call add_* stream of one set quartet: add_prm* add_shell per image pair (with its bound
// when bounds is set), add_qrt, add_qrtt per contraction row, add_set. The workload's set indices are
// shifted by set_off and its P/K offsets by flat_off (several systems in one handle).
static void stream_setq(const gd_workload *w, gd_api *a, void *h, const SetQ &q, int set_off, uint32_t flat_off,
                        bool bounds) {
   const int S = (int)w->sets.size();
   const Set *s4[4] = {&w->sets[q.i], &w->sets[q.j], &w->sets[q.k], &w->sets[q.l]};
   const SetDef *d4[4] = {&w->defs[s4[0]->def], &w->defs[s4[1]->def], &w->defs[s4[2]->def], &w->defs[s4[3]->def]};
   for (uint32_t hs = q.shell_begin; hs < q.shell_end; hs++) {
      if (g_only_shell >= 0 && (long)(hs - q.shell_begin) != g_only_shell) continue;
      const Shell &sh = w->shells[hs];
      for (uint32_t pp = sh.prm_begin; pp < sh.prm_end; pp++) {
         const uint32_t p = g_reverse_prims ? sh.prm_end - 1 - (pp - sh.prm_begin) : pp;
         uint32_t c = w->prims[p];
         a->prm(h, c >> 24, (c >> 16) & 255, (c >> 8) & 255, c & 255);
      }
      if (bounds) a->bound(h, (double)sh.bound);
      a->shell(h, q.i + set_off, q.j + set_off, q.k + set_off, q.l + set_off, sh.n1, sh.n2);
   }
   const int la = d4[0]->l, lb = d4[1]->l, lc = d4[2]->l, ld = d4[3]->l;
   a->qrt(h, la, lb, lc, ld, d4[0]->nl, d4[1]->nl, d4[2]->nl, d4[3]->nl);
   // K/P addressing in the packed block layout: the pair (x,y) lands in block (max, min);
   // T selects the transposed walk when x < y. ld = functions of the block's row set (< 256).
   auto addr = [&](int sx, int sy, int inx, int iny, unsigned &off, int &ldv, bool &T) {
      qrtt_addr(w, S, sx, sy, inx, iny, off, ldv, T);
      off += flat_off;
   };
   for (int ia = 0; ia < d4[0]->nl; ia++) for (int ib = 0; ib < d4[1]->nl; ib++)
   for (int ic = 0; ic < d4[2]->nl; ic++) for (int id = 0; id < d4[3]->nl; id++) {
      unsigned oac, oad, obc, obd; int lac, lad, lbc, lbd; bool Tac, Tad, Tbc, Tbd;
      addr(q.i, q.k, ia, ic, oac, lac, Tac);
      addr(q.i, q.l, ia, id, oad, lad, Tad);
      addr(q.j, q.k, ib, ic, obc, lbc, Tbc);
      addr(q.j, q.l, ib, id, obd, lbd, Tbd);
      a->qrtt(h, (double)q.fac, la, lb, lc, ld, ia, ib, ic, id, lac, lad, lbc, lbd, oac, oad, obc, obd,
              Tac, Tad, Tbc, Tbd);
   }
   a->addset(h);
}

static double build_K_impl(const gd_workload *w, gd_api *a, void *h, const double *P, double *K,
                           long q0, long q1, const long *idx, double *times, bool bulk) {
   using clk = std::chrono::steady_clock;
   if (!idx && (q1 < 0 || q1 > (long)w->setq.size())) q1 = (long)w->setq.size();
   auto t0 = clk::now();
   if (a->fp32thr) a->fp32thr(h, g_fp32_thr);
   const bool bounds = a->bound != nullptr;
   a->setP(h, const_cast<double *>(P ? P : w->Pflat.data()), (int)w->flat_size);
   auto t1 = clk::now();
   if (bulk && a->bulk) stream_bulk(w, a, h, q0, q1, idx);
   else for (long iq0 = q0; iq0 < q1; iq0++) stream_setq(w, a, h, w->setq[idx ? idx[iq0] : iq0], 0, 0, bounds);
   auto t2 = clk::now();
   a->getK(h, K);
   auto t3 = clk::now();
   auto ms = [](clk::time_point x, clk::time_point y) { return std::chrono::duration<double, std::milli>(y - x).count(); };
   if (times) { times[0] = ms(t0, t1); times[1] = ms(t1, t2); times[2] = ms(t2, t3); }
   return ms(t0, t3);
}

// Split of a K build over nh caller threads: cut[0..nh] bounds contiguous shares of the set
// quartets (all of them, or idx[0..n_idx) when idx is given) with about the same number of
// primitive quartets each.
void gd_mt_split(const gd_workload *w, const long *idx, long n_idx, int nh, long *cut) {
   const long nq = idx ? n_idx : (long)w->setq.size();
   std::vector<double> cum(nq + 1, 0.0);
   for (long q = 0; q < nq; q++) {
      const SetQ &s = w->setq[idx ? idx[q] : q];
      long np = 0;
      for (uint32_t hh = s.shell_begin; hh < s.shell_end; hh++) np += w->shells[hh].prm_end - w->shells[hh].prm_begin;
      cum[q + 1] = cum[q] + (double)np;
   }
   cut[0] = 0;
   cut[nh] = nq;
   for (int t = 1; t < nh; t++)
      cut[t] = (long)(std::lower_bound(cum.begin(), cum.end(), cum[nq] * t / nh) - cum.begin());
}

// One K build by nh host threads, thread t driving handles[t] (each set up by gd_setup) over the
// set quartets [cut[t], cut[t+1]) (positions in idx[] when idx is given; see gd_mt_split), as a
// caller with one handle per OpenMP thread does; the threads' K are summed into K. Returns wall
// ms; times[0..2] are thread 0's set_P / stream / get_K, times[3] the slowest thread's build and
// times[4] the summation (ms).
double gd_build_K_mt(const gd_workload *w, gd_api *a, void **handles, int nh, const double *P, double *K,
                     const long *idx, const long *cut, double *times) {
   using clk = std::chrono::steady_clock;
   auto ms = [](clk::time_point x, clk::time_point y) { return std::chrono::duration<double, std::milli>(y - x).count(); };
   std::vector<std::vector<double>> Ks(nh);
   std::vector<double> tt(3 * nh, 0.0), tw(nh, 0.0);
   auto t0 = clk::now();
   std::vector<std::thread> th;
   for (int t = 0; t < nh; t++)
      th.emplace_back([&, t]() {
         Ks[t].assign(w->flat_size, 0.0);
         tw[t] = build_K_impl(w, a, handles[t], P, Ks[t].data(), cut[t], cut[t + 1], idx, &tt[3 * t], g_bulk != 0);
      });
   for (auto &x : th) x.join();
   auto t1 = clk::now();
   std::fill(K, K + w->flat_size, 0.0);
   for (int t = 0; t < nh; t++)
      for (size_t i = 0; i < w->flat_size; i++) K[i] += Ks[t][i];
   auto t2 = clk::now();
   if (times) {
      for (int i = 0; i < 3; i++) times[i] = tt[i];
      times[3] = *std::max_element(tw.begin(), tw.end());
      times[4] = ms(t1, t2);
   }
   return ms(t0, t2);
}

// One K build by an OpenMP team of nh threads, as CP2K's HFX module drives the libGint C-ABI from
// its OpenMP team: thread t uses handles[t] and streams the set quartets [cut[t], cut[t+1])
// (positions in idx[] when idx is given), and every thread passes the same P and K arrays. The
// library's set_P and get_K are collective over the team, so K receives the team's whole K with
// no summation by the caller. Returns wall ms (-1 if the team did not get nh threads); times as
// gd_build_K_mt, with times[4] = 0.
double gd_build_K_team(const gd_workload *w, gd_api *a, void **handles, int nh, const double *P, double *K,
                       const long *idx, const long *cut, double *times) {
   using clk = std::chrono::steady_clock;
   std::vector<double> tt(3 * nh, 0.0), tw(nh, 0.0);
   int got = 0;
   auto t0 = clk::now();
   omp_set_dynamic(0);
#pragma omp parallel num_threads(nh)
   {
      const int t = omp_get_thread_num();
#pragma omp single
      got = omp_get_num_threads();
      if (got == nh)
         tw[t] = build_K_impl(w, a, handles[t], P, K, cut[t], cut[t + 1], idx, &tt[3 * t], g_bulk != 0);
   }
   auto t1 = clk::now();
   if (got != nh) return -1.0;
   if (times) {
      for (int i = 0; i < 3; i++) times[i] = tt[i];
      times[3] = *std::max_element(tw.begin(), tw.end());
      times[4] = 0.0;
   }
   return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

// ----- several independent systems in one handle -----------------------------------------
// The systems' sets are registered one after another (system k's set s is set_off[k] + s) and
// their packed P/K arrays are concatenated (system k's at flat_off[k]); every set quartet lies
// within one system, so the engine sees one class-sorted quartet list over all of them. All
// systems share the potential, the cell and the image list of the first (non-periodic clusters).
void *gd_setup_multi(const gd_workload *const *ws, int n, gd_api *a, int max_mem_mb) {
   void *h = a->create();
   a->init(h);
   gd_workload *w0 = const_cast<gd_workload *>(ws[0]);
   a->pot(h, w0->rc_bohr, w0->C0.data(), (w0->nder + 1) * 105, (int)w0->C0.size());
   a->hf(h, 1.0);
   a->maxmem(h, max_mem_mb);
   a->cell(h, w0->cfg.periodic != 0, w0->cell_h, w0->cell_i);
   a->neighs(h, w0->neighs.data(), w0->Ng);
   int off = 0;
   for (int k = 0; k < n; k++) {
      gd_workload *w = const_cast<gd_workload *>(ws[k]);
      for (size_t s = 0; s < w->sets.size(); s++) {
         const SetDef &d = w->defs[w->sets[s].def];
         a->atom(h, off + (int)s, w->sets[s].R, const_cast<double *>(d.Z.data()), d.np);
         a->atomL(h, off + (int)s, d.l, d.nl, const_cast<double *>(d.Kraw.data()));
      }
      off += (int)w->sets.size();
   }
   return h;
}

// One K build over every set quartet of the n systems in one handle: set_P with the concatenated
// packed P, the add_* stream system after system, get_K into K (the concatenated packed K, sum of
// the systems' flat sizes). Returns wall ms; times as gd_build_K.
double gd_build_K_multi(const gd_workload *const *ws, int n, gd_api *a, void *h, double *K, double *times) {
   using clk = std::chrono::steady_clock;
   size_t tot = 0;
   for (int k = 0; k < n; k++) tot += ws[k]->flat_size;
   std::vector<double> P(tot);
   size_t fo = 0;
   for (int k = 0; k < n; k++) { std::memcpy(P.data() + fo, ws[k]->Pflat.data(), ws[k]->flat_size * 8); fo += ws[k]->flat_size; }
   auto t0 = clk::now();
   if (a->fp32thr) a->fp32thr(h, g_fp32_thr);
   const bool bounds = a->bound != nullptr;
   a->setP(h, P.data(), (int)tot);
   auto t1 = clk::now();
   int so = 0;
   fo = 0;
   for (int k = 0; k < n; k++) {
      for (const SetQ &q : ws[k]->setq) stream_setq(ws[k], a, h, q, so, (uint32_t)fo, bounds);
      so += (int)ws[k]->sets.size();
      fo += ws[k]->flat_size;
   }
   auto t2 = clk::now();
   a->getK(h, K);
   auto t3 = clk::now();
   auto ms = [](clk::time_point x, clk::time_point y) { return std::chrono::duration<double, std::milli>(y - x).count(); };
   if (times) { times[0] = ms(t0, t1); times[1] = ms(t1, t2); times[2] = ms(t2, t3); }
   return ms(t0, t3);
}

void gd_teardown(gd_api *a, void *h) { if (a->destroy) a->destroy(h); }

}  // extern "C"
