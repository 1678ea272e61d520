"""Synthetic water workloads and the C-ABI replayer (ctypes front end of libgint_driver.so).

The driver library plays the caller of the libGint C-ABI: it generates seeded water systems,
screens the set/primitive quartets, and replays the add_* stream through any library exporting
the libgint_* entry points. The named configurations follow the benchmark definitions:

  small_l2      4 water-like molecules, 12 A box, no PBC, l<=2 basis, 20 occupied orbitals
  periodic_l2   32 molecules, 9.86 A cubic cell, 27 images, l<=2, 128 occupied orbitals
  periodic_l2_small  12 molecules at the same density (7.1 A cell), for kernel profiling
  periodic_l3   64 molecules, 12.4 A cell, 125 images, l<=3 basis with general contraction
  periodic_l3_scf  128 molecules, 15.6 A cell, the 256 image cells nearest the origin, l<=3 basis
"""
import ctypes
import os
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(_HERE, "lib")
DRIVER_SO = os.path.join(LIBDIR, "libgint_driver.so")
ENGINE_SO = os.path.join(LIBDIR, "libgint_b200.so")


class GdConfig(ctypes.Structure):
    _fields_ = [("n_mol", ctypes.c_int), ("box_ang", ctypes.c_double), ("periodic", ctypes.c_int),
                ("n_img_1d", ctypes.c_int), ("basis", ctypes.c_int), ("n_occ", ctypes.c_int),
                ("rc_ang", ctypes.c_double), ("eps_schwarz", ctypes.c_double),
                ("seed", ctypes.c_uint64), ("full_enum", ctypes.c_int), ("max_prm", ctypes.c_int),
                ("max_ncontr", ctypes.c_int), ("setq_stride", ctypes.c_int), ("setq_phase", ctypes.c_int),
                ("threads", ctypes.c_int), ("max_images", ctypes.c_int)]


class GdInfo(ctypes.Structure):
    _fields_ = [("n_bf", ctypes.c_int), ("n_sets", ctypes.c_int), ("n_atoms", ctypes.c_int),
                ("Ng", ctypes.c_int), ("n_setq", ctypes.c_long), ("n_shells", ctypes.c_long),
                ("n_prims", ctypes.c_long), ("n_qrtt", ctypes.c_long), ("rc_bohr", ctypes.c_double),
                ("nder", ctypes.c_int), ("ld_C0", ctypes.c_int), ("C0_size", ctypes.c_int),
                ("max_abs_P", ctypes.c_double), ("flat_size", ctypes.c_long)]


CONFIGS = {
    "small_l2": dict(n_mol=4, box_ang=12.0, periodic=0, n_img_1d=1, basis=2, n_occ=20),
    "periodic_l2": dict(n_mol=32, box_ang=9.86, periodic=1, n_img_1d=3, basis=2, n_occ=128),
    "periodic_l2_small": dict(n_mol=12, box_ang=7.1, periodic=1, n_img_1d=3, basis=2, n_occ=48),
    "periodic_l3": dict(n_mol=64, box_ang=12.4, periodic=1, n_img_1d=5, basis=3, n_occ=256),
    "periodic_l3_scf": dict(n_mol=128, box_ang=15.6, periodic=1, n_img_1d=7, basis=3, n_occ=512, max_images=256),
}

_D = ctypes.POINTER(ctypes.c_double)
_lib = None


def driver():
    global _lib
    if _lib is None:
        if not os.path.exists(DRIVER_SO):
            raise RuntimeError(f"{DRIVER_SO} is missing: run libgint_b200.build.build_all()")
        lib = ctypes.CDLL(DRIVER_SO)
        lib.gd_create.restype = ctypes.c_void_p
        lib.gd_create.argtypes = [ctypes.POINTER(GdConfig)]
        lib.gd_free.argtypes = [ctypes.c_void_p]
        lib.gd_get_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(GdInfo)]
        lib.gd_get_P.argtypes = [ctypes.c_void_p, _D]
        lib.gd_get_C0.argtypes = [ctypes.c_void_p, _D]
        lib.gd_get_Pflat.argtypes = [ctypes.c_void_p, _D]
        lib.gd_unpack_K.argtypes = [ctypes.c_void_p, _D, _D]
        lib.gd_get_sets.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        lib.gd_get_setq.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
        lib.gd_api_open.restype = ctypes.c_void_p
        lib.gd_api_open.argtypes = [ctypes.c_char_p]
        lib.gd_api_symbol.restype = ctypes.c_void_p
        lib.gd_api_symbol.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        lib.gd_setup.restype = ctypes.c_void_p
        lib.gd_setup.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.gd_build_K.restype = ctypes.c_double
        lib.gd_build_K.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _D, _D,
                                   ctypes.c_long, ctypes.c_long, _D]
        lib.gd_build_K_subset.restype = ctypes.c_double
        lib.gd_build_K_subset.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _D, _D,
                                          ctypes.POINTER(ctypes.c_long), ctypes.c_long, _D]
        lib.gd_build_K_mt.restype = ctypes.c_double
        lib.gd_build_K_mt.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                      _D, _D, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long), _D]
        lib.gd_build_K_team.restype = ctypes.c_double
        lib.gd_build_K_team.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                        _D, _D, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long), _D]
        lib.gd_mt_split.restype = None
        lib.gd_mt_split.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long), ctypes.c_long, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_long)]
        lib.gd_pack.restype = None
        lib.gd_pack.argtypes = [ctypes.c_void_p, _D, _D]
        lib.gd_setup_multi.restype = ctypes.c_void_p
        lib.gd_setup_multi.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        lib.gd_build_K_multi.restype = ctypes.c_double
        lib.gd_build_K_multi.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p, _D, _D]
        lib.gd_set_fp32_threshold.restype = None
        lib.gd_set_fp32_threshold.argtypes = [ctypes.c_double]
        lib.gd_get_shell_bounds.restype = None
        lib.gd_get_shell_bounds.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]
        lib.gd_set_bulk.restype = None
        lib.gd_set_bulk.argtypes = [ctypes.c_int]
        lib.gd_get_coeffs.restype = ctypes.c_int
        lib.gd_get_coeffs.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, ctypes.POINTER(ctypes.c_int)]
        lib.gd_teardown.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.gd_tcg_table.restype = ctypes.c_int
        lib.gd_tcg_table.argtypes = [ctypes.c_int, _D]
        lib.gd_tcg_exact.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _D]
        lib.gd_boys.argtypes = [ctypes.c_int, ctypes.c_double, _D]
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(_D)


class Workload:
    """A generated system plus its screened add_* call stream."""

    def __init__(self, name=None, seed=0, eps_schwarz=1e-11, rc_ang=6.0, full_enum=False,
                 max_prm=16, max_ncontr=4, setq_stride=1, setq_phase=0, threads=0, max_images=0, **overrides):
        params = dict(CONFIGS[name]) if name else {}
        params.update(overrides)
        max_images = params.pop("max_images", max_images)
        cfg = GdConfig(n_mol=params["n_mol"], box_ang=params["box_ang"],
                       periodic=params["periodic"], n_img_1d=params["n_img_1d"],
                       basis=params["basis"], n_occ=params["n_occ"], rc_ang=rc_ang,
                       eps_schwarz=eps_schwarz, seed=seed, full_enum=int(full_enum),
                       max_prm=max_prm, max_ncontr=max_ncontr, setq_stride=setq_stride,
                       setq_phase=setq_phase, threads=threads, max_images=max_images)
        self.name = name
        self.params = params
        self._w = driver().gd_create(ctypes.byref(cfg))
        if not self._w:
            raise RuntimeError("workload generation failed (too large for the 32-bit trace: sample it with setq_stride)")
        inf = GdInfo()
        driver().gd_get_info(self._w, ctypes.byref(inf))
        self.info = {f: getattr(inf, f) for f, _ in GdInfo._fields_}
        self.n_bf = inf.n_bf

    def __del__(self):
        if getattr(self, "_w", None) and _lib is not None:
            _lib.gd_free(self._w)
            self._w = None

    @property
    def P(self):
        P = np.empty(self.n_bf * self.n_bf)
        driver().gd_get_P(self._w, _dp(P))
        return P

    @property
    def Pflat(self):
        """P in the packed set-pair block layout (what set_P receives)."""
        P = np.empty(self.info["flat_size"])
        driver().gd_get_Pflat(self._w, _dp(P))
        return P

    def pack(self, dense):
        """A dense symmetric n_bf x n_bf matrix in the packed set-pair block layout of P/K."""
        d = np.ascontiguousarray(np.asarray(dense, dtype=np.float64).reshape(self.n_bf, self.n_bf).T)
        flat = np.empty(self.info["flat_size"])
        driver().gd_pack(self._w, _dp(d), _dp(flat))
        return flat

    def unpack_K(self, K_flat):
        """Dense symmetric exchange matrix from the packed K returned by get_K."""
        K = np.empty(self.n_bf * self.n_bf)
        driver().gd_unpack_K(self._w, _dp(np.ascontiguousarray(K_flat)), _dp(K))
        return K.reshape(self.n_bf, self.n_bf)

    def exchange_energy(self, K_flat):
        """E_x = 1/4 sum P K (closed shell, P = 2 C C^T, hf_fac = 1)."""
        n = self.n_bf
        return 0.25 * float(np.sum(self.P.reshape(n, n) * self.unpack_K(K_flat)))

    @property
    def C0(self):
        C0 = np.empty(self.info["C0_size"])
        driver().gd_get_C0(self._w, _dp(C0))
        return C0

    def sets(self):
        out = np.empty((self.info["n_sets"], 4), dtype=np.int32)
        driver().gd_get_sets(self._w, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return out

    def coeffs(self, s):
        """(normalised coefficients [nl, np], exponents [np]) of set s."""
        K = np.zeros(64); Z = np.zeros(16); nl = ctypes.c_int()
        np_ = driver().gd_get_coeffs(self._w, s, _dp(K), _dp(Z), ctypes.byref(nl))
        return K[:nl.value * np_].reshape(nl.value, np_), Z[:np_]

    def shell_bounds(self):
        """The screening estimate sqrt((ab|ab)(cd|cd)) max|P| of every shell quartet."""
        out = np.empty(self.info["n_shells"], dtype=np.float32)
        driver().gd_get_shell_bounds(self._w, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        return out

    def setq(self):
        out = np.empty((self.info["n_setq"], 6), dtype=np.int64)
        driver().gd_get_setq(self._w, out.ctypes.data_as(ctypes.POINTER(ctypes.c_long)))
        return out


class Api:
    """One loaded library that exports the libgint_* C-ABI."""

    def __init__(self, so_path):
        self.path = so_path
        self._a = driver().gd_api_open(so_path.encode())
        if not self._a:
            raise RuntimeError(f"cannot load the libgint C-ABI from {so_path}")

    def symbol(self, name, restype=None, argtypes=None):
        addr = driver().gd_api_symbol(self._a, name.encode())
        if not addr:
            return None
        return ctypes.CFUNCTYPE(restype, *(argtypes or []))(addr)


class Session:
    """A handle of one library set up for one workload (everything before set_P)."""

    def __init__(self, api, wl, max_mem_mb=7000):
        self.api, self.wl = api, wl
        self.h = driver().gd_setup(wl._w, api._a, max_mem_mb)

    def build_K(self, P=None, q0=0, q1=-1):
        """One K build (set_P, add_* stream, get_K). Returns (K_flat, wall_ms, [setP, stream, getK] ms)."""
        K = np.zeros(self.wl.info["flat_size"])
        t = np.zeros(3)
        Pp = None if P is None else _dp(np.ascontiguousarray(P, dtype=np.float64))
        ms = driver().gd_build_K(self.wl._w, self.api._a, self.h, Pp, _dp(K), q0, q1, _dp(t))
        return K, ms, t

    def build_K_subset(self, idx, P=None):
        """K build over the listed set quartets only."""
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        K = np.zeros(self.wl.info["flat_size"])
        t = np.zeros(3)
        Pp = None if P is None else _dp(np.ascontiguousarray(P, dtype=np.float64))
        ms = driver().gd_build_K_subset(self.wl._w, self.api._a, self.h, Pp, _dp(K),
                                        idx.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), idx.size, _dp(t))
        return K, ms, t

    def close(self):
        if self.h:
            driver().gd_teardown(self.api._a, self.h)
            self.h = None




class MultiSession:
    """nthreads handles of one library, driven by nthreads host threads (one handle per thread,
    as a caller with one handle per OpenMP thread uses the C-ABI); each thread streams a
    contiguous share of the set quartets.

    team=False: independent threads, each with its own K array; the threads' K are summed.
    team=True:  the threads form one OpenMP team and pass one shared K array, as CP2K does; the
                library's collective set_P/get_K leave the whole K in it (libraries without
                team-collective calls, such as the oracle, cannot be driven this way)."""

    def __init__(self, api, wl, nthreads, max_mem_mb=1000, team=False):
        self.api, self.wl, self.n, self.team = api, wl, int(nthreads), bool(team)
        self.hs = [driver().gd_setup(wl._w, api._a, max_mem_mb) for _ in range(self.n)]

    def build_K(self, P=None, idx=None):
        """One K build over all set quartets, or over the listed ones. Returns (K_flat, wall_ms,
        times): times[0..2] thread 0's set_P / stream / get_K, [3] the slowest thread's build,
        [4] the summation of the threads' K (ms). The split over threads is computed once per
        set-quartet list."""
        K = np.zeros(self.wl.info["flat_size"])
        t = np.zeros(5)
        Pp = None if P is None else _dp(np.ascontiguousarray(P, dtype=np.float64))
        arr = (ctypes.c_void_p * self.n)(*self.hs)
        if idx is None:
            ip, n, key = None, 0, None
        else:
            idx = np.ascontiguousarray(idx, dtype=np.int64)
            ip, n, key = idx.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), idx.size, (idx.size, int(idx[0]) if idx.size else 0,
                                                                                          int(idx[-1]) if idx.size else 0)
        if getattr(self, "_cut_key", "unset") != key:
            self._cut = np.zeros(self.n + 1, dtype=np.int64)
            driver().gd_mt_split(self.wl._w, ip, n, self.n, self._cut.ctypes.data_as(ctypes.POINTER(ctypes.c_long)))
            self._cut_key = key
            self._idx = idx
        fn = driver().gd_build_K_team if self.team else driver().gd_build_K_mt
        ms = fn(self.wl._w, self.api._a, arr, self.n, Pp, _dp(K), ip,
                self._cut.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), _dp(t))
        if ms < 0:
            raise RuntimeError(f"the OpenMP team did not get {self.n} threads")
        return K, ms, t

    def close(self):
        for h in self.hs:
            if h:
                driver().gd_teardown(self.api._a, h)
        self.hs = []


class SystemBatch:
    """Several independent systems driven through ONE handle: their sets are registered one after
    another and their packed P/K arrays concatenated, so the engine batches all their quartets into
    one class-sorted list (and one recorded replay). Every set quartet lies within one system."""

    def __init__(self, workloads):
        self.wls = list(workloads)
        self._arr = (ctypes.c_void_p * len(self.wls))(*[w._w for w in self.wls])
        self.flat = np.array([w.info["flat_size"] for w in self.wls], dtype=np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.flat)])
        self.info = {k: sum(w.info[k] for w in self.wls) for k in ("n_setq", "n_shells", "n_prims", "n_qrtt", "n_sets")}

    def setup(self, api, max_mem_mb=7000):
        return driver().gd_setup_multi(self._arr, len(self.wls), api._a, max_mem_mb)

    def build_K(self, api, h):
        """One K build of every system through handle h: (K of each system, wall ms)."""
        K = np.zeros(int(self.offsets[-1]))
        t = np.zeros(3)
        ms = driver().gd_build_K_multi(self._arr, len(self.wls), api._a, h, _dp(K), _dp(t))
        return self.split(K), ms

    def split(self, K):
        return [K[self.offsets[i]:self.offsets[i + 1]] for i in range(len(self.wls))]

    def exchange_energies(self, Ks):
        return np.array([w.exchange_energy(k) for w, k in zip(self.wls, Ks)])


def cluster_batch(n_systems=96, seed=0, min_mol=2, max_mol=24, setq_stride=1, threads=0):
    """Independent non-periodic water clusters of min_mol..max_mol molecules (uniform, one seed per
    system), alternating the l <= 2 and l <= 3 bases, at the 4-molecule system's density (12 A box
    for 4 molecules), each with 5 occupied orbitals per molecule."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(min_mol, max_mol + 1, size=n_systems)
    wls = []
    for k, m in enumerate(sizes):
        basis = 3 if k % 2 else 2
        wls.append(Workload(None, seed=seed * 100003 + k + 1, setq_stride=setq_stride, threads=threads,
                            n_mol=int(m), box_ang=12.0 * (m / 4.0) ** (1.0 / 3.0), periodic=0, n_img_1d=1,
                            basis=basis, n_occ=5 * int(m)))
    return SystemBatch(wls)


def set_fp32_threshold(thr):
    """Mixed precision for the following K builds: every build sets this threshold in libraries
    that export libgint_set_fp32_threshold and passes each shell quartet's screening bound
    (libgint_add_shell_bound) before its add_shell; 0 turns it off (FP64)."""
    driver().gd_set_fp32_threshold(float(thr))


def set_bulk(on):
    """Stream the set quartets through libgint_add_set_quartets (one call per chunk of set
    quartets) instead of the per-item add_* calls, for libraries that export it."""
    driver().gd_set_bulk(1 if on else 0)
