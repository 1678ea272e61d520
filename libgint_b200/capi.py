"""ctypes binding of the engine's C-ABI with the reference's method names.

`LibGint` mirrors `module libgint` of the reference (src/interface_libgint.F90:236-241) and the
C entry points (src/extern_functions.cpp:9-190): set_* calls, the add_* stream and get_K. The
engine library must be present; nothing here falls back to another implementation.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_V = ctypes.c_void_p

# name -> (restype, argtypes); declared in include/libgint.h
SIGNATURES = {
    "libgint_create_handle": (_V, []),
    "libgint_init": (None, [_V]),
    "libgint_set_Potential_Truncated": (None, [_V, ctypes.c_double, _D, ctypes.c_int, ctypes.c_int]),
    "libgint_set_hf_fac": (None, [_V, ctypes.c_double]),
    "libgint_set_max_mem": (None, [_V, ctypes.c_int]),
    "libgint_set_P": (None, [_V, _D, ctypes.c_int]),
    "libgint_set_P_polarized": (None, [_V, _D, _D, ctypes.c_int]),
    "libgint_set_K": (None, [_V, _D, ctypes.c_int]),
    "libgint_set_K_polarized": (None, [_V, _D, _D, ctypes.c_int]),
    "libgint_get_K": (None, [_V, _D]),
    "libgint_get_K_polarized": (None, [_V, _D, _D]),
    "libgint_set_cell": (None, [_V, ctypes.c_bool, _D, _D]),
    "libgint_set_neighs": (None, [_V, _D, ctypes.c_int]),
    "libgint_set_Atom": (None, [_V, ctypes.c_int, _D, _D, ctypes.c_int]),
    "libgint_set_Atom_L": (None, [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]),
    "libgint_set_AtomInfo": (None, [_V, ctypes.c_int, _D, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, _I, _D]),
    "libgint_add_prm": (None, [_V] + [ctypes.c_int] * 4),
    "libgint_add_shell": (None, [_V] + [ctypes.c_int] * 6),
    "libgint_add_cell": (None, [_V]),
    "libgint_add_qrt": (None, [_V] + [ctypes.c_int] * 8),
    "libgint_add_qrtt": (None, [_V, ctypes.c_double] + [ctypes.c_int] * 12 + [ctypes.c_uint] * 4
                         + [ctypes.c_bool] * 4),
    "libgint_add_set": (None, [_V]),
    "libgint_dispatch": (None, [_V]),
    "libgint_last_error": (ctypes.c_int, [_V]),
    "libgint_error_string": (ctypes.c_char_p, [_V]),
    "libgint_destroy_handle": (None, [_V]),
    "libgint_plan_sizes": (ctypes.c_int, [ctypes.c_int] * 4 + [_I]),
    "libgint_hrr_program": (ctypes.c_int, [ctypes.c_int] * 4 + [ctypes.POINTER(ctypes.c_uint), ctypes.c_int, _I]),
    "libgint_vrr_program": (ctypes.c_int, [ctypes.c_int] * 4 + [_V, ctypes.c_int, _I, ctypes.c_int]),
    "libgint_record": (None, [_V, ctypes.c_int]),
    "libgint_replay": (ctypes.c_double, [_V]),
    "libgint_replay_incremental": (ctypes.c_double, [_V, ctypes.c_double]),
    "libgint_replay_profile": (ctypes.c_double, [_V, _D]),
    "libgint_replay_noalloc": (ctypes.c_int, [_V, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "libgint_add_set_quartets": (ctypes.c_int, [_V, ctypes.c_int] + [ctypes.c_void_p] * 11),
    "libgint_replay_profile_classes": (ctypes.c_double, [_V, _D, _D]),
    "libgint_plan_flops": (ctypes.c_int, [ctypes.c_int] * 4 + [_D]),
    "libgint_set_counters": (None, [_V, ctypes.c_int]),
    "libgint_get_counters": (None, [_V, ctypes.POINTER(ctypes.c_ulonglong)]),
    "libgint_get_stats": (None, [_V, ctypes.POINTER(ctypes.c_longlong)]),
    "libgint_fp64_peak_tflops": (ctypes.c_double, []),
    "libgint_host_tables": (None, [_D, _D, ctypes.POINTER(ctypes.c_ubyte), _D]),
    "libgint_set_fp32_threshold": (None, [_V, ctypes.c_double]),
    "libgint_autotune": (ctypes.c_int, [_V, _I]),
    "libgint_set_tuning": (None, [_V, _I]),
    "libgint_get_tuning": (None, [_V, _I]),
    "libgint_add_shell_bound": (None, [_V, ctypes.c_double]),
}


def engine_path():
    return os.path.join(_HERE, "lib", "libgint_b200.so")


_engine = None


def load_engine(path=None):
    """Load the engine's shared library (raises if it has not been built)."""
    global _engine
    if path is None and _engine is not None:
        return _engine
    p = path or engine_path()
    if not os.path.exists(p):
        raise RuntimeError(f"engine library {p} is missing; build it with libgint_b200.build.build_all()")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _engine = lib
    return lib


def _dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_D)


class LibGint:
    """One engine handle; method names follow the reference interface."""

    def __init__(self, lib=None):
        self.lib = lib or load_engine()
        self.h = self.lib.libgint_create_handle()
        self._keep = []

    def init(self):
        self.lib.libgint_init(self.h)

    def set_Potential_Truncated(self, R_cut, C0, ld_C0):
        C0 = np.ascontiguousarray(C0, dtype=np.float64)
        self._keep.append(C0)
        self.lib.libgint_set_Potential_Truncated(self.h, R_cut, _dp(C0), ld_C0, C0.size)

    def set_hf_fac(self, fac):
        self.lib.libgint_set_hf_fac(self.h, fac)

    def set_max_mem(self, mb):
        self.lib.libgint_set_max_mem(self.h, int(mb))

    def set_cell(self, periodic, cell_h, cell_i):
        self.lib.libgint_set_cell(self.h, bool(periodic), _dp(cell_h), _dp(cell_i))

    def set_neighs(self, neighs):
        n = np.ascontiguousarray(neighs, dtype=np.float64).reshape(-1)
        self.lib.libgint_set_neighs(self.h, _dp(n), n.size // 3)

    def set_Atom(self, i, R, Z):
        Z = np.ascontiguousarray(Z, dtype=np.float64)
        self.lib.libgint_set_Atom(self.h, i, _dp(R), _dp(Z), Z.size)

    def set_Atom_L(self, i, l, nl, K):
        self.lib.libgint_set_Atom_L(self.h, i, l, nl, _dp(K))

    def set_P(self, P):
        P = np.ascontiguousarray(P, dtype=np.float64)
        self.lib.libgint_set_P(self.h, _dp(P), P.size)

    def set_K(self, K):
        K = np.ascontiguousarray(K, dtype=np.float64)
        self.lib.libgint_set_K(self.h, _dp(K), K.size)

    def add_prm(self, ipa, ipb, ipc, ipd):
        self.lib.libgint_add_prm(self.h, ipa, ipb, ipc, ipd)

    def add_shell(self, i, j, k, l, n1, n2):
        self.lib.libgint_add_shell(self.h, i, j, k, l, n1, n2)

    def add_qrt(self, la, lb, lc, ld, nla, nlb, nlc, nld):
        self.lib.libgint_add_qrt(self.h, la, lb, lc, ld, nla, nlb, nlc, nld)

    def add_qrtt(self, symm_fac, la, lb, lc, ld, inla, inlb, inlc, inld, ld_ac, ld_ad, ld_bc, ld_bd,
                 off_ac, off_ad, off_bc, off_bd, Tac, Tad, Tbc, Tbd):
        self.lib.libgint_add_qrtt(self.h, symm_fac, la, lb, lc, ld, inla, inlb, inlc, inld,
                                  ld_ac, ld_ad, ld_bc, ld_bd, off_ac, off_ad, off_bc, off_bd,
                                  Tac, Tad, Tbc, Tbd)

    def add_set(self):
        self.lib.libgint_add_set(self.h)

    def dispatch(self):
        self.lib.libgint_dispatch(self.h)

    def get_K(self, size):
        K = np.zeros(size)
        self.lib.libgint_get_K(self.h, K.ctypes.data_as(_D))
        return K

    def last_error(self):
        return self.lib.libgint_last_error(self.h), self.lib.libgint_error_string(self.h).decode()

    def close(self):
        if self.h:
            self.lib.libgint_destroy_handle(self.h)
            self.h = None
