"""The engine library exports the C-ABI of include/libgint.h; host-side validation of the
stream works without a GPU (no device work is issued by these calls)."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT


def _declared():
    txt = open(os.path.join(ROOT, "include", "libgint.h")).read()
    return sorted(set(re.findall(r"\b(libgint_\w+)\s*\(", txt)))


def test_header_symbols_exported():
    from libgint_b200.capi import SIGNATURES, load_engine
    lib = load_engine()
    names = _declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    # the Python binding declares every symbol the header declares
    assert set(names) <= set(SIGNATURES), set(names) - set(SIGNATURES)


def test_reference_entry_points_present():
    """Every extern "C" entry point of the reference's src/extern_functions.cpp exists."""
    from libgint_b200.capi import load_engine
    lib = load_engine()
    ref = ["libgint_create_handle", "libgint_init", "libgint_set_Potential_Truncated", "libgint_set_hf_fac",
           "libgint_set_max_mem", "libgint_set_P", "libgint_set_P_polarized", "libgint_set_K",
           "libgint_set_K_polarized", "libgint_get_K", "libgint_get_K_polarized", "libgint_set_cell",
           "libgint_set_neighs", "libgint_set_Atom", "libgint_set_Atom_L", "libgint_set_AtomInfo",
           "libgint_add_prm", "libgint_add_shell", "libgint_add_cell", "libgint_add_qrt",
           "libgint_add_qrtt", "libgint_add_set", "libgint_dispatch"]
    for n in ref:
        assert hasattr(lib, n), n


def _handle():
    from libgint_b200.capi import LibGint
    return LibGint()


def test_limits_are_errors_not_aborts():
    g = _handle()
    R = np.zeros(3)
    g.set_Atom(0, R, np.arange(1.0, 18.0))          # 17 primitives > 16
    code, msg = g.last_error()
    assert code != 0 and "np" in msg
    g.close()
    g = _handle()
    g.set_Atom(0, R, np.array([1.0, 2.0]))
    g.set_Atom_L(0, 4, 1, np.array([1.0, 1.0]))      # l = 4 > 3
    assert g.last_error()[0] != 0
    g.close()
    g = _handle()
    g.add_qrtt(1.0, 0, 0, 0, 0, 0, 0, 0, 0, 300, 1, 1, 1, 0, 0, 0, 0, False, False, False, False)
    assert g.last_error()[0] != 0                   # leading dimension >= 256
    g.close()


def test_stream_validation():
    g = _handle()
    R = np.zeros(3)
    for s in range(2):
        g.set_Atom(s, R, np.array([1.0, 0.5]))
        g.set_Atom_L(s, 0, 1, np.array([0.5, 0.5]))
    g.set_neighs(np.zeros(3))
    g.add_prm(0, 0, 5, 0)                           # primitive index 5 >= 2
    g.add_shell(0, 1, 0, 1, 0, 0)
    code, msg = g.last_error()
    assert code != 0 and "primitive" in msg
    g.close()
    g = _handle()
    for s in range(2):
        g.set_Atom(s, R, np.array([1.0]))
        g.set_Atom_L(s, 0, 1, np.array([1.0]))
    g.add_prm(0, 0, 0, 0)
    g.add_shell(0, 1, 0, 7, 0, 0)                   # set 7 undefined
    assert g.last_error()[0] != 0
    g.close()


def test_qrtt_count_mismatch_is_reported():
    g = _handle()
    R = np.zeros(3)
    for s in range(2):
        g.set_Atom(s, R, np.array([1.0]))
        g.set_Atom_L(s, 0, 2, np.array([1.0, 0.5]))  # two contractions
    g.add_prm(0, 0, 0, 0)
    g.add_shell(0, 1, 0, 1, 0, 0)
    g.add_qrt(0, 0, 0, 0, 2, 2, 2, 2)
    g.add_qrtt(1.0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 0, 0, 0, 0, False, False, False, False)
    g.add_set()                                     # 1 row for 16 contraction combinations
    code, msg = g.last_error()
    assert code != 0 and "add_qrtt" in msg
    g.close()
