"""Parity with the reference libGint CUDA library on the same B200 and the same call stream.

oracle/_ref/libref_gint.so is the reference's own CUDA code (src/*.cpp), compiled unchanged for
sm_100a by `make -C oracle ref` in the development container; it travels with the tree. Both
libraries receive the identical add_* stream from the workload driver. The reference sums K with
atomics in a nondeterministic order; the bound is 1e-12 * max|K| for l <= 3.

The reference's own K depends on its batch size (libgint_set_max_mem). For the l = 3 system
below, multi-GB batches drift from run to run by ~3e-10 of max|K| (2.8e-10 and 3.3e-10 in two
runs of the same input) while 150 MB batches agree with the oracle to 1.6e-13; other systems
make its batch memset fail ("invalid argument", after which it exits) at small batch sizes. Each
case therefore names a batch size at which the reference is known to run and agree with itself,
and the reference runs in a child process (tests/ref_runner.py). The engine's and the oracle's K
do not depend on the batch size.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import ORACLE_SO, REF_GINT_SO
from libgint_b200.workload import Api, Session, Workload

TOL = 1e-12

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(REF_GINT_SO), reason="reference CUDA build absent")]


def _build(path, wl):
    s = Session(Api(path), wl)
    K, ms, _ = s.build_K()
    return K, ms


def _ref(spec, max_mem_mb=7000):
    from ref_runner import reference_K
    return reference_K(dict(spec), max_mem_mb)


def test_small_l2_matches_reference_cuda(engine_so):
    wl = Workload("small_l2")
    Kr, ms_r = _ref({"name": "small_l2"})
    Ke, ms_e = _build(engine_so, wl)
    Ko, _ = _build(ORACLE_SO, wl)
    scale = np.abs(Kr).max()
    rel_e = np.abs(Ke - Kr).max() / scale
    rel_o = np.abs(Ko - Kr).max() / scale
    print(f"small_l2: engine vs reference {rel_e:.3e}, oracle vs reference {rel_o:.3e}, "
          f"E_x ref {wl.exchange_energy(Kr):.12f} engine {wl.exchange_energy(Ke):.12f}; "
          f"reference {ms_r:.1f} ms engine {ms_e:.1f} ms")
    assert rel_o <= TOL
    assert rel_e <= TOL


def test_periodic_small_matches_reference_cuda(engine_so):
    wl = Workload("periodic_l2", n_mol=3, box_ang=7.0, n_occ=20)
    Kr, ms_r = _ref({"name": "periodic_l2", "n_mol": 3, "box_ang": 7.0, "n_occ": 20})
    Ke, ms_e = _build(engine_so, wl)
    scale = np.abs(Kr).max()
    rel = np.abs(Ke - Kr).max() / scale
    print(f"periodic 3 molecules: engine vs reference {rel:.3e}; reference {ms_r:.1f} ms engine {ms_e:.1f} ms")
    assert rel <= TOL


def test_periodic_l3_matches_reference_cuda(engine_so):
    spec = {"name": "periodic_l3", "n_mol": 2, "box_ang": 6.5, "n_img_1d": 3, "n_occ": 16, "max_prm": 3,
            "max_ncontr": 2}
    wl = Workload(**spec)
    Kr, ms_r = _ref(spec, max_mem_mb=150)
    Ke, ms_e = _build(engine_so, wl)
    scale = np.abs(Kr).max()
    rel = np.abs(Ke - Kr).max() / scale
    dex = abs(wl.exchange_energy(Ke) - wl.exchange_energy(Kr))
    print(f"periodic l3 (f shells, general contractions): engine vs reference {rel:.3e}, |dEx| {dex:.3e}; "
          f"reference {ms_r:.1f} ms engine {ms_e:.1f} ms")
    assert rel <= TOL
