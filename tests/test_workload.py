"""The workload generator / replayer (the stand-in caller) and the oracle on small systems."""
import numpy as np
import pytest

from conftest import ORACLE_SO
from libgint_b200.workload import Api, MultiSession, Session, Workload, set_bulk


def test_deterministic():
    a, b = Workload("small_l2"), Workload("small_l2")
    assert a.info == b.info
    assert np.array_equal(a.P, b.P)
    assert np.array_equal(a.setq(), b.setq())
    c = Workload("small_l2", seed=1)
    assert c.info["n_setq"] != a.info["n_setq"] or not np.array_equal(c.P, a.P)


def test_density_is_a_projector():
    w = Workload("small_l2")
    n = w.n_bf
    P = w.P.reshape(n, n)
    assert np.allclose(P, P.T)
    assert np.allclose(P @ P, 2.0 * P, atol=1e-10)
    assert abs(np.trace(P) - 2 * 20) < 1e-9


def test_packed_layout_roundtrip():
    """P in the packed set-pair layout unpacks (as a K would) to the dense P."""
    w = Workload("small_l2")
    n = w.n_bf
    # unpack_K halves and symmetrises: feed 2x the lower-triangle blocks, which for a symmetric
    # input returns the matrix itself
    Pd = w.P.reshape(n, n)
    flat = w.Pflat
    K = w.unpack_K(flat)
    sets = w.sets()
    for x in range(len(sets)):
        bx, lx, nlx, _ = sets[x]
        nx = (2 * lx + 1) * nlx
        blk = K[bx:bx + nx, bx:bx + nx]
        assert np.allclose(blk, Pd[bx:bx + nx, bx:bx + nx])


def test_unique_quartets_reproduce_full_enumeration():
    """K from the unique set quartets with symmetry factors equals K from all (i,j,k,l) with
    factor 1/4, up to the reference's unscreened (00|00) contributions (see the oracle)."""
    ora = Api(ORACLE_SO)
    wu = Workload("small_l2")
    wf = Workload("small_l2", full_enum=True)
    Ku = wu.unpack_K(Session(ora, wu).build_K()[0])
    Kf = wf.unpack_K(Session(ora, wf).build_K()[0])
    rel = np.abs(Ku - Kf).max() / np.abs(Kf).max()
    assert rel < 1e-7, rel
    assert np.allclose(Ku, Ku.T)


def test_oracle_thread_count_invariance():
    import ctypes
    ora = Api(ORACLE_SO)
    w = Workload("small_l2")
    s1 = Session(ora, w)
    set_threads = ora.symbol("oracle_set_threads", None, [ctypes.c_void_p, ctypes.c_int])
    set_threads(s1.h, 1)
    K1 = s1.build_K()[0]
    s8 = Session(ora, w)
    K8 = s8.build_K()[0]
    assert np.abs(K1 - K8).max() <= 1e-12 * np.abs(K1).max()


def test_exchange_energy_negative_and_stable():
    ora = Api(ORACLE_SO)
    w = Workload("small_l2")
    K = Session(ora, w).build_K()[0]
    ex = w.exchange_energy(K)
    assert ex < 0
    # subset replays add up to the full K (K is additive over set quartets)
    s = Session(ora, w)
    nq = w.info["n_setq"]
    Ka = s.build_K_subset(np.arange(0, nq, 2))[0]
    Kb = s.build_K_subset(np.arange(1, nq, 2))[0]
    assert np.abs(Ka + Kb - K).max() <= 1e-12 * np.abs(K).max()


def test_multithreaded_caller_sums_to_single_handle():
    """Three host threads with one handle each (contiguous shares of the set quartets) give the
    single-handle K up to summation order."""
    import ctypes
    ora = Api(ORACLE_SO)
    w = Workload("small_l2")
    s1 = Session(ora, w)
    K1 = s1.build_K()[0]
    s1.close()
    m = MultiSession(ora, w, 3)
    set_threads = ora.symbol("oracle_set_threads", None, [ctypes.c_void_p, ctypes.c_int])
    for h in m.hs:
        set_threads(h, 1)
    Km, ms, _ = m.build_K()
    idx = np.arange(0, w.info["n_setq"], 2)
    Ks, _, _ = m.build_K(idx=idx)
    m.close()
    assert ms > 0
    assert np.abs(Km - K1).max() <= 1e-13 * np.abs(K1).max()
    s2 = Session(ora, w)
    K2 = s2.build_K_subset(idx)[0]
    s2.close()
    assert np.abs(Ks - K2).max() <= 1e-13 * np.abs(K2).max()


def test_bulk_stream_equals_per_item_stream():
    """libgint_add_set_quartets carries the same call stream: identical K from the oracle."""
    import ctypes
    ora = Api(ORACLE_SO)
    w = Workload("small_l2")
    s = Session(ora, w)
    set_threads = ora.symbol("oracle_set_threads", None, [ctypes.c_void_p, ctypes.c_int])
    set_threads(s.h, 1)     # one summation order, so the two K agree bit for bit
    K1 = s.build_K()[0]
    set_bulk(True)
    try:
        K2 = s.build_K()[0]
    finally:
        set_bulk(False)
    s.close()
    assert np.array_equal(K1, K2)
