"""Parity of the CUDA engine with the CPU oracle on identical call streams (through the C-ABI).

FP64 path: the tolerance is max|K_engine - K_oracle| <= 1e-11 * max|K_oracle| for every class up
to l = 3 (the engine sums in a different order than the oracle and uses FMA; both are FP64).

Decisions are exact, not within a tolerance: the minimum-image shift of P - Q, the truncation
test, the Boys/Chebyshev branch and the patch index are evaluated with the same rounded
operations on both sides. That matters for symmetric quartets, (ab|ab') with b' an image of b and
equal exponents, where P - Q lies exactly on half a lattice vector: there one ulp of P or Q moves
the 27-image window by a cell and changes K by up to ~5e-8 of max|K| on the l = 3 systems below.
"""
import numpy as np
import pytest

from libgint_b200.workload import Api, Session, Workload

TOL = 1e-11


def _k(api_path, wl):
    api = Api(api_path)
    s = Session(api, wl)
    K, ms, _ = s.build_K()
    err = api.symbol("libgint_last_error", restype=__import__("ctypes").c_int,
                     argtypes=[__import__("ctypes").c_void_p])
    code = err(s.h) if err else 0
    s.close()
    return K, ms, code


def _compare(engine_so, oracle_path, wl, tol=TOL):
    Ke, ms_e, code = _k(engine_so, wl)
    assert code == 0
    Ko, ms_o, _ = _k(oracle_path, wl)
    scale = np.abs(Ko).max()
    assert scale > 0
    rel = np.abs(Ke - Ko).max() / scale
    ex_e, ex_o = wl.exchange_energy(Ke), wl.exchange_energy(Ko)
    print(f"{wl.name or 'custom'}: shells={wl.info['n_shells']} prims={wl.info['n_prims']} "
          f"rel max|dK|={rel:.3e} |dEx|={abs(ex_e-ex_o):.3e} engine {ms_e:.1f} ms oracle {ms_o:.1f} ms")
    assert rel <= tol, rel
    assert abs(ex_e - ex_o) <= tol * max(1.0, abs(ex_o))
    return rel


@pytest.mark.gpu
def test_small_l2_vs_oracle(engine_so, oracle_path):
    _compare(engine_so, oracle_path, Workload("small_l2"))


@pytest.mark.gpu
def test_periodic_l2_small_vs_oracle(engine_so, oracle_path):
    wl = Workload("periodic_l2", n_mol=3, box_ang=7.0, n_occ=20)
    _compare(engine_so, oracle_path, wl)


@pytest.mark.gpu
def test_periodic_l3_general_contraction_vs_oracle(engine_so, oracle_path):
    wl = Workload("periodic_l3", n_mol=2, box_ang=6.5, n_img_1d=3, n_occ=16, max_prm=3, max_ncontr=2)
    _compare(engine_so, oracle_path, wl)


@pytest.mark.gpu
def test_ill_conditioned_general_contraction_vs_reference(engine_so, oracle_path):
    """Two primitives per set with N(0,1) general contractions: the normalised coefficients reach
    2.4e4 with cancelling signs, so (ff|..) classes amplify rounding by ~1e8. The system also holds
    half-lattice-vector ties of P - Q; evaluating the weighted distances without the reference's
    FMA moves K by 5e-8 of max|K|. Checked against the oracle and against the reference CUDA build
    (in a child process: the reference exits on a CUDA API error)."""
    import os
    from conftest import REF_GINT_SO
    wl = Workload("periodic_l3", n_mol=1, box_ang=5.0, n_img_1d=3, n_occ=8, max_prm=2, max_ncontr=2)
    _compare(engine_so, oracle_path, wl)
    if os.path.exists(REF_GINT_SO):
        from ref_runner import reference_K
        Ke, _, _ = _k(engine_so, wl)
        Kr, _ = reference_K({"name": "periodic_l3", "n_mol": 1, "box_ang": 5.0, "n_img_1d": 3, "n_occ": 8,
                             "max_prm": 2, "max_ncontr": 2}, 7000)
        rel = np.abs(Ke - Kr).max() / np.abs(Kr).max()
        print(f"ill-conditioned l3: engine vs reference {rel:.3e}")
        assert rel <= TOL, rel


@pytest.mark.gpu
def test_record_replay_matches_stream(engine_so):
    """K recomputed from the recorded device batches equals K of the streamed build."""
    import ctypes
    from libgint_b200.capi import load_engine
    lib = load_engine()
    wl = Workload("small_l2")
    s = Session(Api(engine_so), wl)
    h = ctypes.c_void_p(s.h)
    lib.libgint_record(h, 1)
    K1, _, _ = s.build_K()
    lib.libgint_record(h, 0)
    P = wl.Pflat
    lib.libgint_set_P(h, P.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), P.size)
    ms = lib.libgint_replay(h)
    K2 = np.zeros_like(K1)
    lib.libgint_get_K(h, K2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert ms > 0 and lib.libgint_last_error(h) == 0
    assert np.abs(K1 - K2).max() <= 1e-13 * np.abs(K1).max()
    # a scaled density gives a scaled K (K is linear in P)
    P2 = 0.5 * P
    lib.libgint_set_P(h, P2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), P2.size)
    lib.libgint_replay(h)
    lib.libgint_get_K(h, K2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert np.abs(0.5 * K1 - K2).max() <= 1e-13 * np.abs(K1).max()
    s.close()


@pytest.mark.gpu
def test_multi_batch_replay_matches_stream(engine_so):
    """A recording of many batches replays to the streamed K, twice in a row. The worker streams
    run consecutive batches at the same time, so each batch must keep its own image-summed
    targets (the two halves of the replay buffer) until the batch after next."""
    import ctypes
    from libgint_b200.capi import load_engine
    lib = load_engine()
    wl = Workload("periodic_l2_small")
    s = Session(Api(engine_so), wl, max_mem_mb=150)
    h = ctypes.c_void_p(s.h)
    lib.libgint_record(h, 1)
    K1, _, _ = s.build_K()
    lib.libgint_record(h, 0)
    stats = (ctypes.c_longlong * 8)()
    lib.libgint_get_stats(h, stats)
    assert stats[3] >= 4, f"expected a recording of several batches, got {stats[3]}"
    P = wl.Pflat
    lib.libgint_set_P(h, P.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), P.size)
    K2 = np.zeros_like(K1)
    for _ in range(2):
        assert lib.libgint_replay(h) > 0 and lib.libgint_last_error(h) == 0
        lib.libgint_get_K(h, K2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert np.abs(K1 - K2).max() <= 1e-13 * np.abs(K1).max()
    s.close()


@pytest.mark.gpu
def test_out_of_range_update_is_an_error(engine_so):
    """An add_qrtt offset beyond P_size is caught by the kernel's bounds check (no fault)."""
    from libgint_b200.capi import LibGint
    g = LibGint()
    g.init()
    wl = Workload("small_l2")
    C0 = wl.C0
    g.set_Potential_Truncated(wl.info["rc_bohr"], C0, wl.info["ld_C0"])
    g.set_max_mem(500)
    g.set_cell(False, np.eye(3).ravel() * 1024.0, np.eye(3).ravel() / 1024.0)
    g.set_neighs(np.zeros(3))
    for s in range(2):
        g.set_Atom(s, np.array([0.0, 0.0, 1.0 * s]), np.array([1.0]))
        g.set_Atom_L(s, 0, 1, np.array([1.0]))
    g.set_P(np.ones(16))
    g.add_prm(0, 0, 0, 0)
    g.add_shell(0, 1, 0, 1, 0, 0)
    g.add_qrt(0, 0, 0, 0, 1, 1, 1, 1)
    g.add_qrtt(1.0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 0, 0, 1000, 0, False, False, False, False)
    g.add_set()
    g.get_K(16)
    code, msg = g.last_error()
    assert code == 3 and "outside" in msg
    g.close()


@pytest.mark.gpu
def test_multithreaded_caller_matches_oracle(engine_so, oracle_path):
    """Four host threads with one engine handle each on one GPU (contiguous shares of the set
    quartets, K summed): the oracle's K within the FP64 tolerance."""
    from libgint_b200.workload import MultiSession
    wl = Workload("periodic_l2_small")
    m = MultiSession(Api(engine_so), wl, 4)
    Ke, ms, _ = m.build_K()
    m.close()
    Ko, _, _ = _k(oracle_path, wl)
    rel = np.abs(Ke - Ko).max() / np.abs(Ko).max()
    print(f"4 caller threads: engine vs oracle {rel:.3e}, {ms:.1f} ms")
    assert rel <= TOL, rel


@pytest.mark.gpu
def test_bulk_submission_matches_stream(engine_so, oracle_path):
    """libgint_add_set_quartets (the bulk form of the add_* stream) gives the per-item stream's K."""
    from libgint_b200.workload import set_bulk
    wl = Workload("small_l2")
    Ke, _, code = _k(engine_so, wl)
    assert code == 0
    set_bulk(True)
    try:
        Kb, _, code_b = _k(engine_so, wl)
    finally:
        set_bulk(False)
    assert code_b == 0
    rel = np.abs(Kb - Ke).max() / np.abs(Ke).max()
    print(f"bulk submission vs per-item stream: {rel:.3e}")
    assert rel <= TOL, rel
