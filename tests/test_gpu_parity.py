"""Parity of the CUDA engine with the CPU oracle on identical call streams (through the C-ABI).

FP64 path, two bounds (the engine sums in a different order than the oracle and uses FMA; both
are FP64):
  * every element: |K_engine - K_oracle| <= 1e-13 * Kabs, Kabs being the oracle's K evaluated
    with every factor replaced by its magnitude (the sum of the magnitudes of the terms each
    element adds up, the scale of any FP64 evaluation's rounding error); E_x likewise;
  * for well-conditioned systems (max Kabs < 1e3 max|K|, every l <= 2 system and the small-
    contraction l = 3 ones): max|K_engine - K_oracle| <= 1e-12 * max|K_oracle|.
The l <= 3 basis of the 64-molecule workload (16-primitive sets with 4 N(0,1) general
contractions) is ill-conditioned: there max Kabs / max|K| is ~1e7, and the oracle differs from
itself with the primitives summed in reverse order by 3e-11 of max|K| (at 5e-16 Kabs), so only the
element-wise bound is meaningful for it.

Decisions are exact, not within a tolerance: the minimum-image shift of P - Q, the truncation
test, the Boys/Chebyshev branch, the patch index and the Fm[0] > 1e-12 screen are evaluated with
the same rounded operations on both sides, and the tests compare the per-class decision counters
of the two (Chebyshev evaluations, Boys evaluations, images through the VRR, primitive quartets)
for equality. That matters for symmetric quartets, (ab|ab') with b' an image of b and equal
exponents, where P - Q lies exactly on half a lattice vector: there one ulp of P or Q moves the
image window by a cell and changes K by up to ~5e-8 of max|K| on the l = 3 systems below.
"""
import ctypes

import numpy as np
import pytest

from libgint_b200.workload import Api, Session, Workload

TOL = 1e-12


def _k(api_path, wl, counters=False, max_mem_mb=7000):
    """One K build through the C-ABI of the library at api_path: (K, ms, error code, counters)."""
    api = Api(api_path)
    s = Session(api, wl, max_mem_mb=max_mem_mb)
    V = ctypes.c_void_p
    cnt = None
    if counters:
        api.symbol("libgint_set_counters", None, [V, ctypes.c_int])(s.h, 1)
    K, ms, _ = s.build_K()
    if counters:
        buf = (ctypes.c_ulonglong * 1024)()
        api.symbol("libgint_get_counters", None, [V, ctypes.POINTER(ctypes.c_ulonglong)])(s.h, buf)
        cnt = np.frombuffer(buf, dtype=np.uint64).reshape(256, 4).copy()
    err = api.symbol("libgint_last_error", restype=ctypes.c_int, argtypes=[V])
    code = err(s.h) if err else 0
    s.close()
    return K, ms, code, cnt


ELEM_TOL = 1e-13
WELL_CONDITIONED = 1e3


def magnitude_K(oracle_path, wl):
    """The oracle's K with every factor replaced by its magnitude (see the module docstring)."""
    api = Api(oracle_path)
    s = Session(api, wl)
    api.symbol("oracle_set_absmode", None, [ctypes.c_void_p, ctypes.c_int])(s.h, 1)
    K, _, _ = s.build_K()
    s.close()
    return K


def assert_fp64_parity(Ke, Ko, Kabs, wl, label=""):
    """The two bounds of the module docstring; returns (max relative difference, conditioning)."""
    scale = np.abs(Ko).max()
    assert scale > 0
    d = np.abs(Ke - Ko)
    rel = d.max() / scale
    cond = Kabs.max() / scale
    elem = (d / np.maximum(Kabs, 1e-300)).max()
    ex_e, ex_o = wl.exchange_energy(Ke), wl.exchange_energy(Ko)
    ex_scale = 0.25 * float(np.sum(np.abs(wl.P.reshape(wl.n_bf, wl.n_bf)) * wl.unpack_K(Kabs)))
    print(f"{label}{wl.name or 'custom'}: shells={wl.info['n_shells']} prims={wl.info['n_prims']} "
          f"rel max|dK|={rel:.3e} max|dK|/Kabs={elem:.3e} (Kabs/max|K| {cond:.2e}) |dEx|={abs(ex_e - ex_o):.3e}")
    assert np.all(d <= ELEM_TOL * Kabs + 1e-300), elem
    assert abs(ex_e - ex_o) <= ELEM_TOL * ex_scale + 1e-300
    if cond < WELL_CONDITIONED:
        assert rel <= TOL, rel
        assert abs(ex_e - ex_o) <= TOL * max(1.0, abs(ex_o))
    return rel, cond


def _compare(engine_so, oracle_path, wl, counters=True):
    Ke, ms_e, code, ce = _k(engine_so, wl, counters)
    assert code == 0
    Ko, ms_o, _, co = _k(oracle_path, wl, counters)
    print(f"engine {ms_e:.1f} ms oracle {ms_o:.1f} ms")
    rel, _ = assert_fp64_parity(Ke, Ko, magnitude_K(oracle_path, wl), wl)
    if counters:
        assert_same_decisions(ce, co, wl)
    return rel


def assert_same_decisions(ce, co, wl):
    """The per-class screening decisions of the engine and the oracle are identical: the same
    number of Chebyshev and Boys evaluations (truncation test and branch), of images through the
    VRR (Fm[0] > 1e-12), and of primitive quartets."""
    assert int(co[:, 3].sum()) == wl.info["n_prims"]
    bad = np.nonzero((ce != co).any(axis=1))[0]
    names = ["cheb", "boys", "vrr", "prims"]
    detail = [(f"({c >> 6}{(c >> 4) & 3}|{(c >> 2) & 3}{c & 3})",
               {n: (int(ce[c, i]), int(co[c, i])) for i, n in enumerate(names)}) for c in bad[:6]]
    assert bad.size == 0, f"screening decisions differ (engine, oracle): {detail}"
    print(f"  decisions equal: {int(co[:, 0].sum())} Chebyshev, {int(co[:, 1].sum())} Boys, "
          f"{int(co[:, 2].sum())} VRR images over {int((co[:, 3] > 0).sum())} classes")


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
def test_periodic_l3_full_sets_125_images_vs_oracle(engine_so, oracle_path):
    """The l <= 3 basis of the 64-molecule workload at full size per set (an s set of 16
    primitives with 4 general contractions, so 65536 primitive quartets and 256 contraction rows
    per (ss|ss) shell quartet; p sets of 8 primitives with 3 contractions, d sets of 4 with 2) and
    its 125 image cells, on one molecule in a 6.2 A cell (the workload's density)."""
    wl = Workload("periodic_l3", n_mol=1, box_ang=6.2, n_img_1d=5, n_occ=8)
    assert wl.info["Ng"] == 125
    _compare(engine_so, oracle_path, wl)


@pytest.mark.gpu
def test_periodic_l3_sampled_at_size_vs_oracle(engine_so, oracle_path):
    """A hash sample of the set quartets of the 64-molecule, 125-image l <= 3 workload itself (the
    bench's workload), at a rate the oracle finishes in seconds."""
    wl = Workload("periodic_l3", setq_stride=1 << 16, setq_phase=3)
    assert wl.info["n_setq"] > 0
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
        Ke, _, _, _ = _k(engine_so, wl)
        Kr, _ = reference_K({"name": "periodic_l3", "n_mol": 1, "box_ang": 5.0, "n_img_1d": 3, "n_occ": 8,
                             "max_prm": 2, "max_ncontr": 2}, 7000)
        rel = np.abs(Ke - Kr).max() / np.abs(Kr).max()
        print(f"ill-conditioned l3: engine vs reference {rel:.3e}")
        assert rel <= TOL, rel


@pytest.mark.gpu
def test_record_replay_matches_stream(engine_so):
    """K recomputed from the recorded device batches equals K of the streamed build."""
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
def test_merged_recording_replays_the_same_K_in_fewer_launches(engine_so, oracle_path):
    """libgint_record(h, 2) merges a many-batch recording into one segment per class when it
    stops: its replays (twice in a row, and after the autotuner) give the streamed K and the
    oracle's decisions with fewer launches than the same recording kept as batches."""
    from libgint_b200.capi import load_engine
    lib = load_engine()
    wl = Workload("periodic_l2_small")
    stats = (ctypes.c_longlong * 8)()
    D = ctypes.POINTER(ctypes.c_double)
    P = wl.Pflat
    launches = {}
    for mode in (1, 2):
        s = Session(Api(engine_so), wl, max_mem_mb=150)
        h = ctypes.c_void_p(s.h)
        lib.libgint_record(h, mode)
        K1, _, _ = s.build_K()
        lib.libgint_record(h, 0)
        lib.libgint_get_stats(h, stats)
        assert stats[3] >= 4, f"expected a recording of several batches, got {stats[3]}"
        lib.libgint_set_P(h, P.ctypes.data_as(D), P.size)
        K2 = np.zeros_like(K1)
        for _ in range(2):
            lib.libgint_get_stats(h, stats)
            l0 = int(stats[4])
            assert lib.libgint_replay(h) > 0 and lib.libgint_last_error(h) == 0
            lib.libgint_get_stats(h, stats)
            launches[mode] = int(stats[4]) - l0
            lib.libgint_get_K(h, K2.ctypes.data_as(D))
            assert np.abs(K1 - K2).max() <= 1e-13 * np.abs(K1).max()
        if mode == 2:
            assert lib.libgint_autotune(h, None) == 0
            lib.libgint_set_counters(h, 1)
            assert lib.libgint_replay(h) > 0 and lib.libgint_last_error(h) == 0
            buf = (ctypes.c_ulonglong * 1024)()
            lib.libgint_get_counters(h, buf)
            lib.libgint_set_counters(h, 0)
            lib.libgint_get_K(h, K2.ctypes.data_as(D))
            Ko, _, _, co = _k(oracle_path, wl, counters=True)
            assert_same_decisions(np.frombuffer(buf, dtype=np.uint64).reshape(256, 4).copy(), co, wl)
            assert_fp64_parity(K2, Ko, magnitude_K(oracle_path, wl), wl)
        s.close()
    print(f"{launches[1]} launches per replay as recorded, {launches[2]} merged")
    assert launches[2] < launches[1]


@pytest.mark.gpu
def test_multi_batch_replay_matches_stream(engine_so):
    """A recording of many batches replays to the streamed K, twice in a row. The worker streams
    run the batches' segments side by side, each stream in its own buffer of image-summed
    targets, so no segment may overwrite another's before its group kernel has read them."""
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
    Ko, _, _, _ = _k(oracle_path, wl)
    assert_fp64_parity(Ke, Ko, magnitude_K(oracle_path, wl), wl, f"4 caller threads ({ms:.1f} ms): ")


@pytest.mark.gpu
def test_openmp_team_shares_P_and_K(engine_so, oracle_path):
    """Four OpenMP threads with one handle each pass ONE shared K array, as CP2K's HFX module does
    (src/libGint.cpp:436-447, 613-628): set_P and get_K are collective over the team, every
    handle's kernels add into the team's one device K, and after get_K the shared array holds the
    whole K (no summation by the caller). Run twice, so the second build reuses the team's
    buffers."""
    from libgint_b200.workload import MultiSession
    wl = Workload("periodic_l2_small")
    Ko, _, _, _ = _k(oracle_path, wl)
    Kabs = magnitude_K(oracle_path, wl)
    m = MultiSession(Api(engine_so), wl, 4, team=True)
    for rep in range(2):
        Ke, ms, _ = m.build_K()
        assert_fp64_parity(Ke, Ko, Kabs, wl, f"OpenMP team of 4, shared K (build {rep}, {ms:.1f} ms): ")
    m.close()


@pytest.mark.gpu
def test_bulk_submission_matches_oracle(engine_so, oracle_path):
    """libgint_add_set_quartets (the bulk form of the add_* stream) gives the oracle's K, and the
    same screening decisions, on an l <= 3 system with several contractions per set."""
    from libgint_b200.workload import set_bulk
    wl = Workload("periodic_l3", n_mol=2, box_ang=6.5, n_img_1d=3, n_occ=16, max_prm=4, max_ncontr=3)
    Ko, _, _, co = _k(oracle_path, wl, counters=True)
    set_bulk(True)
    try:
        Kb, _, code_b, cb = _k(engine_so, wl, counters=True)
    finally:
        set_bulk(False)
    assert code_b == 0
    assert_fp64_parity(Kb, Ko, magnitude_K(oracle_path, wl), wl, "bulk submission: ")
    assert_same_decisions(cb, co, wl)


@pytest.mark.gpu
def test_autotuned_graph_replay_matches_oracle(engine_so, oracle_path):
    """The replay as a CUDA graph with the autotuner's per-class kernel choice: the oracle's K, with
    the same screening decisions, for every choice table (the tuned one, all per-warp, all per-lane);
    a second replay relaunches the captured graph."""
    from libgint_b200.capi import load_engine
    lib = load_engine()
    wl = Workload("periodic_l3", n_mol=2, box_ang=6.5, n_img_1d=3, n_occ=16, max_prm=4, max_ncontr=3)
    Ko, _, _, co = _k(oracle_path, wl, counters=True)
    Kabs = magnitude_K(oracle_path, wl)
    s = Session(Api(engine_so), wl)
    h = ctypes.c_void_p(s.h)
    lib.libgint_record(h, 1)
    s.build_K()
    lib.libgint_record(h, 0)
    P = wl.Pflat
    D = ctypes.POINTER(ctypes.c_double)
    lib.libgint_set_P(h, P.ctypes.data_as(D), P.size)
    table = (ctypes.c_int * 512)()
    assert lib.libgint_autotune(h, table) == 0, lib.libgint_error_string(h)
    tuned = np.array(table).reshape(256, 2)
    print(f"autotune: per-warp primitive kernel for {int(tuned[:, 0].sum())} classes, per-warp group kernel "
          f"for {int(tuned[:, 1].sum())}")
    K = np.zeros(P.size)
    for label, tab in [("tuned", tuned), ("per-warp", np.ones((256, 2), dtype=np.int32)),
                       ("per-lane", np.zeros((256, 2), dtype=np.int32))]:
        t = np.ascontiguousarray(tab, dtype=np.int32)
        lib.libgint_set_tuning(h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        lib.libgint_set_counters(h, 1)
        for _ in range(2):
            assert lib.libgint_replay(h) > 0, lib.libgint_error_string(h)
        buf = (ctypes.c_ulonglong * 1024)()
        lib.libgint_get_counters(h, buf)
        lib.libgint_set_counters(h, 0)
        lib.libgint_get_K(h, K.ctypes.data_as(D))
        assert lib.libgint_last_error(h) == 0
        assert_fp64_parity(K, Ko, Kabs, wl, f"graph replay, {label} kernels: ")
        ce = np.frombuffer(buf, dtype=np.uint64).reshape(256, 4) // 2   # two replays counted
        assert_same_decisions(ce, co, wl)
    s.close()
