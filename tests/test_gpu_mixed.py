"""The mixed-precision K build against the all-FP64 oracle.

Shell quartets whose screening bound sqrt((ab|ab)(cd|cd)) max|P| is below the threshold (1e-5 for
the 64-molecule l <= 3 workload) run G_m, VRR, image sum, contraction, HRR and the spherical
transform in FP32 (classes with la+lb+lc+ld <= 3); the decisions, the other classes and the K
update stay FP64. The bounds: max|dK| <= 1e-9 and |dE_x| <= 1e-8 Ha against the FP64 oracle.
"""
import ctypes

import numpy as np
import pytest

from libgint_b200.workload import Api, Session, Workload, set_fp32_threshold

MAX_DK = 1e-9
MAX_DEX = 1e-8
THRESHOLD = 1e-5


def _engine_K(engine_so, wl, thr):
    from libgint_b200.capi import load_engine
    lib = load_engine()
    set_fp32_threshold(thr)
    try:
        s = Session(Api(engine_so), wl)
        K, ms, _ = s.build_K()
        h = ctypes.c_void_p(s.h)
        stats = (ctypes.c_longlong * 8)()
        lib.libgint_get_stats(h, stats)
        assert lib.libgint_last_error(h) == 0, lib.libgint_error_string(h)
        s.close()
    finally:
        set_fp32_threshold(0.0)
    return K, ms, list(stats)


def _oracle_K(oracle_path, wl):
    s = Session(Api(oracle_path), wl)
    K, _, _ = s.build_K()
    s.close()
    return K


@pytest.mark.gpu
@pytest.mark.parametrize("spec,vs_oracle", [
    # a sample of the 64-molecule workload: against the FP64 oracle
    (dict(setq_stride=1 << 16, setq_phase=3), True),
    # one molecule in a 6.2 A cell with 125 images, full 16-primitive sets: every set meets 125
    # images of itself. Its K is so ill-conditioned (sum of term magnitudes ~1e7 max|K|) that two
    # FP64 evaluations in different orders already differ by ~1.7e-9; the FP32 effect is measured
    # against the engine's own FP64 K (same order of operations, only the precision differs)
    (dict(n_mol=1, box_ang=6.2, n_img_1d=5, n_occ=8), False),
])
def test_mixed_precision_within_bounds_of_fp64(engine_so, oracle_path, spec, vs_oracle):
    wl = Workload("periodic_l3", **spec)
    Ko = _oracle_K(oracle_path, wl)
    K64, _, _ = _engine_K(engine_so, wl, 0.0)
    Km, ms, st = _engine_K(engine_so, wl, THRESHOLD)
    frac = st[6] / max(1, st[0])
    Kref = Ko if vs_oracle else K64
    dk = float(np.abs(Km - Kref).max())
    dex = abs(wl.exchange_energy(Km) - wl.exchange_energy(Kref))
    print(f"mixed (threshold {THRESHOLD:g}): {frac:.1%} of {st[0]} shell quartets in FP32 "
          f"({st[7]} of {st[1]} primitive quartets); against the FP64 {'oracle' if vs_oracle else 'engine'}: "
          f"max|dK| {dk:.3e} (max|K| {np.abs(Ko).max():.3e}), |dE_x| {dex:.3e} Ha; FP64 engine vs oracle "
          f"max|dK| {np.abs(K64 - Ko).max():.3e}")
    assert frac > 0.25
    assert dk <= MAX_DK, dk
    assert dex <= MAX_DEX, dex


@pytest.mark.gpu
def test_threshold_zero_is_the_fp64_path(engine_so):
    """With the threshold off, passing bounds changes nothing: the K of the FP64 path (up to the
    order of the K-update atomics)."""
    wl = Workload("periodic_l3", n_mol=2, box_ang=6.5, n_img_1d=3, n_occ=16, max_prm=3, max_ncontr=2)
    s = Session(Api(engine_so), wl)
    K64, _, _ = s.build_K()
    s.close()
    K0, _, st = _engine_K(engine_so, wl, 0.0)
    assert st[6] == 0
    assert np.abs(K0 - K64).max() <= 1e-13 * np.abs(K64).max()
