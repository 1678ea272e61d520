"""CPU checks of the oracle's two comparison aids: the magnitude mode (the per-element scale of
FP64 rounding error that the GPU parity tests bound the engine's K against) and the screening
decision counters (compared with the engine's for equality)."""
import ctypes

import numpy as np

from conftest import ORACLE_SO
from libgint_b200.workload import Api, Session, Workload, driver


def _oracle(wl, absmode=False, reverse=False, counters=False):
    api = Api(ORACLE_SO)
    s = Session(api, wl)
    V = ctypes.c_void_p
    api.symbol("oracle_set_absmode", None, [V, ctypes.c_int])(s.h, int(absmode))
    if counters:
        api.symbol("libgint_set_counters", None, [V, ctypes.c_int])(s.h, 1)
    d = driver()
    d.gd_set_reverse_prims.argtypes = [ctypes.c_int]
    d.gd_set_reverse_prims(int(reverse))
    try:
        K, _, _ = s.build_K()
    finally:
        d.gd_set_reverse_prims(0)
    cnt = None
    if counters:
        buf = (ctypes.c_ulonglong * 1024)()
        api.symbol("libgint_get_counters", None, [V, ctypes.POINTER(ctypes.c_ulonglong)])(s.h, buf)
        cnt = np.frombuffer(buf, dtype=np.uint64).reshape(256, 4).copy()
    s.close()
    return K, cnt


def test_magnitude_mode_bounds_K_and_the_order_dependence():
    """Kabs >= |K| element by element, and summing every shell's primitives in reverse order moves
    K by far less than 1e-13 Kabs (the element-wise parity bound) on a general-contraction l = 3
    system whose max-norm relative change is orders of magnitude larger."""
    wl = Workload("periodic_l3", n_mol=1, box_ang=5.0, n_img_1d=3, n_occ=8)
    K, _ = _oracle(wl)
    Kr, _ = _oracle(wl, reverse=True)
    Kabs, _ = _oracle(wl, absmode=True)
    assert np.all(Kabs >= np.abs(K) * (1 - 1e-12))
    d = np.abs(K - Kr)
    assert np.all(d <= 1e-13 * Kabs + 1e-300)
    assert Kabs.max() > 1e3 * np.abs(K).max()   # the workload's basis is ill-conditioned
    assert d.max() > 1e-13 * np.abs(K).max()     # so a max-norm bound would not separate orders
    print(f"reverse order: rel max|dK| {d.max() / np.abs(K).max():.2e}, max|dK|/Kabs "
          f"{(d / np.maximum(Kabs, 1e-300)).max():.2e}, Kabs/max|K| {Kabs.max() / np.abs(K).max():.2e}")


def test_decision_counters_are_consistent():
    wl = Workload("small_l2")
    _, cnt = _oracle(wl, counters=True)
    assert int(cnt[:, 3].sum()) == wl.info["n_prims"]
    assert cnt[0, 2] == 0                       # (ss|ss) has no VRR beyond (00|00)
    assert np.all(cnt[:, 2] <= cnt[:, 0] + cnt[:, 1])
    assert int(cnt[:, 0].sum()) > 0
