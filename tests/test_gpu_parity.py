"""Parity of the CUDA engine with the CPU oracle on identical call streams (through the C-ABI).

FP64 path: the tolerance is max|K_engine - K_oracle| <= 1e-11 * max|K_oracle| (the engine sums in a
different order than the oracle and uses FMA; both are FP64). Screening decisions are the same
formula on both sides, so the quartet lists agree exactly.
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
