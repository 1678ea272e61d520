"""The allocation-free K rebuild (libgint_replay_noalloc) against the ordinary replay and the oracle.

Some callers cannot allocate device memory while K is built: their framework owns every device
byte through its own pool, or a cudaMalloc/cudaFree would synchronise a pipeline they must not
stall. For them libgint_replay_noalloc writes into device buffers they own and keeps its
intermediates in a fixed scratch array inside the library. These tests own P and K on the device
(allocated here, by the caller), call the entry point twice in a row through the C-ABI, and check
both results against libgint_replay + libgint_get_K and against the CPU oracle at the parity
tolerance (1e-12 of max|K|).
"""
import ctypes

import numpy as np
import pytest

from libgint_b200.workload import Api, Session, Workload

TOL = 1e-12
D = ctypes.POINTER(ctypes.c_double)


def _oracle_K(oracle_path, wl):
    s = Session(Api(oracle_path), wl)
    K, _, _ = s.build_K()
    s.close()
    return K


def _noalloc_twice(lib, h, P, K_ref, K_oracle, stream_first_call_after_record=False):
    import torch
    P_dev = torch.from_numpy(P).cuda()
    K_dev = torch.full((P.size,), 7.0, dtype=torch.float64, device="cuda")   # stale contents are cleared
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    scale = np.abs(K_oracle).max()
    for call in range(2):
        rc = lib.libgint_replay_noalloc(h, ctypes.c_void_p(P_dev.data_ptr()), ctypes.c_void_p(K_dev.data_ptr()),
                                        P.size, ctypes.c_void_p(stream))
        assert rc == 0, lib.libgint_error_string(h)
        torch.cuda.synchronize()
        K = K_dev.cpu().numpy()
        if K_ref is not None:
            assert np.abs(K - K_ref).max() / scale <= TOL, (call, "vs replay")
        rel = np.abs(K - K_oracle).max() / scale
        assert rel <= TOL, (call, rel)


@pytest.mark.gpu
def test_replay_noalloc_matches_replay_and_oracle(engine_so, oracle_path):
    import torch
    from libgint_b200.capi import load_engine
    torch.cuda.set_device(0)
    lib = load_engine()
    wl = Workload("small_l2")
    s = Session(Api(engine_so), wl)
    h = ctypes.c_void_p(s.h)
    lib.libgint_set_max_mem(h, 150)          # small recorded batches: each fits the fixed scratch
    lib.libgint_record(h, 1)
    s.build_K()
    lib.libgint_record(h, 0)
    P = wl.Pflat
    lib.libgint_set_P(h, P.ctypes.data_as(D), P.size)
    assert lib.libgint_replay(h) > 0
    K_ref = np.zeros(P.size)
    lib.libgint_get_K(h, K_ref.ctypes.data_as(D))
    assert lib.libgint_last_error(h) == 0, lib.libgint_error_string(h)
    _noalloc_twice(lib, h, P, K_ref, _oracle_K(oracle_path, wl))
    # the ordinary path still sees no device error afterwards
    lib.libgint_get_K(h, K_ref.ctypes.data_as(D))
    assert lib.libgint_last_error(h) == 0
    s.close()


@pytest.mark.gpu
def test_replay_noalloc_right_after_recording_multi_batch_periodic(engine_so, oracle_path):
    """The first call comes straight after libgint_record(h, 0), on the caller's own stream, with
    nothing in between that waits for the recording's uploads: the call itself orders the caller's
    stream after them. A periodic system recorded in many small batches."""
    import torch
    from libgint_b200.capi import load_engine
    torch.cuda.set_device(0)
    lib = load_engine()
    wl = Workload("periodic_l2_small")
    s = Session(Api(engine_so), wl, max_mem_mb=150)
    h = ctypes.c_void_p(s.h)
    lib.libgint_record(h, 1)
    s.build_K()
    lib.libgint_record(h, 0)
    stats = (ctypes.c_longlong * 8)()
    lib.libgint_get_stats(h, stats)
    assert stats[3] >= 4, f"expected a recording of several batches, got {stats[3]}"
    _noalloc_twice(lib, h, wl.Pflat, None, _oracle_K(oracle_path, wl))
    assert lib.libgint_last_error(h) == 0
    # K_size must be the recorded build's P_size (the K updates index up to it)
    import torch
    P_dev = torch.from_numpy(wl.Pflat).cuda()
    rc = lib.libgint_replay_noalloc(h, ctypes.c_void_p(P_dev.data_ptr()), ctypes.c_void_p(P_dev.data_ptr()),
                                    wl.Pflat.size - 1, None)
    assert rc == 2 and b"K_size" in lib.libgint_error_string(h)
    s.close()


@pytest.mark.gpu
def test_replay_noalloc_rejects_a_segment_beyond_the_scratch(engine_so):
    """A recording made with a large work budget holds class segments larger than the fixed
    scratch: the call fails with error 5 before launching anything, and the caller's K is left
    as it was."""
    import torch
    from libgint_b200.capi import load_engine
    torch.cuda.set_device(0)
    lib = load_engine()
    wl = Workload("periodic_l2_small")
    s = Session(Api(engine_so), wl, max_mem_mb=7000)
    h = ctypes.c_void_p(s.h)
    lib.libgint_record(h, 1)
    s.build_K()
    lib.libgint_record(h, 0)
    assert lib.libgint_last_error(h) == 0
    P = wl.Pflat
    P_dev = torch.from_numpy(P).cuda()
    K_dev = torch.full((P.size,), 3.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.libgint_replay_noalloc(h, ctypes.c_void_p(P_dev.data_ptr()), ctypes.c_void_p(K_dev.data_ptr()),
                                    P.size, None)
    torch.cuda.synchronize()
    assert rc == 5, (rc, lib.libgint_error_string(h))
    assert b"maximum" in lib.libgint_error_string(h)
    assert bool((K_dev == 3.0).all())
    s.close()


@pytest.mark.gpu
def test_replay_noalloc_rejects_missing_recording(engine_so):
    from libgint_b200.capi import LibGint
    g = LibGint()
    g.init()
    rc = g.lib.libgint_replay_noalloc(g.h, None, None, 0, None)
    code, msg = g.last_error()
    assert rc != 0 and code != 0 and "libgint_record" in msg
    g.close()
