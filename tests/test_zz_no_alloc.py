"""The allocation-free K rebuild (libgint_replay_noalloc) against the ordinary replay.

Some callers cannot allocate device memory while K is built: their framework owns every device
byte through its own pool, or a cudaMalloc/cudaFree would synchronise a pipeline they must not
stall. For them libgint_replay_noalloc writes into device buffers they own and keeps its
intermediates in a fixed scratch array inside the library. This test owns P and K on the device
(allocated here, by the caller), calls the entry point twice in a row through the C-ABI, and
checks both results against libgint_replay + libgint_get_K at the parity tolerance (1e-11).
"""
import ctypes

import numpy as np
import pytest

from libgint_b200.workload import Api, Session, Workload

TOL = 1e-11


@pytest.mark.gpu
def test_replay_noalloc_matches_replay(engine_so):
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
    D = ctypes.POINTER(ctypes.c_double)
    lib.libgint_set_P(h, P.ctypes.data_as(D), P.size)
    assert lib.libgint_replay(h) > 0
    K_ref = np.zeros(P.size)
    lib.libgint_get_K(h, K_ref.ctypes.data_as(D))
    assert lib.libgint_last_error(h) == 0, lib.libgint_error_string(h)

    P_dev = torch.from_numpy(P).cuda()
    K_dev = torch.full((P.size,), 7.0, dtype=torch.float64, device="cuda")   # stale contents are cleared
    stream = torch.cuda.current_stream().cuda_stream
    scale = np.abs(K_ref).max()
    for call in range(2):
        rc = lib.libgint_replay_noalloc(h, ctypes.c_void_p(P_dev.data_ptr()), ctypes.c_void_p(K_dev.data_ptr()),
                                        P.size, ctypes.c_void_p(stream))
        assert rc == 0, lib.libgint_error_string(h)
        torch.cuda.synchronize()
        K = K_dev.cpu().numpy()
        rel = np.abs(K - K_ref).max() / scale
        assert rel <= TOL, (call, rel)
    # the ordinary path still sees no device error afterwards
    lib.libgint_get_K(h, K_ref.ctypes.data_as(D))
    assert lib.libgint_last_error(h) == 0
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
