"""One recorded K build replayed a few times: the case that kernel profiles are taken on.

    python -m libgint_b200.replay_case [--workload periodic_l3] [--setq-stride 4096]
                                       [--fp32-threshold 0] [--replays 3] [--autotune]

streams the sampled set quartets of a named workload through the engine once with recording on
(``libgint_record``, batches merged per class), then replays the recording ``--replays`` times as a CUDA graph and once more
with the kernels serialised (``libgint_replay_profile``), and prints one JSON line: replay times,
the prim/group family times of the serialised replay, shell quartets and launches per replay.
A profiler skips the streamed build's and the warm-up replay's launches with ``-s`` (their counts
are printed as ``launches_before_timed``) and captures launches of the timed replays.
"""
import argparse
import ctypes
import json

import numpy as np

from .capi import engine_path, load_engine
from .workload import CONFIGS, Api, Session, Workload, set_fp32_threshold


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="periodic_l3", choices=sorted(CONFIGS))
    ap.add_argument("--setq-stride", type=int, default=4096)
    ap.add_argument("--fp32-threshold", type=float, default=0.0)
    ap.add_argument("--replays", type=int, default=3)
    ap.add_argument("--max-mem-mb", type=int, default=40000)
    ap.add_argument("--autotune", action="store_true")
    args = ap.parse_args(argv)

    wl = Workload(args.workload, setq_stride=args.setq_stride)
    lib = load_engine()
    stats = (ctypes.c_longlong * 8)()
    set_fp32_threshold(args.fp32_threshold)
    try:
        sess = Session(Api(engine_path()), wl, max_mem_mb=args.max_mem_mb)
        h = ctypes.c_void_p(sess.h)
        lib.libgint_record(h, 2)
        K0, _, _ = sess.build_K()
        lib.libgint_record(h, 0)
    finally:
        set_fp32_threshold(0.0)
    if args.autotune:
        tune = (ctypes.c_int * 512)()
        lib.libgint_autotune(h, tune)
    lib.libgint_get_stats(h, stats)
    before = int(stats[4])
    lib.libgint_replay(h)                      # warm-up
    lib.libgint_get_stats(h, stats)
    per_replay = int(stats[4]) - before
    before_timed = int(stats[4])
    ms = [lib.libgint_replay(h) for _ in range(args.replays)]
    kt = (ctypes.c_double * 2)()
    lib.libgint_replay_profile(h, kt)
    err = lib.libgint_last_error(h)
    K = np.zeros_like(K0)
    lib.libgint_get_K(h, K.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    dev = float(np.abs(K - K0).max() / max(1e-300, np.abs(K0).max()))
    lib.libgint_get_stats(h, stats)
    print(json.dumps({"workload": args.workload, "setq_stride": args.setq_stride,
                      "fp32_threshold": args.fp32_threshold, "autotuned": args.autotune,
                      "shell_quartets": int(stats[0]), "primitive_quartets": int(stats[1]),
                      "replay_ms": ms, "serialised_prim_ms": kt[0], "serialised_group_ms": kt[1],
                      "launches_per_replay": per_replay, "launches_before_timed": before_timed,
                      "replay_vs_stream_rel_dK": dev, "error": int(err)}), flush=True)
    sess.close()
    # the same terms summed in another order: on the ill-conditioned l <= 3 basis that moves K by up
    # to ~1e-10 max|K|; a lost or doubled class segment moves it by far more
    if err or not dev <= 1e-10:
        raise SystemExit(1)


if __name__ == "__main__":
    main()
