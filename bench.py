#!/usr/bin/env python
"""Benchmark of the exchange-matrix (K) build on the periodic 64-molecule l <= 3 workload.

Workload: 64 water-like molecules in a 12.4 A periodic cell, 125 image cells, an l <= 3 basis with
16-primitive sets and up to 4 N(0,1) general contractions, P from 256 random occupied orbitals,
truncated Coulomb R_c = 6 A, Schwarz 1e-11, seed 0. P is dense (random orbitals), so the screened
set-quartet list grows as N^2: the whole K build holds ~6.4e9 set quartets, 7.2e9 shell quartets
and 1.05e11 primitive quartets (extrapolated from uniform samples). One step processes a uniform
sample of 1/stride of its set quartets (--setq-stride, every stride-th ket pair of each bra pair
from a hashed offset; 1/256 by default, 1.3 s per step), and the sample is named in
config.workload.

One step = one K build over the sample's screened quartet list:
  value  device-resident throughput of the mixed-precision, batched build: shell quartets whose
         Schwarz bound is below --fp32-threshold (1e-5) run in FP32 (classes with
         la+lb+lc+ld <= 3), the quartet list is recorded on the GPU (libgint_record, few large
         batches) and K is recomputed from it as one CUDA graph (libgint_replay) with the per-class
         kernels chosen by libgint_autotune; CUDA events on the engine's stream; shell quartets per
         second over all ranks. The same all-FP64 build is timed beside it ("fp64"), with the
         mixed build's max|dK| and |dE_x| against it.
  e2e    the mixed build through the C-ABI as CP2K drives it: an OpenMP team of --host-threads
         threads with one handle each, every thread streaming its share of the set quartets
         (libgint_set_P from host memory, the add_* calls with each shell quartet's bound,
         libgint_get_K into one shared host K); set_P and get_K are collective over the team.
The reference arm (--impl reference) times the CPU restatement of the path (the oracle) on the host
cores over a strided sub-sample of the same workload. The reference's own CUDA library is timed on
a small sample of the workload beside ours ("reference_cuda").

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("K-build screened quartets/s & ms/SCF-iter: mixed+batched vs FP64 at "
          "|ΔE_x|≤1e-8 Ha")
UNIT = "shell quartets/s"
ORACLE_SO = os.path.join(ROOT, "oracle", "lib", "liboracle_gint.so")
REF_GINT_SO = os.path.join(ROOT, "oracle", "_ref", "libref_gint.so")
WORKLOADS = {
    "periodic_l3": ("64 water-like molecules in a 12.4 A periodic cell, 125 image cells, l<=3 basis "
                    "(O: s16/4c s1 p8/3c p1 d4/2c d1 d1 f1, H: s6/2c s1 p1; N(0,1) general contractions), "
                    "P from 256 occupied orbitals, truncated Coulomb R_c = 6 A, Schwarz 1e-11, seed 0"),
    "periodic_l2": ("32 water-like molecules in a 9.86 A periodic cell, 27 image cells, l<=2 basis "
                    "(O: s6 s1 p3 p1 d1, H: s3 s1 p1), P from 128 occupied orbitals, truncated "
                    "Coulomb R_c = 6 A, Schwarz 1e-11, seed 0"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="periodic_l3", choices=sorted(WORKLOADS))
    ap.add_argument("--setq-stride", type=int, default=256,
                    help="process a uniform 1/stride sample of the set quartets (1 = all)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--host-threads", type=int, default=0,
                    help="OpenMP team size of the end-to-end leg per rank (one handle per thread; "
                         "0: the host's cores shared among the ranks, at most 16)")
    ap.add_argument("--device-only", action="store_true",
                    help="record and replay only (no end-to-end, CPU or reference legs)")
    ap.add_argument("--max-mem-mb", type=int, default=120000,
                    help="libgint_set_max_mem of the recording handle (large: few batches, one launch per class each)")
    ap.add_argument("--clusters-stride", type=int, default=64,
                    help="set-quartet sample of the batched-systems leg (0 = skip the leg)")
    ap.add_argument("--scf-stride", type=int, default=1 << 14,
                    help="set-quartet sample of the SCF-loop leg (0 = skip the leg)")
    ap.add_argument("--fp32-threshold", type=float, default=1e-5,
                    help="Schwarz bound below which shell quartets run in FP32 (the mixed path)")
    ap.add_argument("--host-mem-mb", type=int, default=4000,
                    help="libgint_set_max_mem of each end-to-end handle (large: few flushes and launches per "
                         "thread; 16 handles hold about 58 GB of device memory)")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip timing the reference CUDA library on a small sample")
    return ap.parse_args()


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.rows)}
        if not self.rows:
            return out
        try:
            sm = [float(r[1]) for r in self.rows]
            out["sm_max_mhz"] = max(float(r[2]) for r in self.rows)
            load = [s for s in sm if s > 0.5 * out["sm_max_mhz"]] or sm
            out["sm_mhz"] = statistics.median(load)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for k, n in enumerate(names):
                if any(r[5 + k].lower().startswith("active") for r in self.rows):
                    out["reasons"].append(n)
        except (ValueError, IndexError):
            pass
        return out


def dist_setup():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def make_workload(args):
    from libgint_b200.workload import Workload
    if args.workload == "periodic_l3":
        return Workload("periodic_l3", setq_stride=args.setq_stride)
    return Workload(args.workload, setq_stride=args.setq_stride)


def workload_desc(args, wl):
    samp = "all set quartets" if args.setq_stride <= 1 else f"a uniform 1/{args.setq_stride} sample of the set quartets"
    return f"{args.workload}: {WORKLOADS[args.workload]}; {samp} ({wl.info['n_setq']} set quartets)"


def oracle_sample(wl, seconds, max_steps=1):
    """A strided sub-sample of the workload's set quartets sized so one oracle K build (all host
    threads) takes about `seconds`; returns (index list, shell quartets in it, description)."""
    from libgint_b200.workload import Api, Session
    nq = wl.info["n_setq"]
    setq = wl.setq()
    ora = Session(Api(ORACLE_SO), wl)
    stride0 = max(1, nq // 4000)
    idx0 = np.arange(0, nq, stride0)
    _, ms0, _ = ora.build_K_subset(idx0)
    ora.close()
    per = ms0 / max(1, len(idx0))
    want = int(min(nq, max(len(idx0), seconds * 1e3 / max(per, 1e-6))))
    stride = max(1, nq // want)
    idx = np.arange(0, nq, stride)
    shells = int(setq[idx, 4].sum())
    return idx, shells, f"every {stride}th set quartet of the step's sample ({len(idx)} set quartets, {shells} shell quartets)"


def run_reference(args, world, rank):
    """Reference arm: the CPU restatement of the path (the oracle port) on the host cores."""
    if rank != 0:
        return
    from libgint_b200.workload import Api, Session
    wl = make_workload(args)
    per_step = max(2.0, min(args.cpu_seconds, 240.0 / max(1, args.steps + args.warmup)))
    idx, shells, sample = oracle_sample(wl, per_step)
    s = Session(Api(ORACLE_SO), wl)
    for _ in range(args.warmup):
        s.build_K_subset(idx)
    times = []
    for _ in range(args.steps):
        _, ms, _ = s.build_K_subset(idx)
        times.append(ms)
    s.close()
    ms = float(np.mean(times))
    value = shells / (ms / 1e3)
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_desc(args, wl), "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def group_flops(lib, wl):
    """Algorithmic FP64 operations of the group stage (contraction, HRR, spherical transform, K
    update) over the workload, counted from the reference recursion with the per-class counts of
    libgint_plan_flops: [4] per primitive and row, [5] per shell and row, [6] and [7] per row."""
    sq = wl.setq()
    sets = wl.sets()
    l, nl = sets[:, 1], sets[:, 2]
    i, j, k, m = sq[:, 0], sq[:, 1], sq[:, 2], sq[:, 3]
    cls = l[i] * 64 + l[j] * 16 + l[k] * 4 + l[m]
    rows = (nl[i] * nl[j] * nl[k] * nl[m]).astype(np.float64)
    fl = np.zeros((256, 8))
    buf = (ctypes.c_double * 8)()
    for c in np.unique(cls):
        lib.libgint_plan_flops(int(c) >> 6, (int(c) >> 4) & 3, (int(c) >> 2) & 3, int(c) & 3, buf)
        fl[c] = list(buf)
    f = fl[cls]
    return float(np.sum(rows * (sq[:, 5] * f[:, 4] + sq[:, 4] * f[:, 5] + f[:, 6] + f[:, 7])))


def scf_leg(args, lib, api):
    """The SCF-loop workload (128 molecules, 15.6 A cell, the 256 nearest image cells, l <= 3 basis),
    on a uniform 1/--scf-stride sample of its set quartets: the quartet list is recorded once with
    P_0 (mixed precision, 7000 MB recording budget, batches merged per class), then 10 K updates follow
    P_k = P_0 + eps_k sym(N(0,1)), eps_k log-spaced from 1e-2 to 1e-6, each one
    K_k = K_{k-1} + K(P_k - P_{k-1}) from the recording with incremental dP screening at the Schwarz
    threshold 1e-11 (libgint_replay_incremental, one CUDA graph). Device time per iteration; the
    last K against a full replay with P_10."""
    import torch
    from libgint_b200.workload import Session, Workload, set_fp32_threshold
    D = ctypes.POINTER(ctypes.c_double)
    t0 = time.perf_counter()
    wl = Workload("periodic_l3_scf", setq_stride=args.scf_stride)
    gen_s = time.perf_counter() - t0
    free0, total = torch.cuda.mem_get_info()
    set_fp32_threshold(args.fp32_threshold)
    try:
        s = Session(api, wl, max_mem_mb=7000)
        h = ctypes.c_void_p(s.h)
        lib.libgint_record(h, 2)
        K, _, _ = s.build_K()
        lib.libgint_record(h, 0)
    finally:
        set_fp32_threshold(0.0)
    lib.libgint_autotune(h, None)
    rng = np.random.default_rng(5)
    P0 = wl.Pflat
    P = P0.copy()
    eps = np.logspace(-2, -6, 10)
    iters = []
    for k, e in enumerate(eps):
        A = rng.standard_normal((wl.n_bf, wl.n_bf))
        Pk = P0 + e * wl.pack(0.5 * (A + A.T))
        dP = Pk - P
        lib.libgint_set_P(h, dP.ctypes.data_as(D), dP.size)
        lib.libgint_set_K(h, K.ctypes.data_as(D), K.size)
        ms = lib.libgint_replay_incremental(h, 1e-11)
        lib.libgint_get_K(h, K.ctypes.data_as(D))
        iters.append(ms)
        if k == 0:
            free1, _ = torch.cuda.mem_get_info()   # recording + replay buffers + P/K, after the first update
        P = Pk
    err = lib.libgint_last_error(h)
    # the last K against a full build (replay without screening) with P_10
    lib.libgint_set_P(h, P.ctypes.data_as(D), P.size)
    full_ms = lib.libgint_replay(h)
    Kf = np.zeros_like(K)
    lib.libgint_get_K(h, Kf.ctypes.data_as(D))
    s.close()
    return {"workload": f"periodic_l3_scf: 128 water-like molecules, 15.6 A cell, the 256 image cells nearest the "
                        f"origin, l<=3 basis as periodic_l3; a uniform 1/{args.scf_stride} sample of the set "
                        f"quartets ({wl.info['n_setq']} set quartets, {wl.info['n_shells']} shell quartets, "
                        f"{wl.info['n_prims']} primitive quartets)",
            "generation_s": gen_s, "error": int(err),
            "ms_per_scf_iter": float(np.mean(iters)), "iteration_ms": [float(x) for x in iters],
            "full_build_ms": full_ms, "eps": [float(x) for x in eps],
            "final_max_dK_vs_full_build": float(np.abs(K - Kf).max()),
            "final_abs_dEx_vs_full_build": abs(wl.exchange_energy(K) - wl.exchange_energy(Kf)),
            "device_mem_mb_held": (free0 - free1) / 2**20,
            "device_mem_cap_mb": 7000}


def clusters_leg(args, lib, api):
    """The batched-systems workload: 96 independent non-periodic water clusters of 2-24 molecules
    (uniform, one seed per system), alternating l <= 2 and l <= 3 bases, all in one handle, on a
    uniform 1/--clusters-stride sample of each system's set quartets: one recording of all systems'
    quartets (one class-sorted list) replayed as one CUDA graph with autotuned kernels, FP64 and
    mixed precision."""
    from libgint_b200.workload import cluster_batch, set_fp32_threshold
    t0 = time.perf_counter()
    b = cluster_batch(96, seed=0, setq_stride=args.clusters_stride)
    gen_s = time.perf_counter() - t0
    out = {"workload": f"96 water clusters of 2-24 molecules (l<=2 and l<=3 bases alternating), one handle; a "
                       f"uniform 1/{args.clusters_stride} sample of each system's set quartets "
                       f"({b.info['n_setq']} set quartets, {b.info['n_shells']} shell quartets, "
                       f"{b.info['n_prims']} primitive quartets, {b.info['n_sets']} sets)",
           "generation_s": gen_s}
    Ks = {}
    for name, thr in (("fp64", 0.0), ("mixed", args.fp32_threshold)):
        set_fp32_threshold(thr)
        try:
            h = b.setup(api, args.max_mem_mb)
            hv = ctypes.c_void_p(h)
            lib.libgint_record(hv, 1)
            b.build_K(api, h)
            lib.libgint_record(hv, 0)
        finally:
            set_fp32_threshold(0.0)
        lib.libgint_autotune(hv, None)
        for _ in range(args.warmup):
            lib.libgint_replay(hv)
        ms = float(np.mean([lib.libgint_replay(hv) for _ in range(args.steps)]))
        K = np.zeros(int(b.offsets[-1]))
        lib.libgint_get_K(hv, K.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        lib.libgint_get_stats(hv, (ctypes.c_longlong * 8)())
        err = lib.libgint_last_error(hv)
        lib.libgint_destroy_handle(hv)
        Ks[name] = b.split(K)
        out[name] = {"ms_per_step": ms, "value": b.info["n_shells"] / (ms / 1e3), "unit": UNIT, "error": int(err)}
    out["mixed_max_dK_vs_fp64"] = max(float(np.abs(a - c).max()) for a, c in zip(Ks["mixed"], Ks["fp64"]))
    out["mixed_max_abs_dEx_vs_fp64"] = float(np.max(np.abs(b.exchange_energies(Ks["mixed"]) -
                                                            b.exchange_energies(Ks["fp64"]))))
    out["mixed_speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    return out


def reference_cuda_leg(timeout_s=600):
    """The reference's own CUDA library (compiled unchanged from its sources for sm_100a) through the
    same C-ABI call stream, on a sample of the workload it can run: its encode_shell asserts
    nla < 4 (src/util.cpp:50), so the sets keep at most 3 contractions. Runs in a child process
    (the reference calls exit() on a CUDA error) and compares its K with the engine's."""
    if not os.path.exists(REF_GINT_SO):
        return {"unavailable": "reference CUDA build absent (make -C oracle ref)"}
    code = r"""
import sys, json, time, numpy as np
sys.path.insert(0, %r)
from libgint_b200.workload import Workload, Api, Session
from libgint_b200.capi import engine_path
wl = Workload("periodic_l3", setq_stride=1 << 15, setq_phase=1, max_ncontr=3)
out = {"sample": "1/32768 sample of the 64-molecule l<=3 workload with at most 3 contractions per set",
       "shell_quartets": int(wl.info["n_shells"]), "primitive_quartets": int(wl.info["n_prims"])}
s = Session(Api(engine_path()), wl); Ke, mse, _ = s.build_K(); s.close()
s = Session(Api(%r), wl, max_mem_mb=7000); Kr, msr, _ = s.build_K(); s.close()
out["reference_ms"] = msr; out["engine_stream_ms"] = mse
out["reference_value"] = wl.info["n_shells"] / (msr / 1e3)
out["rel_max_dK_engine_vs_reference"] = float(np.abs(Ke - Kr).max() / np.abs(Kr).max())
print("REFJSON" + json.dumps(out))
""" % (ROOT, REF_GINT_SO)
    try:
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=timeout_s)
    except subprocess.TimeoutExpired:
        return {"unavailable": f"reference CUDA build did not finish the sample in {timeout_s} s"}
    for line in r.stdout.splitlines():
        if line.startswith("REFJSON"):
            return json.loads(line[7:])
    return {"unavailable": f"reference CUDA run failed (rc={r.returncode}): {(r.stdout + r.stderr)[-300:]}"}


def run_ours(args, world, rank, local):
    import torch
    from libgint_b200.capi import engine_path, load_engine
    from libgint_b200.workload import Api, MultiSession, Session, set_fp32_threshold

    torch.cuda.set_device(local)
    pg = False
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = True

    if args.host_threads <= 0:
        args.host_threads = max(1, min(16, (os.cpu_count() or 1) // world))
    lib = load_engine()
    t_gen = time.perf_counter()
    wl = make_workload(args)
    t_gen = time.perf_counter() - t_gen
    nq = wl.info["n_setq"]
    setq = wl.setq()
    idx = np.arange(rank, nq, world)            # this rank's share of the set quartets
    total_shells = int(setq[:, 4].sum())
    api = Api(engine_path())
    stats = (ctypes.c_longlong * 8)()
    D = ctypes.POINTER(ctypes.c_double)

    def check(hh):
        e = lib.libgint_last_error(hh)
        if e:
            raise RuntimeError(f"engine error {e}: {lib.libgint_error_string(hh).decode()}")

    def barrier():
        torch.cuda.synchronize()
        if pg:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if not pg:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def sum_K(K):
        if not pg:
            return K
        t = torch.from_numpy(K).cuda()
        torch.distributed.all_reduce(t)
        return t.cpu().numpy()

    clocks = ClockSampler(local)

    def device_leg(thr, sampler):
        """Record this rank's share (FP32 threshold thr, 0 = FP64), autotune the per-class kernels,
        then time args.steps graph replays (CUDA events on the engine stream); one more replay with
        the kernels serialised gives the per-family kernel times and the decision counters."""
        set_fp32_threshold(thr)
        try:
            sess = Session(api, wl, max_mem_mb=args.max_mem_mb)
            h = ctypes.c_void_p(sess.h)
            lib.libgint_record(h, 2)
            K_rec, ms_rec, _ = sess.build_K_subset(idx)
            lib.libgint_record(h, 0)
        finally:
            set_fp32_threshold(0.0)
        check(h)
        lib.libgint_get_stats(h, stats)
        st = list(stats)
        tune = (ctypes.c_int * 512)()
        if lib.libgint_autotune(h, tune):
            check(h)
        tune = np.array(tune).reshape(256, 2)
        for _ in range(args.warmup):
            lib.libgint_replay(h)
        barrier()
        lib.libgint_get_stats(h, stats)
        launches0 = stats[4]
        sampler.start()
        step_ms = [lib.libgint_replay(h) for _ in range(args.steps)]
        barrier()
        clk = sampler.stop()
        check(h)
        K = np.zeros_like(K_rec)
        lib.libgint_get_K(h, K.ctypes.data_as(D))
        check(h)
        # the replayed K (same P) must be the streamed build's, checked on the timed replays' result.
        # Both sum the same terms in another order (atomics; the merged replay runs its classes in
        # other launches): on this ill-conditioned basis (terms up to 1e7-1e8 max|K| in the oracle's
        # magnitude mode) that moves K by up to ~1e-10 max|K|, while a lost or doubled class
        # segment moves it by orders of magnitude more
        dev = max_over_ranks(float(np.abs(K - K_rec).max() / max(1e-300, np.abs(K_rec).max())))
        if not dev <= 1e-10:
            raise RuntimeError(f"replayed K differs from the streamed build's K: rel max|dK| = {dev:.3e}")
        lib.libgint_get_stats(h, stats)
        launches = (stats[4] - launches0) // max(1, args.steps)
        ms = max_over_ranks(float(np.sum(step_ms))) / args.steps
        lib.libgint_set_counters(h, 1)
        kt = (ctypes.c_double * 2)()
        lib.libgint_replay_profile(h, kt)
        cnt = (ctypes.c_ulonglong * 1024)()
        lib.libgint_get_counters(h, cnt)
        lib.libgint_set_counters(h, 0)
        sess.close()
        return {"K": sum_K(K), "ms": ms, "launches": int(launches), "kt": (kt[0], kt[1]), "cnt": np.array(cnt),
                "clk": clk, "batches": int(st[3]), "fp32_shells": int(st[6]), "fp32_prims": int(st[7]),
                "shells": int(st[0]), "prims": int(st[1]), "rec_bytes": int(st[5]), "replay_vs_stream": dev,
                "tune": {"per_warp_prim_classes": int(tune[:, 0].sum()), "per_warp_group_classes": int(tune[:, 1].sum())}}

    # 1) the all-FP64 path and 2) the mixed-precision path, both batched (one recording replayed as a
    #    CUDA graph with autotuned per-class kernels)
    fp64 = device_leg(0.0, ClockSampler(local))
    mixed = device_leg(args.fp32_threshold, clocks)
    value = total_shells / (mixed["ms"] / 1e3)
    value_fp64 = total_shells / (fp64["ms"] / 1e3)
    K64, Km = fp64["K"], mixed["K"]
    mixed_dK = float(np.abs(Km - K64).max())
    mixed_dEx = abs(wl.exchange_energy(Km) - wl.exchange_energy(K64)) if world == 1 or rank == 0 else None

    # 3) roofline of the dominant kernel family of the mixed run (kernels serialised, CUDA events)
    fl = (ctypes.c_double * 8)()
    flops_prim = 0.0
    cnt = mixed["cnt"]
    for c in range(256):
        ch, bo, vr = cnt[c * 4], cnt[c * 4 + 1], cnt[c * 4 + 2]
        if not (ch or bo or vr):
            continue
        lib.libgint_plan_flops(c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3, fl)
        flops_prim += ch * fl[0] + bo * fl[1] + vr * (fl[2] + fl[3])
    flops_group = group_flops(lib, wl) / world
    peak = lib.libgint_fp64_peak_tflops()
    kt = mixed["kt"]
    fam = {
        "k_prim (Fm + VRR + image sum)": (flops_prim, kt[0]),
        "k_group (contraction + HRR + spherical + K update)": (flops_group, kt[1]),
    }
    families = {name: {"flops_per_step": f, "kernel_ms_per_step": t,
                       "achieved_tflops": f / (t * 1e-3) / 1e12 if t > 0 else 0.0}
                for name, (f, t) in fam.items()}
    dom = max(families, key=lambda n: families[n]["kernel_ms_per_step"])
    achieved = families[dom]["achieved_tflops"]

    if args.device_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "ms_per_step": mixed["ms"],
                              "fp64": {"value": value_fp64, "ms_per_step": fp64["ms"]}, "device_only": True,
                              "workload": workload_desc(args, wl), "families": families,
                              "mixed_max_dK_vs_fp64": mixed_dK}), flush=True)
        if pg:
            torch.distributed.destroy_process_group()
        return

    # 4) CPU baseline (rank 0 at N=1): the oracle on a strided sub-sample, and parity there (FP64
    #    engine element-wise against the oracle's magnitude K; mixed engine against the oracle)
    cpu = None
    parity = None
    if rank == 0 and world == 1:
        cidx, cshells, csample = oracle_sample(wl, args.cpu_seconds)
        ora = Session(Api(ORACLE_SO), wl)
        Ko, cms, _ = ora.build_K_subset(cidx)
        ora.close()
        ora = Session(Api(ORACLE_SO), wl)
        Api(ORACLE_SO).symbol("oracle_set_absmode", None, [ctypes.c_void_p, ctypes.c_int])(ora.h, 1)
        Kabs, _, _ = ora.build_K_subset(cidx)
        ora.close()
        Ks = {}
        for name, thr in (("fp64", 0.0), ("mixed", args.fp32_threshold)):
            set_fp32_threshold(thr)
            try:
                sess = Session(api, wl)
                Ks[name], _, _ = sess.build_K_subset(cidx)
                check(ctypes.c_void_p(sess.h))
                sess.close()
            finally:
                set_fp32_threshold(0.0)
        parity = {"sample": "the CPU baseline's sub-sample",
                  "fp64_rel_max_dK": float(np.abs(Ks["fp64"] - Ko).max() / max(1e-300, np.abs(Ko).max())),
                  "fp64_max_dK_over_Kabs": float((np.abs(Ks["fp64"] - Ko) / np.maximum(Kabs, 1e-300)).max()),
                  "Kabs_over_maxK": float(Kabs.max() / max(1e-300, np.abs(Ko).max())),
                  "mixed_max_dK": float(np.abs(Ks["mixed"] - Ko).max()),
                  "mixed_abs_dEx": abs(wl.exchange_energy(Ks["mixed"]) - wl.exchange_energy(Ko))}
        cpu = {"value": cshells / (cms / 1e3), "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": csample}

    # 5) e2e through the C-ABI with host buffers, driven as CP2K's OpenMP team drives it, on the
    #    mixed path (each thread passes its shell quartets' Schwarz bounds)
    set_fp32_threshold(args.fp32_threshold)
    try:
        msess = MultiSession(api, wl, args.host_threads, max_mem_mb=args.host_mem_mb, team=True)

        def h2d_total():
            tot = 0
            for hh in msess.hs:
                lib.libgint_get_stats(ctypes.c_void_p(hh), stats)
                tot += int(stats[5])
            return tot

        for _ in range(max(1, args.warmup - 1)):
            msess.build_K(idx=idx)
        barrier()
        h2d0 = h2d_total()
        e2e_ms = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            K, _, _ = msess.build_K(idx=idx)
            K = sum_K(K)
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
        barrier()
        for hh in msess.hs:
            check(ctypes.c_void_p(hh))
        h2d = (h2d_total() - h2d0) // max(1, args.steps)
        msess.close()
    finally:
        set_fp32_threshold(0.0)
    e2e_dev = float(np.abs(K - Km).max())
    e2e_ms_step = max_over_ranks(float(np.sum(e2e_ms))) / args.steps
    e2e_value = total_shells / (e2e_ms_step / 1e3)
    d2h = wl.info["flat_size"] * 8

    ref_cuda = None
    if rank == 0 and world == 1 and not args.no_reference_cuda:
        ref_cuda = reference_cuda_leg()

    scf = None
    if rank == 0 and world == 1 and args.scf_stride > 0:
        scf = scf_leg(args, lib, api)
    clusters = None
    if rank == 0 and world == 1 and args.clusters_stride > 0:
        clusters = clusters_leg(args, lib, api)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mixed["ms"], "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32/f64",
            "data": "synthetic",
            "config": {"workload": workload_desc(args, wl),
                       "shell_quartets": total_shells, "primitive_quartets": wl.info["n_prims"],
                       "set_quartets": nq, "contraction_rows": wl.info["n_qrtt"], "n_bf": wl.n_bf,
                       "images": wl.info["Ng"], "generation_s": t_gen,
                       "fp32_threshold": args.fp32_threshold,
                       "l2": f"inputs larger than L2: {mixed['rec_bytes'] / 1e9:.2f} GB of quartet records "
                             "are read from HBM per step (L2 is 126 MB)",
                       "step": "one full K build over the sample's screened quartets: mixed precision, one "
                               "recording replayed as a CUDA graph with autotuned per-class kernels"},
            "mixed": {"value": value, "ms_per_step": mixed["ms"], "gpu_launches": mixed["launches"],
                      "batches": mixed["batches"], "fp32_shell_fraction": mixed["fp32_shells"] / max(1, mixed["shells"]),
                      "fp32_primitive_fraction": mixed["fp32_prims"] / max(1, mixed["prims"]),
                      "max_dK_vs_fp64_engine": mixed_dK, "abs_dEx_vs_fp64_engine": mixed_dEx,
                      "autotune": mixed["tune"]},
            "fp64": {"value": value_fp64, "ms_per_step": fp64["ms"], "gpu_launches": fp64["launches"],
                     "batches": fp64["batches"], "autotune": fp64["tune"], "clocks": fp64["clk"]},
            "mixed_speedup_vs_fp64": fp64["ms"] / mixed["ms"],
            "ms_per_scf_iter": e2e_ms_step,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms_step,
                    "host_threads": args.host_threads, "handle_max_mem_mb": args.host_mem_mb,
                    "caller": "OpenMP team, one handle per thread, shared K, mixed precision",
                    "max_dK_vs_device_mixed_build": e2e_dev},
            "gpu_launches": mixed["launches"],
            "roofline": {"bound": "fp64", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak if peak > 0 else None, "traffic": None,
                         "peak_source": "FP64 FMA rate measured on this GPU by libgint_fp64_peak_tflops "
                                        "(MEASURED_PEAKS.json has no FP64 figure)",
                         "families": families},
            "clocks": mixed["clk"],
            "replay_rel_max_dK_vs_stream": max(fp64["replay_vs_stream"], mixed["replay_vs_stream"]),
        }
        if cpu:
            line["cpu_baseline"] = cpu
            line["parity_vs_oracle"] = parity
        if ref_cuda is not None:
            line["reference_cuda"] = ref_cuda
        if scf is not None:
            line["scf_loop"] = scf
        if clusters is not None:
            line["batched_systems"] = clusters
        print(json.dumps(line), flush=True)
    if pg:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
