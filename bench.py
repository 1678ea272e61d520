#!/usr/bin/env python
"""Benchmark of the K build (exchange matrix) on the periodic 32-water workload.

One step = one K build over the whole screened quartet list of the workload:
  value  device-resident throughput: the quartet list recorded on the GPU (libgint_record) and
         K recomputed from it (libgint_replay: zero K, all kernels), timed with CUDA events on
         the engine's stream; shell quartets per second over all ranks.
  e2e    the same metric through the C-ABI as a caller uses it: libgint_set_P from host memory,
         the full add_* call stream, libgint_get_K back to host memory, from --host-threads
         caller threads with one handle each (the reference's one handle per OpenMP thread);
         the threads' K are summed on the host inside the timed region.
The reference arm (--impl reference) times the CPU restatement of the path (the oracle) on
the host cores over a strided sample of the same workload.

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
WORKLOAD = "periodic_l2"
WORKLOAD_DESC = ("32 water-like molecules in a 9.86 A periodic cell, 27 image cells, l<=2 basis "
                 "(O: s6 s1 p3 p1 d1, H: s3 s1 p1), P from 128 occupied orbitals, truncated "
                 "Coulomb R_c = 6 A, Schwarz 1e-11, seed 0, FP64")
ORACLE_SO = os.path.join(ROOT, "oracle", "lib", "liboracle_gint.so")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--host-threads", type=int, default=min(16, os.cpu_count() or 1),
                    help="caller threads (one handle each) of the end-to-end leg")
    ap.add_argument("--device-only", action="store_true",
                    help="record and replay only (no end-to-end or CPU legs); prints the device line "
                         "(for profiling a fixed number of identical K builds)")
    ap.add_argument("--host-mem-mb", type=int, default=300,
                    help="libgint_set_max_mem of each end-to-end handle (smaller batches start the GPU sooner)")
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


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_oracle_sample(wl, seconds, idx_all=None):
    """Time the oracle (all host threads) on a strided sample sized to about `seconds`."""
    from libgint_b200.workload import Api, Session
    ora = Session(Api(ORACLE_SO), wl)
    nq = wl.info["n_setq"]
    setq = wl.setq()
    # calibration on a small strided sample
    stride0 = max(1, nq // 20000)
    idx0 = np.arange(0, nq, stride0)
    _, ms0, _ = ora.build_K_subset(idx0)
    per = ms0 / max(1, len(idx0))
    want = int(min(nq, max(len(idx0), seconds * 1e3 / max(per, 1e-6))))
    stride = max(1, nq // want)
    idx = np.arange(0, nq, stride)
    K, ms, _ = ora.build_K_subset(idx)
    shells = int(setq[idx, 4].sum())
    ora.close()
    return {"value": shells / (ms / 1e3), "ms": ms, "idx": idx, "shells": shells, "K": K,
            "sample": f"every {stride}th set quartet ({len(idx)} set quartets, {shells} shell quartets)"}


def run_reference(args, world, rank):
    """Reference arm: the CPU restatement of the path on the host cores."""
    if rank != 0:
        return
    from libgint_b200.workload import Workload, Api, Session
    wl = Workload(args.workload)
    nq = wl.info["n_setq"]
    setq = wl.setq()
    ora_api = Api(ORACLE_SO)
    s = Session(ora_api, wl)
    stride0 = max(1, nq // 20000)
    idx0 = np.arange(0, nq, stride0)
    _, ms0, _ = s.build_K_subset(idx0)
    per = ms0 / len(idx0)
    per_step = max(2.0, min(args.cpu_seconds, 240.0 / max(1, args.steps + args.warmup)))
    want = int(min(nq, max(len(idx0), per_step * 1e3 / max(per, 1e-6))))
    stride = max(1, nq // want)
    idx = np.arange(0, nq, stride)
    shells = int(setq[idx, 4].sum())
    for _ in range(args.warmup):
        s.build_K_subset(idx)
    times = []
    for _ in range(args.steps):
        _, ms, _ = s.build_K_subset(idx)
        times.append(ms)
    ms = float(np.mean(times))
    value = shells / (ms / 1e3)
    cores = os.cpu_count()
    sample = f"every {stride}th set quartet ({len(idx)} set quartets, {shells} shell quartets)"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {WORKLOAD_DESC}", "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch
    from libgint_b200.capi import engine_path, load_engine
    from libgint_b200.workload import Workload, Api, Session

    torch.cuda.set_device(local)
    pg = False
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = True

    lib = load_engine()
    wl = Workload(args.workload)
    nq = wl.info["n_setq"]
    setq = wl.setq()
    idx = np.arange(rank, nq, world)            # this rank's share of the set quartets
    my_shells = int(setq[idx, 4].sum())
    total_shells = int(setq[:, 4].sum())
    api = Api(engine_path())
    sess = Session(api, wl)
    h = ctypes.c_void_p(sess.h)
    stats = (ctypes.c_longlong * 8)()

    def check():
        e = lib.libgint_last_error(h)
        if e:
            raise RuntimeError(f"engine error {e}: {lib.libgint_error_string(h).decode()}")

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

    # 1) first K build through the C-ABI, recording the device-resident quartet list
    lib.libgint_record(h, 1)
    K0, ms_rec, _ = sess.build_K_subset(idx)
    lib.libgint_record(h, 0)
    lib.libgint_get_stats(h, stats)
    rec_bytes = int(stats[5])
    err = lib.libgint_last_error(h)
    if err:
        raise RuntimeError(f"engine error {err}: {lib.libgint_error_string(h).decode()}")
    K0_local = K0.copy()
    K0 = sum_K(K0)

    # 2) value: device-resident K builds (replay), timed with CUDA events on the engine stream
    for _ in range(args.warmup):
        lib.libgint_replay(h)
    barrier()
    lib.libgint_get_stats(h, stats)
    launches0 = stats[4]
    clocks = ClockSampler(local)
    clocks.start()
    step_ms = []
    for _ in range(args.steps):
        step_ms.append(lib.libgint_replay(h))
    barrier()
    clk = clocks.stop()
    check()
    # the replayed K (same P as the recorded build) must be the streamed build's K; checked after
    # the timed region, so the timed replays are the ones whose result is verified
    Krep = np.zeros_like(K0_local)
    lib.libgint_get_K(h, Krep.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    check()
    replay_dev = max_over_ranks(float(np.abs(Krep - K0_local).max() / max(1e-300, np.abs(K0_local).max())))
    if not replay_dev <= 1e-12:
        raise RuntimeError(f"replayed K differs from the streamed build's K: rel max|dK| = {replay_dev:.3e}")
    lib.libgint_get_stats(h, stats)
    launches = (stats[4] - launches0) // max(1, args.steps)
    tot_ms = max_over_ranks(float(np.sum(step_ms)))
    ms_per_step = tot_ms / args.steps
    value = total_shells / (ms_per_step / 1e3)

    # 3) roofline of the dominant kernel from one profiled replay with event counters
    lib.libgint_set_counters(h, 1)
    kt = (ctypes.c_double * 2)()
    lib.libgint_replay_profile(h, kt)
    cnt = (ctypes.c_ulonglong * 1024)()
    lib.libgint_get_counters(h, cnt)
    lib.libgint_set_counters(h, 0)
    fl = (ctypes.c_double * 8)()
    flops_prim = 0.0
    n_img = 0
    for c in range(256):
        ch, bo, vr, npq = cnt[c * 4], cnt[c * 4 + 1], cnt[c * 4 + 2], cnt[c * 4 + 3]
        if not (ch or bo or vr or npq):
            continue
        lib.libgint_plan_flops(c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3, fl)
        flops_prim += ch * fl[0] + bo * fl[1] + vr * (fl[2] + fl[3])
        n_img += ch + bo
    peak = lib.libgint_fp64_peak_tflops()
    prim_tflops = flops_prim / (kt[0] * 1e-3) / 1e12 if kt[0] > 0 else 0.0
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_k_prim.txt")
    if os.path.exists(tpath):
        for line in open(tpath):
            if line.startswith("bytes_per_launch:"):
                traffic = float(line.split(":")[1])

    if args.device_only:
        # the record build, the warm-up and timed replays and the profiled replay: warmup + steps + 2
        # identical K builds
        sess.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "ms_per_step": ms_per_step,
                              "device_only": True, "k_builds": args.warmup + args.steps + 2,
                              "replay_rel_max_dK_vs_stream": replay_dev,
                              "kernel_ms_per_step": kt[0], "group_kernel_ms_per_step": kt[1]}), flush=True)
        if pg:
            torch.distributed.destroy_process_group()
        return

    # 4) CPU baseline (rank 0 at N=1): the oracle on a strided sample, plus parity on it
    cpu = None
    parity = None
    if rank == 0 and world == 1:
        cb = cpu_oracle_sample(wl, args.cpu_seconds)
        Ke, _, _ = sess.build_K_subset(cb["idx"])
        parity = float(np.abs(Ke - cb["K"]).max() / max(1e-300, np.abs(cb["K"]).max()))
        cpu = {"value": cb["value"], "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": cb["sample"]}
    # the recording session's device batches and pinned queues are released before the
    # end-to-end leg, which sets up its own handles
    sess.close()

    # 5) e2e through the C-ABI with host buffers: set_P, add_* stream, get_K, driven as a caller
    #    with one handle per host thread does (each thread streams a contiguous share of this
    #    rank's set quartets; the threads' K are summed on the host)
    from libgint_b200.workload import MultiSession
    msess = MultiSession(api, wl, args.host_threads, max_mem_mb=args.host_mem_mb)

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
    e2e_ms, e2e_parts = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        K, _, tparts = msess.build_K(idx=idx)
        K = sum_K(K)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        e2e_parts.append(tparts)
    barrier()
    for hh in msess.hs:
        e = lib.libgint_last_error(ctypes.c_void_p(hh))
        if e:
            raise RuntimeError(f"engine error {e}: {lib.libgint_error_string(ctypes.c_void_p(hh)).decode()}")
    h2d = (h2d_total() - h2d0) // max(1, args.steps)
    # the same through libgint_add_set_quartets (one call per chunk of set quartets)
    from libgint_b200.workload import set_bulk
    set_bulk(True)
    try:
        msess.build_K(idx=idx)
        barrier()
        bulk_ms = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            Kb, _, _ = msess.build_K(idx=idx)
            Kb = sum_K(Kb)
            bulk_ms.append((time.perf_counter() - t0) * 1e3)
        barrier()
    finally:
        set_bulk(False)
    bulk_ms_step = max_over_ranks(float(np.sum(bulk_ms))) / args.steps
    bulk_dev = float(np.abs(Kb - K).max() / max(1e-300, np.abs(K).max()))
    msess.close()
    e2e_tot = max_over_ranks(float(np.sum(e2e_ms)))
    e2e_ms_step = e2e_tot / args.steps
    e2e_value = total_shells / (e2e_ms_step / 1e3)
    d2h = wl.info["flat_size"] * 8 * args.host_threads
    ex = wl.exchange_energy(K)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.workload}: {WORKLOAD_DESC}",
                       "shell_quartets": total_shells, "primitive_quartets": wl.info["n_prims"],
                       "set_quartets": nq, "n_bf": wl.n_bf, "images": wl.info["Ng"],
                       "l2": f"inputs larger than L2: {rec_bytes / 1e9:.2f} GB of quartet records "
                             "are read from HBM per step (L2 is 126 MB)",
                       "step": "one full K build (all screened quartets)"},
            "ms_per_scf_iter": e2e_ms_step,
            "E_x": ex,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms_step,
                    "host_threads": args.host_threads,
                    "slowest_thread_ms": float(np.mean([t[3] for t in e2e_parts])),
                    "k_sum_ms": float(np.mean([t[4] for t in e2e_parts]))},
            "e2e_bulk": {"value": total_shells / (bulk_ms_step / 1e3), "unit": UNIT, "ms_per_step": bulk_ms_step,
                         "api": "libgint_add_set_quartets", "max_rel_dK_vs_e2e": bulk_dev},
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp64", "kernel": "k_prim (Fm + VRR + image sum)",
                         "achieved": prim_tflops, "peak": peak, "unit": "TFLOP/s",
                         "frac": prim_tflops / peak if peak > 0 else None, "traffic": traffic,
                         "traffic_unit": "DRAM bytes of the primitive kernels per K build (ncu, scaled; "
                                         "profiles/launches_periodic_l2_small.md)",
                         "peak_source": "FP64 FMA rate measured by libgint_fp64_peak_tflops on this GPU",
                         "kernel_ms_per_step": kt[0], "group_kernel_ms_per_step": kt[1],
                         "flops_per_step": flops_prim, "images_evaluated": int(n_img)},
            "clocks": clk,
            "replay_rel_max_dK_vs_stream": replay_dev,
        }
        if cpu:
            line["cpu_baseline"] = cpu
            line["parity_rel_max_dK_vs_oracle"] = parity
        print(json.dumps(line), flush=True)
    if pg:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
