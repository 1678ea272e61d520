#!/usr/bin/env python
"""Benchmark of the exchange-matrix (K) build on the periodic 64-molecule l <= 3 workload.

Workload: 64 water-like molecules in a 12.4 A periodic cell, 125 image cells, an l <= 3 basis with
16-primitive sets and up to 4 N(0,1) general contractions, P from 256 random occupied orbitals,
truncated Coulomb R_c = 6 A, Schwarz 1e-11, seed 0. P is dense (random orbitals), so the screened
set-quartet list grows as N^2: the whole K build holds ~6.4e9 set quartets, 7.2e9 shell quartets
and 1.05e11 primitive quartets (extrapolated from uniform samples). One step processes a uniform
sample of 1/stride of its set quartets (--setq-stride, every stride-th ket pair of each bra pair
from a hashed offset), so that a step takes about a second; the sample is named in
config.workload.

One step = one K build over the sample's screened quartet list:
  value  device-resident throughput: the quartet list recorded on the GPU (libgint_record) and K
         recomputed from it (libgint_replay: zero K, every kernel), timed with CUDA events on the
         engine's stream; shell quartets per second over all ranks.
  e2e    the same metric through the C-ABI as CP2K drives it: an OpenMP team of --host-threads
         threads with one handle each, every thread streaming its share of the set quartets
         (libgint_set_P from host memory, the add_* calls, libgint_get_K into one shared host K);
         set_P and get_K are collective over the team.
The reference arm (--impl reference) times the CPU restatement of the path (the oracle) on the host
cores over a strided sub-sample of the same workload.

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
    ap.add_argument("--setq-stride", type=int, default=512,
                    help="process a uniform 1/stride sample of the set quartets (1 = all)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--host-threads", type=int, default=min(16, os.cpu_count() or 1),
                    help="OpenMP team size of the end-to-end leg (one handle per thread)")
    ap.add_argument("--device-only", action="store_true",
                    help="record and replay only (no end-to-end, CPU or reference legs)")
    ap.add_argument("--max-mem-mb", type=int, default=7000, help="libgint_set_max_mem of the recording handle")
    ap.add_argument("--host-mem-mb", type=int, default=300,
                    help="libgint_set_max_mem of each end-to-end handle (smaller batches start the GPU sooner)")
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
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
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
    from libgint_b200.workload import Api, MultiSession, Session

    torch.cuda.set_device(local)
    pg = False
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = True

    lib = load_engine()
    t_gen = time.perf_counter()
    wl = make_workload(args)
    t_gen = time.perf_counter() - t_gen
    nq = wl.info["n_setq"]
    setq = wl.setq()
    idx = np.arange(rank, nq, world)            # this rank's share of the set quartets
    total_shells = int(setq[:, 4].sum())
    api = Api(engine_path())
    sess = Session(api, wl, max_mem_mb=args.max_mem_mb)
    h = ctypes.c_void_p(sess.h)
    stats = (ctypes.c_longlong * 8)()

    def check(hh=h):
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

    # 1) first K build through the C-ABI, recording the device-resident quartet list
    lib.libgint_record(h, 1)
    K0, ms_rec, _ = sess.build_K_subset(idx)
    lib.libgint_record(h, 0)
    check()
    lib.libgint_get_stats(h, stats)
    rec_bytes = int(stats[5])
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

    # 3) roofline: one profiled replay (kernels serialised on one stream) with event counters
    lib.libgint_set_counters(h, 1)
    kt = (ctypes.c_double * 2)()
    lib.libgint_replay_profile(h, kt)
    cnt = (ctypes.c_ulonglong * 1024)()
    lib.libgint_get_counters(h, cnt)
    lib.libgint_set_counters(h, 0)
    fl = (ctypes.c_double * 8)()
    flops_prim = 0.0
    for c in range(256):
        ch, bo, vr = cnt[c * 4], cnt[c * 4 + 1], cnt[c * 4 + 2]
        if not (ch or bo or vr):
            continue
        lib.libgint_plan_flops(c >> 6, (c >> 4) & 3, (c >> 2) & 3, c & 3, fl)
        flops_prim += ch * fl[0] + bo * fl[1] + vr * (fl[2] + fl[3])
    flops_group = group_flops(lib, wl) / world
    peak = lib.libgint_fp64_peak_tflops()
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
        sess.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "ms_per_step": ms_per_step,
                              "device_only": True, "k_builds": args.warmup + args.steps + 2,
                              "workload": workload_desc(args, wl), "families": families,
                              "replay_rel_max_dK_vs_stream": replay_dev}), flush=True)
        if pg:
            torch.distributed.destroy_process_group()
        return

    # 4) CPU baseline (rank 0 at N=1): the oracle on a strided sub-sample, plus parity on it
    cpu = None
    parity = None
    if rank == 0 and world == 1:
        from libgint_b200.workload import Api as _Api
        cidx, cshells, csample = oracle_sample(wl, args.cpu_seconds)
        ora = Session(_Api(ORACLE_SO), wl)
        Ko, cms, _ = ora.build_K_subset(cidx)
        ora.close()
        Ke, _, _ = sess.build_K_subset(cidx)
        check()
        # the sub-sample's K against the oracle, also element by element against the oracle's
        # magnitude K (the scale of FP64 rounding error of each element; the basis is ill-conditioned)
        ora = Session(_Api(ORACLE_SO), wl)
        _Api(ORACLE_SO).symbol("oracle_set_absmode", None, [ctypes.c_void_p, ctypes.c_int])(ora.h, 1)
        Kabs, _, _ = ora.build_K_subset(cidx)
        ora.close()
        parity = {"rel_max_dK": float(np.abs(Ke - Ko).max() / max(1e-300, np.abs(Ko).max())),
                  "max_dK_over_Kabs": float((np.abs(Ke - Ko) / np.maximum(Kabs, 1e-300)).max()),
                  "Kabs_over_maxK": float(Kabs.max() / max(1e-300, np.abs(Ko).max())),
                  "sample": "the CPU baseline's sub-sample"}
        cpu = {"value": cshells / (cms / 1e3), "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": csample}
    # the recording session's device batches and pinned queues are released before the
    # end-to-end leg, which sets up its own handles
    sess.close()

    # 5) e2e through the C-ABI with host buffers, driven as CP2K's OpenMP team drives it
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
    e2e_dev = float(np.abs(K - K0).max() / max(1e-300, np.abs(K0).max()))
    e2e_tot = max_over_ranks(float(np.sum(e2e_ms)))
    e2e_ms_step = e2e_tot / args.steps
    e2e_value = total_shells / (e2e_ms_step / 1e3)
    d2h = wl.info["flat_size"] * 8

    ref_cuda = None
    if rank == 0 and world == 1 and not args.no_reference_cuda:
        ref_cuda = reference_cuda_leg()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak" if world > 1 else "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": workload_desc(args, wl),
                       "shell_quartets": total_shells, "primitive_quartets": wl.info["n_prims"],
                       "set_quartets": nq, "contraction_rows": wl.info["n_qrtt"], "n_bf": wl.n_bf,
                       "images": wl.info["Ng"], "generation_s": t_gen,
                       "l2": f"inputs larger than L2: {rec_bytes / 1e9:.2f} GB of quartet records "
                             "are read from HBM per step (L2 is 126 MB)",
                       "step": "one full K build over the sample's screened quartets (FP64)"},
            "ms_per_scf_iter": e2e_ms_step,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms_step,
                    "host_threads": args.host_threads, "caller": "OpenMP team, one handle per thread, shared K",
                    "rel_max_dK_vs_recorded_build": e2e_dev},
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp64", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak if peak > 0 else None, "traffic": None,
                         "peak_source": "FP64 FMA rate measured on this GPU by libgint_fp64_peak_tflops "
                                        "(MEASURED_PEAKS.json has no FP64 figure)",
                         "families": families},
            "clocks": clk,
            "replay_rel_max_dK_vs_stream": replay_dev,
        }
        if cpu:
            line["cpu_baseline"] = cpu
            line["parity_rel_max_dK_vs_oracle"] = parity
        if ref_cuda is not None:
            line["reference_cuda"] = ref_cuda
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
