#!/usr/bin/env python
"""Benchmark: exact kNN queries/s (k=32, self-query) over a 16.7M-point clustered
periodic catalogue on one B200, plus build Mpt/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one kNN pass of every point of the catalogue (2^24 queries, k=32,
sorted) through the library with inputs resident in HBM.  Timing: CUDA events on
the launching stream, barrier + synchronize around the timed region, max over
ranks.  Inputs (tree ~0.6 GB, outputs 8.6 GB per step) are far larger than L2.
Under torchrun each rank builds and searches its own catalogue (seed + rank) with
no collective on the data path (weak scaling); rank 0 prints one JSON line.

--impl reference times the reference algorithm's CPU implementation (the C++
restatement in oracle/, OpenMP over queries like src/cosmokdtree2py.f90:132-141) on
the host cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import csv
import ctypes
import io
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (n_points, k, periodic, leaf, seed)
    "clustered_periodic_2p24_k32": (1 << 24, 32, True, 16, 1),
    "uniform_2p20_k16": (1 << 20, 16, False, 16, 0),
    "clustered_periodic_2p22_k32": (1 << 22, 32, True, 16, 1),
}
DEFAULT_WORKLOAD = "clustered_periodic_2p24_k32"


def make_points(name, seed_offset=0):
    from cosmokdtree_b200 import synth
    n, k, periodic, leaf, seed = WORKLOADS[name]
    if periodic:
        return synth.clustered_periodic(n, seed=seed + seed_offset)
    return synth.uniform(n, 3, seed=seed + seed_offset)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for r in csv.reader(io.StringIO(open(self.path).read())):
                if len(r) >= 9:
                    rows.append([x.strip() for x in r])
        except Exception:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def cpu_knn_rate(tree, P, k, target_s, seed=0):
    """Oracle kNN over a growing random sample until one pass takes >= target_s."""
    rng = np.random.default_rng(seed)
    m = 4096
    while True:
        idx = rng.integers(0, P.shape[0], m)
        Q = np.ascontiguousarray(P[idx])
        t0 = time.perf_counter()
        tree.knn(Q, k)
        dt = time.perf_counter() - t0
        if dt >= target_s or m >= P.shape[0]:
            return m / dt, m, dt
        m = min(P.shape[0], int(m * max(2.0, 1.2 * target_s / max(dt, 1e-3))))


def run_reference(args):
    """CPU arm: the reference algorithm (C++ restatement) on all host cores."""
    import oracle
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    name = args.workload
    n, k, periodic, leaf, seed = WORKLOADS[name]
    P = make_points(name)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    tree = oracle.OracleTree(P, leaf, 1.0 if periodic else None, threads=threads)
    build_s = time.perf_counter() - t0
    # size one step to a few seconds
    rate0, m, dt = cpu_knn_rate(tree, P, k, target_s=2.0)
    m_step = int(min(P.shape[0], max(4096, rate0 * 5.0)))
    rng = np.random.default_rng(123)
    samples = []
    for s in range(args.warmup + args.steps):
        Q = np.ascontiguousarray(P[rng.integers(0, P.shape[0], m_step)])
        t0 = time.perf_counter()
        tree.knn(Q, k)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            samples.append(dt)
    value = m_step * len(samples) / sum(samples)
    out = {
        "impl": "reference", "metric": "knn_queries_per_s", "value": value, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(samples) / len(samples), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(name),
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "port",
                         "sample": f"{m_step} random self-queries of the {n}-point catalogue "
                                   "per step, reference traversal (hyperplane DFS, periodic)"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "build": {"cpu_s": build_s, "cpu_mpts_per_s": n / build_s / 1e6},
    }
    print(json.dumps(out))
    return 0


def workload_config(name):
    n, k, periodic, leaf, seed = WORKLOADS[name]
    return {"workload": name, "n_points": n, "n_queries": n, "k": k, "sorted": True,
            "periodic": periodic, "leaf": leaf, "seed": seed, "dims": 3,
            "l2": "inputs larger than L2 (tree ~0.6 GB, outputs 8.6 GB per step)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--variant", type=int, default=0, help="kNN kernel: 0 auto, 1 fp64, 2 screened")
    ap.add_argument("--stats", action="store_true", help="report traversal statistics (profile mode)")
    ap.add_argument("--tune", default="", help="comma list key=value of ckd_set_tuning knobs")
    ap.add_argument("--profile", action="store_true",
                    help="one build and the kNN steps only (for ncu captures)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device(f"cuda:{local}"))

    def barrier():
        if world > 1:
            dist.barrier()

    def allmax(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    from cosmokdtree_b200 import _lib, kdtree
    L = _lib.load()
    _lib.check(L.ckd_set_knn_variant(args.variant))
    for kv in filter(None, args.tune.split(",")):
        key, val = kv.split("=")
        _lib.check(L.ckd_set_tuning(int(key), int(val)))
    name = args.workload
    n, k, periodic, leaf, seed = WORKLOADS[name]
    P = make_points(name, seed_offset=rank)
    box = [1.0, 1.0, 1.0] if periodic else None
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    # ---- build (device-resident input), Mpt/s
    Pd = torch.from_numpy(P).cuda()
    build_ms = []
    n_builds = 1 if args.profile else 3
    for it in range(n_builds):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        tree = kdtree.build_kdtree(Pd, leaf=leaf, boxsize=box)
        e1.record(stream)
        torch.cuda.synchronize()
        if it > 0 or n_builds == 1:
            build_ms.append(e0.elapsed_time(e1))
        if it < n_builds - 1:
            tree.close()
    build_ms_v = allmax(float(np.mean(build_ms)))

    # ---- kNN, inputs resident in HBM
    nq = P.shape[0]
    Q = Pd
    dist_t = torch.empty((nq, k), dtype=torch.float64, device="cuda")
    idx_t = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    order = torch.empty(nq, dtype=torch.int32, device="cuda")

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        _lib.check(L.ckd_knn(tree.handle, ctypes.c_void_p(Q.data_ptr()), nq, k, 1,
                             ctypes.c_void_p(dist_t.data_ptr()),
                             ctypes.c_void_p(idx_t.data_ptr()), sp))
        if ev is not None:
            ev[1].record(stream)

    def kernel_ms(reps=3):
        """Average device time of the main search kernel alone (CUDA events
        recorded by the library around that launch)."""
        _lib.check(L.ckd_set_kernel_timing(1))
        vals = []
        for _ in range(reps):
            step()
            v = ctypes.c_float()
            _lib.check(L.ckd_kernel_ms(ctypes.byref(v)))
            vals.append(v.value)
        _lib.check(L.ckd_set_kernel_timing(0))
        return float(np.mean(vals))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    if args.stats:
        _lib.check(L.ckd_knn_stats(1, None))
    launches0 = L.ckd_launch_count()
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for s in range(args.steps):
            step(evs[s])
        t_end.record(stream)
        torch.cuda.synchronize()
        barrier()
    launches = L.ckd_launch_count() - launches0
    total_ms = allmax(t_start.elapsed_time(t_end))
    step_ms = [e[0].elapsed_time(e[1]) for e in evs]
    knn_kernel_ms = kernel_ms()
    ms_per_step = total_ms / args.steps
    value = world * nq * args.steps / (total_ms / 1e3)
    clocks = clk.summary()
    stats = None
    if args.stats:
        st = (ctypes.c_int64 * 8)()
        _lib.check(L.ckd_knn_stats(0, st))
        names = ["pops", "needed_pops", "leaf_visits", "points_screened", "insert_rounds",
                 "fp64_evals", "inserts", "lanes_on_leaf_visits"]
        warps = args.steps * ((nq + 31) // 32)
        stats = {nm: st[i] / warps for i, nm in enumerate(names)}
        stats["per_query_fp64_evals"] = st[5] / (args.steps * nq)
        stats["per_query_inserts"] = st[6] / (args.steps * nq)
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "workload": name, "ms_per_step": ms_per_step,
                              "variant": args.variant, "tune": args.tune, "stats_per_warp": stats,
                              "knn_kernel_ms": knn_kernel_ms, "step_ms": float(np.mean(step_ms)),
                              "build_ms": build_ms_v, "depth": tree.depth, "n_nodes": tree.n_nodes}))
        tree.close()
        return 0

    # ---- end to end through the public API with host buffers
    e2e_ms = []
    for it in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        hd, hi = kdtree.knn_search(tree, P, k, sorted=True)
        e1.record(stream)
        torch.cuda.synchronize()
        if it > 0:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_ms_v = allmax(float(np.mean(e2e_ms)))

    out = None
    if rank == 0:
        import oracle
        peak, peak_kind = measured_peaks()
        threads = os.cpu_count() or 1
        # reference-algorithm tree on the host: algorithmic bytes, parity sample, CPU baseline
        t0 = time.perf_counter()
        otree = oracle.OracleTree(P, leaf, 1.0 if periodic else None, threads=threads)
        cpu_build_s = time.perf_counter() - t0
        rng = np.random.default_rng(7)
        samp = rng.integers(0, nq, 20000)
        od, oi = otree.knn(P[samp], k)
        parity = bool(np.array_equal(oi, hi[samp]) and np.array_equal(od, hd[samp]))
        ab = otree.knn_algbytes(P[samp], k, od[:, -1] ** 2)
        bytes_per_q = ab["bytes"] / len(samp)
        knn_avg_ms = knn_kernel_ms
        achieved = bytes_per_q * nq / (knn_avg_ms / 1e3) / 1e9
        cpu = None
        if world == 1 and not args.no_cpu:
            rate, m, dt = cpu_knn_rate(otree, P, k, target_s=args.cpu_seconds)
            cpu = {"value": rate, "unit": "queries/s", "cores": threads, "kind": "port",
                   "sample": f"{m} random self-queries of the catalogue in {dt:.1f} s, "
                             "reference traversal, FP64"}
        out = {
            "metric": "knn_queries_per_s", "value": value, "unit": "queries/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(name),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "k_knn_bucket", "kernel_ms": knn_avg_ms,
                         "alg_bytes_per_query": bytes_per_q, "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": world * nq / (e2e_ms_v / 1e3), "unit": "queries/s",
                    "h2d_bytes_per_step": nq * 3 * 8, "d2h_bytes_per_step": nq * k * 16,
                    "ms_per_step": e2e_ms_v},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "build": {"ms": build_ms_v, "mpts_per_s": n / (build_ms_v / 1e3) / 1e6,
                      "cpu_s": cpu_build_s, "cpu_mpts_per_s": n / cpu_build_s / 1e6,
                      "n_nodes": tree.n_nodes, "depth": tree.depth},
            "breakdown_ms": {"step": float(np.mean(step_ms)), "knn_kernel": knn_avg_ms},
            "parity_sample": {"rows": int(len(samp)), "bit_exact": parity},
        }
        print(json.dumps(out))
    tree.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
