#!/usr/bin/env python
"""Benchmark: exact kNN queries/s (k=32, self-query) over a 16.7M-point clustered
periodic catalogue on one B200 -- the default search (headline ``value``) and the
learned-bound search (``learned``, with its ratio), both exact and checked equal --
plus build Mpt/s and ball search (r = half the mean spacing, CSR).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one kNN pass of every point of the catalogue (2^24 queries, k=32,
sorted) through the library with inputs resident in HBM.  The network is trained
beforehand (untimed, like the tree build) on 10^6 exact k-th distances of a
separate catalogue drawn with another seed.  Timing: CUDA events on
the launching stream, barrier + synchronize around the timed region, max over
ranks.  Inputs (tree ~0.6 GB, outputs 8.6 GB per step) are far larger than L2.
With --gpus N > 1 (one process per GPU: launched by torchrun, or relaunched under
torchrun by this script when started plainly) every rank builds a replica of the
same tree in its own HBM and searches a contiguous shard of the 2^24 queries
(distributed.knn_sharded), with no collective on the data path: the job is fixed,
so scaling is strong; rank 0 prints one JSON line.

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
# DRAM bytes (read + write) of one launch of the default kNN kernel per query, from
# an ncu capture of the 2^22-point form of the default workload (4.02 GB per
# 2^22-query launch, profiles/knn_lane2_clustered_2p22_k32.md); the traffic of a
# launch grows with its queries (each reads its neighbourhood and writes its row)
KNN_DRAM_BYTES_PER_QUERY = 4.02e9 / (1 << 22)
KNN_TRAFFIC_NOTE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the 2^22-point "
                    "case, scaled by the query count")
# learned-bound configurations with their own query sets (several k, other dims)
MULTI_WORKLOADS = {
    # 2^26 clustered periodic, 10^7 queries (half particles, half uniform), k in {8,32,64}
    "learned_mixed_2p26": dict(n=1 << 26, d=3, periodic=True, leaf=16, ks=(8, 32, 64),
                               nq=10_000_000, query="mixed", dtype="f64", seed=1,
                               train_seed=3, query_seed=4),
    "learned_mixed_2p22": dict(n=1 << 22, d=3, periodic=True, leaf=16, ks=(8, 32, 64),
                               nq=1_000_000, query="mixed", dtype="f64", seed=1,
                               train_seed=3, query_seed=4),
    # 2^27 6-D phase space, float32 input, leaf 32, 2x10^7 queries, k = 64
    "phase6d_2p27_k64": dict(n=1 << 27, d=6, periodic=False, leaf=32, ks=(64,),
                             nq=20_000_000, query="particles", dtype="f32", seed=5,
                             train_seed=6, query_seed=7),
    "phase6d_2p22_k64": dict(n=1 << 22, d=6, periodic=False, leaf=32, ks=(64,),
                             nq=1_000_000, query="particles", dtype="f32", seed=5,
                             train_seed=6, query_seed=7),
}
# forests: name -> (n_trees, k, boxes per tree, box side, seed)
FOREST_WORKLOADS = {
    "forest_2000_nfw_k8": (2000, 8, 64, 0.05, 2),
    "forest_200_nfw_k8": (200, 8, 64, 0.05, 2),
}


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
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(name, args.gpus),
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "port",
                         "sample": f"{m_step} random self-queries of the {n}-point catalogue "
                                   "per step, reference traversal (hyperplane DFS, periodic)"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "build": {"cpu_s": build_s, "cpu_mpts_per_s": n / build_s / 1e6},
    }
    print(json.dumps(out))
    return 0


def run_forest(args):
    """Batched uneven trees: every tree an NFW-like cluster in its own periodic unit
    box, sizes log-uniform in [10^3, 10^6]; all trees built in one pass, 10% of each
    tree's points queried (kNN k=8) by one captured CUDA graph per step, 64 boxes
    of side 0.05 per tree."""
    import torch
    from cosmokdtree_b200 import _lib, build_forest, synth
    n_trees, k, nbox, side, seed = FOREST_WORKLOADS[args.workload]
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    L = _lib.load()
    stream = torch.cuda.current_stream()
    Pd, off = synth.forest_catalogue(n_trees, seed=seed)
    n = int(off[-1])
    sizes = np.diff(off)
    build_ms = []
    for it in range(2):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        f = build_forest(Pd, off, leaf=16, boxsize=1.0)
        e1.record(stream)
        torch.cuda.synchronize()
        build_ms.append(e0.elapsed_time(e1))
        if it == 0:
            f.close()
    rng = np.random.default_rng(seed + 10)
    qsz = np.maximum(1, sizes // 10)
    qidx = np.concatenate([o + rng.integers(0, m, q) for o, m, q in zip(off[:-1], sizes, qsz)])
    qoff = np.concatenate([[0], np.cumsum(qsz)]).astype(np.int64)
    Q = Pd[torch.from_numpy(qidx).cuda()].contiguous()
    qo = torch.from_numpy(qoff).cuda()
    nq = Q.shape[0]
    out = (torch.empty((nq, k), dtype=torch.float64, device="cuda"),
           torch.empty((nq, k), dtype=torch.int64, device="cuda"))
    f.knn_device(Q, qo, k, out=out)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        f.knn_device(Q, qo, k, out=out)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()
    l0 = L.ckd_launch_count()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            graph.replay()
        e1.record(stream)
        torch.cuda.synchronize()
    knn_ms = e0.elapsed_time(e1) / args.steps
    knn_i, knn_d = out[1].clone(), out[0].clone()
    persistent = run_forest_persistent(args, Pd, off, Q, qoff, k, knn_d, knn_i, stream)
    # boxes: 64 per tree, uniform centres
    B = np.empty((n_trees * nbox, 6))
    cen = rng.random((n_trees * nbox, 3)) - 0.5
    B[:, 0::2] = cen - side / 2
    B[:, 1::2] = cen + side / 2
    boff = np.arange(0, n_trees * nbox + 1, nbox, dtype=np.int64)
    Bd = torch.from_numpy(B).cuda()
    f.box_csr(Bd, boff)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        bo, bi = f.box_csr(Bd, boff)
    torch.cuda.synchronize()
    box_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    # end to end: host queries in, host results out
    Qh = Q.cpu().numpy()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dh, ih = f.knn(Qh, qoff, k)
    dh, ih = dh.cpu().numpy(), ih.cpu().numpy()
    e2e_s = time.perf_counter() - t0
    # oracle: exactness and CPU baseline on a sample of trees
    import oracle
    threads = os.cpu_count() or 1
    samp = rng.choice(n_trees, size=min(12, n_trees), replace=False)
    Ph = None
    ok = True
    cpu_q, cpu_s, ab_bytes, ab_q = 0, 0.0, 0.0, 0
    for t in samp:
        Pt = Pd[off[t]:off[t + 1]].cpu().numpy()
        ot = oracle.OracleTree(Pt, 16, [1.0, 1.0, 1.0], threads=threads)
        Qt = Qh[qoff[t]:qoff[t + 1]]
        t0 = time.perf_counter()
        od, oi = ot.knn(Qt, k)
        cpu_s += time.perf_counter() - t0
        cpu_q += len(Qt)
        ok = ok and np.array_equal(oi, ih[qoff[t]:qoff[t + 1]]) and \
            np.array_equal(od, dh[qoff[t]:qoff[t + 1]])
        ab = ot.knn_algbytes(Qt, k, od[:, -1] ** 2)
        ab_bytes += ab["bytes"]
        ab_q += len(Qt)
        ot.close()
    del Ph
    peak, peak_kind = measured_peaks()
    bpq = ab_bytes / max(1, ab_q)
    ach = bpq * nq / (knn_ms / 1e3) / 1e9
    outl = {
        "metric": "forest_knn_queries_per_s", "value": nq / (knn_ms / 1e3), "unit": "queries/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": knn_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "n_trees": n_trees, "n_points": n, "n_queries": int(nq),
                   "k": k, "boxes": int(len(B)), "box_side": side, "leaf": 16, "periodic": True,
                   "tree_sizes": "log-uniform [1e3, 1e6]", "seed": seed,
                   "l2": "inputs larger than L2", "launch": "kNN step replayed as one CUDA graph"},
        "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "traffic": None, "kernel": "k_knn_lane (forest roots)",
                     "kernel_ms": knn_ms, "alg_bytes_per_query": bpq, "peak_kind": peak_kind},
        "cpu_baseline": {"value": cpu_q / cpu_s, "unit": "queries/s", "cores": threads,
                         "kind": "port", "sample": f"{cpu_q} queries over {len(samp)} sampled "
                                                   "trees, reference traversal, FP64"},
        "e2e": {"value": nq / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": int(nq * 24),
                "d2h_bytes_per_step": int(nq * k * 16)},
        "gpu_launches": int(L.ckd_launch_count() - l0),
        "clocks": clk.summary(),
        "build": {"ms": build_ms[-1], "mpts_per_s": n / (build_ms[-1] / 1e3) / 1e6,
                  "n_nodes": f.n_nodes, "max_depth": f.depth},
        "boxes": {"ms": box_ms, "boxes_per_s": len(B) / (box_ms / 1e3),
                  "results": int(bo[-1].item())},
        "parity_sample": {"trees": int(len(samp)), "bit_exact": bool(ok)},
        "persistent": persistent,
    }
    print(json.dumps(outl))
    del graph
    f.close()
    return 0


def run_forest_persistent(args, Pd, off, Q, qoff, k, ref_d, ref_i, stream):
    """The whole forest built and queried by ONE persistent launch over a device
    work queue (ForestPlan), replayed as a CUDA graph: build + kNN per step.  The
    queries per work item come from the autotuner (timed on this forest, results
    checked equal across candidates, cached)."""
    import torch
    from cosmokdtree_b200 import ForestPlan
    from cosmokdtree_b200.autotune import Autotuner
    tuner = Autotuner()
    cfg = tuner.tune_forest_plan(Pd, off, Q, qoff, k, boxsize=1.0, reps=2)
    plan = ForestPlan(Pd, off, Q, qoff, k, leaf=cfg["leaf"], boxsize=1.0,
                      queries_per_block=cfg["queries_per_block"])
    plan.run()
    plan.check()
    exact = bool(torch.equal(plan.idx, ref_i) and torch.equal(plan.dist, ref_d))
    side = torch.cuda.Stream()
    side.wait_stream(stream)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            plan.run()
    stream.wait_stream(side)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    plan.check()
    exact = exact and bool(torch.equal(plan.idx, ref_i) and torch.equal(plan.dist, ref_d))
    n, nq = int(off[-1]), int(Q.shape[0])
    pf = plan.forest()
    out = {"method": "one persistent launch: (tree, level) build items and (tree, query "
                     "block) kNN items on a device work queue, replayed as a CUDA graph",
           "ms_per_step": ms, "points_per_s": n / (ms / 1e3), "queries_per_s": nq / (ms / 1e3),
           "exact_vs_forest_knn": exact, "n_nodes": pf.n_nodes, "depth": pf.depth,
           "tuned": {"leaf": cfg["leaf"], "queries_per_block": cfg["queries_per_block"],
                     "key": cfg.get("key"), "candidates_ms": cfg.get("candidates_ms")}}
    del graph
    plan.close()
    return out


def run_small_uniform(args):
    """The reference's small configuration: 2^20 uniform points in [0,1)^3, non-periodic,
    leaf 16; 10^5 uniform queries: kNN k=16 sorted, ball r=0.01 sorted (CSR), 10^3 boxes
    of side 0.02 at uniform centres; seed 0.  GPU times with CUDA events (inputs on the
    device), the CPU oracle on all host cores for the same calls, results compared."""
    import torch
    import oracle
    from cosmokdtree_b200 import _lib, kdtree
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    L = _lib.load()
    rng = np.random.default_rng(0)
    P = rng.random((1 << 20, 3))
    Qh = rng.random((100_000, 3))
    cen = rng.random((1000, 3))
    B = np.empty((1000, 6))
    B[:, 0::2] = cen - 0.01
    B[:, 1::2] = cen + 0.01
    Pd, Qd, Bd = (torch.from_numpy(x).cuda() for x in (P, Qh, B))
    stream = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps, out

    holder = {}

    def build():
        if "t" in holder:
            holder["t"].close()
        holder["t"] = kdtree.build_kdtree(Pd, leaf=16)
        return holder["t"]

    l0 = L.ckd_launch_count()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        build_ms, t = timed(build)
        knn_ms, (kd, ki) = timed(lambda: kdtree.knn_search_batch(t, Qd, 16, sorted=True))
        ball_ms, (bo, bi, bd) = timed(lambda: kdtree.ball_search_csr(t, Qd, 0.01, sorted=True))
        box_ms, (xo, xi) = timed(lambda: kdtree.box_search_csr(t, Bd))
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    ot = oracle.OracleTree(P, 16, None, threads=threads)
    cpu_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    od, oi = ot.knn(Qh, 16)
    cpu_knn = time.perf_counter() - t0
    t0 = time.perf_counter()
    oo, ob, obd = ot.ball_csr(Qh, 0.01, sorted=True)
    cpu_ball = time.perf_counter() - t0
    t0 = time.perf_counter()
    xo_o, xi_o = ot.box_csr(B)
    cpu_box = time.perf_counter() - t0
    exact = (np.array_equal(ki.cpu().numpy(), oi) and np.array_equal(kd.cpu().numpy(), od) and
             np.array_equal(bo.cpu().numpy(), oo) and np.array_equal(bi.cpu().numpy(), ob) and
             np.array_equal(bd.cpu().numpy(), obd) and np.array_equal(xo.cpu().numpy(), xo_o) and
             np.array_equal(xi.cpu().numpy(), xi_o))
    nq = len(Qh)
    out = {
        "metric": "knn_queries_per_s", "value": nq / (knn_ms / 1e3), "unit": "queries/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": knn_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "uniform_2p20_small", "n_points": 1 << 20, "n_queries": nq, "k": 16,
                   "ball_radius": 0.01, "boxes": 1000, "box_side": 0.02, "periodic": False,
                   "leaf": 16, "seed": 0, "l2": "tree and queries fit in L2 (small configuration)"},
        "knn": {"gpu_ms": knn_ms, "cpu_ms": cpu_knn * 1e3, "speedup": cpu_knn * 1e3 / knn_ms},
        "ball": {"gpu_ms": ball_ms, "cpu_ms": cpu_ball * 1e3, "speedup": cpu_ball * 1e3 / ball_ms,
                 "hits": int(bo[-1].item()), "sorted": True},
        "box": {"gpu_ms": box_ms, "cpu_ms": cpu_box * 1e3, "speedup": cpu_box * 1e3 / box_ms,
                "hits": int(xo[-1].item())},
        "build": {"gpu_ms": build_ms, "cpu_ms": cpu_build * 1e3,
                  "mpts_per_s": (1 << 20) / (build_ms / 1e3) / 1e6},
        "cpu_baseline": {"value": nq / cpu_knn, "unit": "queries/s", "cores": threads,
                         "kind": "port", "sample": "the full configuration (10^5 queries)"},
        "gpu_launches": int(L.ckd_launch_count() - l0),
        "clocks": clk.summary(),
        "exact_vs_oracle": bool(exact),
    }
    print(json.dumps(out))
    t.close()
    return 0


def run_multi(args):
    """Learned-bound vs plain kNN on a configuration with its own queries: a k per
    query drawn from the configuration's set, every step one mixed-k call (the
    queries are grouped by k on the device), optional 6-D float32 input.  The
    network is trained on 10^6 exact k-th distances of a separate catalogue of the
    same size and kind (train_seed) with queries drawn the same way."""
    import torch
    from cosmokdtree_b200 import _lib, kdtree, synth
    from cosmokdtree_b200.learned import LearnedBound
    cfg = MULTI_WORKLOADS[args.workload]
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    L = _lib.load()
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    n, d, ks, nq = cfg["n"], cfg["d"], cfg["ks"], cfg["nq"]
    box = [1.0] * d if cfg["periodic"] else None

    def catalogue(seed):
        if d == 6:
            return synth.phase_space(n, seed=seed, dtype=np.float32 if cfg["dtype"] == "f32"
                                     else np.float64)
        return synth.clustered_periodic(n, seed=seed)

    def queries(P, seed, m):
        if cfg["query"] == "mixed":
            return synth.mixed_queries(P, m, seed)
        rng = np.random.default_rng(seed)
        return np.ascontiguousarray(P[rng.integers(0, P.shape[0], m)].astype(np.float64))

    t0 = time.perf_counter()
    P = catalogue(cfg["seed"])
    gen_s = time.perf_counter() - t0
    Pd = torch.from_numpy(P).cuda()
    build_ms = []
    for it in range(2):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        tree = kdtree.build_kdtree(Pd, leaf=cfg["leaf"], boxsize=box)
        e1.record(stream)
        torch.cuda.synchronize()
        build_ms.append(e0.elapsed_time(e1))
        if it == 0:
            tree.close()
    del Pd
    # training on a separate catalogue
    t0 = time.perf_counter()
    Ptr = catalogue(cfg["train_seed"])
    ttr = kdtree.build_kdtree(torch.from_numpy(Ptr).cuda(), leaf=cfg["leaf"], boxsize=box)
    Qtr = torch.from_numpy(queries(Ptr, cfg["train_seed"] + 100, 1_000_000)).cuda()
    lb = LearnedBound(seed=0)
    fit = lb.fit(ttr, Qtr, list(ks), epochs=30, batch=4096, lr=3e-3, quantile=0.97)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    ttr.close()
    del Ptr, Qtr
    # evaluation queries with a k per query drawn from ks; one mixed-k call per step
    Qh = queries(P, cfg["query_seed"], nq)
    kq = np.asarray(ks, dtype=np.int32)[np.random.default_rng(cfg["query_seed"] + 1)
                                        .integers(0, len(ks), nq)]
    kmax = int(max(ks))
    Qd = torch.from_numpy(np.ascontiguousarray(Qh)).cuda()
    Kd = torch.from_numpy(kq).cuda()
    outs = [(torch.empty((nq, kmax), dtype=torch.float64, device="cuda"),
             torch.empty((nq, kmax), dtype=torch.int64, device="cuda")) for _ in range(2)]
    nfb = ctypes.c_int64()
    fallbacks = {}
    vp = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731

    def plain_step():
        _lib.check(L.ckd_knn_multi_k(tree.handle, vp(Qd), nq, vp(Kd), kmax, 1, vp(outs[0][0]),
                                     vp(outs[0][1]), sp))

    def learned_step():
        _lib.check(L.ckd_knn_learned_multi_k(tree.handle, lb.handle, vp(Qd), nq, vp(Kd), kmax, 1,
                                             vp(outs[1][0]), vp(outs[1][1]), ctypes.byref(nfb),
                                             sp))
        fallbacks["all"] = int(nfb.value)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    l0 = L.ckd_launch_count()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        plain_ms = timed(plain_step)
        learned_ms = timed(learned_step)
    launches = (L.ckd_launch_count() - l0) // (2 * (args.steps + args.warmup))
    exact = bool(torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1]))
    # oracle parity on a sample and CPU baseline
    import oracle
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    ot = oracle.OracleTree(P.astype(np.float64), cfg["leaf"], box, threads=threads)
    cpu_build_s = time.perf_counter() - t0
    parity = True
    cpu_q, cpu_s = 0, 0.0
    for k in ks:
        rows = np.nonzero(kq == k)[0][:2000]
        qs = Qh[rows]
        t1 = time.perf_counter()
        od, oi = ot.knn(qs, k)
        cpu_s += time.perf_counter() - t1
        cpu_q += len(qs)
        rsel = torch.from_numpy(rows).cuda()
        parity = parity and np.array_equal(oi, outs[1][1][rsel, :k].cpu().numpy()) and \
            np.array_equal(od, outs[1][0][rsel, :k].cpu().numpy())
    ot.close()
    out = {
        "metric": "knn_queries_per_s", "value": nq / (learned_ms / 1e3), "unit": "queries/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": learned_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "n_points": n, "dims": d, "n_queries": nq,
                   "k": list(ks), "queries": cfg["query"], "input_dtype": cfg["dtype"],
                   "leaf": cfg["leaf"], "periodic": cfg["periodic"], "seed": cfg["seed"],
                   "l2": "inputs larger than L2"},
        "plain": {"value": nq / (plain_ms / 1e3), "ms_per_step": plain_ms},
        "learned": {"value": nq / (learned_ms / 1e3), "speedup_vs_plain": plain_ms / learned_ms,
                    "exact_vs_plain": bool(exact),
                    "fallback_rate": fallbacks["all"] / nq,
                    "calls_per_step": "one mixed-k call (ckd_knn_multi_k / "
                                      "ckd_knn_learned_multi_k)",
                    "train_s": train_s, "margin_log2": fit["margin"],
                    "holdout_rms_log2": fit["holdout_rms_log2"]},
        "cpu_baseline": {"value": cpu_q / cpu_s, "unit": "queries/s", "cores": threads,
                         "kind": "port", "sample": f"{cpu_q} queries (2000 per k), FP64"},
        "gpu_launches_per_step": int(launches),
        "clocks": clk.summary(),
        "build": {"ms": build_ms[-1], "mpts_per_s": n / (build_ms[-1] / 1e3) / 1e6,
                  "cpu_s": cpu_build_s, "depth": tree.depth},
        "parity_sample": {"rows": cpu_q, "bit_exact": bool(parity)},
        "generation_s": gen_s,
    }
    print(json.dumps(out))
    tree.close()
    lb.close()
    return 0


def workload_config(name, world=1):
    n, k, periodic, leaf, seed = WORKLOADS[name]
    return {"workload": name, "n_points": n, "n_queries": n, "k": k, "sorted": True,
            "periodic": periodic, "leaf": leaf, "seed": seed, "dims": 3,
            "parallelism": f"tree replica per GPU, {world} contiguous query shard(s)",
            "l2": "inputs larger than L2 (tree ~0.6 GB, outputs 8.6 GB per step)"}


# DRAM bytes per working point and level of the build's three large kernels (k_seg_box,
# k_flags, k_scatter), from one ncu capture of each at a mid-depth level of the 16.7M-point
# clustered build (322.5 + 143.1 + 673.0 MB over ~11.3M working points)
BUILD_DRAM_BYTES_PER_POINT_LEVEL = 100.8
BUILD_TRAFFIC_NOTE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of k_seg_box, k_flags "
                      "and k_scatter at one mid-depth level, per working point, scaled by the "
                      "tree's point-levels (the per-level box, flag and scatter passes each "
                      "read the working set)")


def build_roofline(tree, n, d, ms):
    """Build roofline from the algorithmic bytes of a level-synchronous build: the
    input read once (N·D·8), every point read and written once per level above its
    leaf (Σ_p depth(p)·2·(D·8 + 4)), and the leaf-ordered write (N·(D·8 + 4))."""
    ex = tree.export()
    left, right, count, axis = ex["left"], ex["right"], ex["count"], ex["axis"]
    depth = np.zeros(len(left), dtype=np.int64)
    internal = np.nonzero(left >= 0)[0]
    for _ in range(int(tree.depth) + 1):  # preorder parents precede children
        depth[left[internal]] = depth[internal] + 1
        depth[right[internal]] = depth[internal] + 1
    leaves = axis < 0
    point_levels = int((depth[leaves] * count[leaves]).sum())
    rec = d * 8 + 4
    alg = n * d * 8 + point_levels * 2 * rec + n * rec
    peak, kind = measured_peaks()
    a = alg / (ms / 1e3) / 1e9
    traffic = BUILD_DRAM_BYTES_PER_POINT_LEVEL * point_levels if d == 3 else None
    return {"bound": "hbm", "achieved": a, "peak": peak, "unit": "GB/s", "frac": a / peak,
            "traffic": traffic, "traffic_note": BUILD_TRAFFIC_NOTE if traffic else None,
            "alg_bytes": alg, "point_levels_per_point": point_levels / n,
            "kernel": "whole build (all levels)", "peak_kind": kind}


def launch_ranks(n_gpus):
    """Relaunch this command under torchrun with one process per GPU (rendezvous on
    127.0.0.1) and return its exit status."""
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n_gpus}", "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    choices=sorted(WORKLOADS) + sorted(FOREST_WORKLOADS) +
                    sorted(MULTI_WORKLOADS) + ["uniform_2p20_small"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--variant", type=int, default=0, help="kNN kernel: 0 auto, 1 fp64, 2 screened")
    ap.add_argument("--stats", action="store_true", help="report traversal statistics (profile mode)")
    ap.add_argument("--tune", default="", help="comma list key=value of ckd_set_tuning knobs")
    ap.add_argument("--profile", action="store_true",
                    help="one build and the kNN steps only (for ncu captures)")
    ap.add_argument("--build-only", action="store_true",
                    help="warmup + steps builds of the workload's tree, nothing else (build "
                         "profiling; prints one line with the build times, not a bench line)")
    args = ap.parse_args()
    if args.impl == "reference":
        if args.workload in FOREST_WORKLOADS or args.workload in MULTI_WORKLOADS or \
                args.workload == "uniform_2p20_small":
            print(json.dumps({"impl": "reference", "unavailable": "this workload's CPU "
                              "baseline is reported inside the ours line (sampled queries)"}))
            return 0
        return run_reference(args)
    if args.workload in FOREST_WORKLOADS:
        return run_forest(args)
    if args.workload in MULTI_WORKLOADS:
        return run_multi(args)
    if args.workload == "uniform_2p20_small":
        return run_small_uniform(args)

    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        return launch_ranks(args.gpus)
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        print(json.dumps({"error": f"--gpus {args.gpus} but WORLD_SIZE={world}: launch one "
                                   "process per GPU"}))
        return 2
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
    P = make_points(name)  # the same catalogue on every rank: a tree replica per GPU
    box = [1.0, 1.0, 1.0] if periodic else None
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    # ---- build (device-resident input), Mpt/s
    Pd = torch.from_numpy(P).cuda()
    if args.build_only:
        stream = torch.cuda.current_stream()
        times = []
        for it in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            tree = kdtree.build_kdtree(Pd, leaf=leaf, boxsize=box)
            e1.record(stream)
            torch.cuda.synchronize()
            if it >= args.warmup:
                times.append(e0.elapsed_time(e1))
            tree.close()
        ms = float(np.mean(times))
        print(json.dumps({"mode": "build-only", "workload": name, "n": n, "leaf": leaf,
                          "build_ms": ms, "build_mpts": n / ms / 1e3, "all_ms": times}))
        return 0
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
    build_roof = build_roofline(tree, n, 3, build_ms_v) if rank == 0 else None
    # the input's host-to-device copy (pinned host buffer), reported beside the build
    P_pin = torch.from_numpy(P).pin_memory()
    Pd2 = torch.empty_like(Pd)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    Pd2.copy_(P_pin, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    build_h2d_ms = allmax(e0.elapsed_time(e1))
    del P_pin, Pd2

    # ---- kNN, inputs resident in HBM: every point of the catalogue is a query;
    # this rank searches its contiguous shard [lo, hi) against its replica
    from cosmokdtree_b200.distributed import knn_sharded, shard_bounds
    n_all = P.shape[0]
    lo, hi = shard_bounds(n_all, rank, world)
    nq = hi - lo
    Q = Pd[lo:hi]
    dist_t = torch.empty((nq, k), dtype=torch.float64, device="cuda")
    idx_t = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    dist_l = torch.empty((nq, k), dtype=torch.float64, device="cuda")
    idx_l = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    qp, dp, ip = (ctypes.c_void_p(x.data_ptr()) for x in (Q, dist_t, idx_t))
    dlp, ilp = (ctypes.c_void_p(x.data_ptr()) for x in (dist_l, idx_l))
    nfb = ctypes.c_int64()

    def search_into(t, q, kk, srt):
        _lib.check(L.ckd_knn(t.handle, ctypes.c_void_p(q.data_ptr()), q.shape[0], kk, int(srt),
                             dp, ip, sp))
        return dist_t, idx_t

    def plain_step():
        knn_sharded(tree, Pd, k, True, search=search_into)

    def learned_step():
        _lib.check(L.ckd_knn_learned(tree.handle, lb.handle, qp, nq, k, 1, dlp, ilp,
                                     ctypes.byref(nfb), sp))

    def timed(fn, steps, warmup):
        """W untimed steps, then K steps between barrier + synchronize; max over ranks."""
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
        l0 = L.ckd_launch_count()
        barrier()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for s_ in range(steps):
            evs[s_][0].record(stream)
            fn()
            evs[s_][1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
        barrier()
        total = allmax(t0.elapsed_time(t1))
        return total, [e[0].elapsed_time(e[1]) for e in evs], L.ckd_launch_count() - l0

    def kernel_ms(fn, reps=3):
        """Device time of the search kernels alone (CUDA events the library records
        on the launching stream around them)."""
        _lib.check(L.ckd_set_kernel_timing(1))
        vals = []
        for _ in range(reps):
            fn()
            v = ctypes.c_float()
            _lib.check(L.ckd_kernel_ms(ctypes.byref(v)))
            vals.append(v.value)
        _lib.check(L.ckd_set_kernel_timing(0))
        return float(np.mean(vals))

    def stats_of(fn):
        st = (ctypes.c_int64 * 8)()
        _lib.check(L.ckd_knn_stats(1, None))
        fn()
        _lib.check(L.ckd_knn_stats(0, st))
        return [v / nq for v in st]

    # ---- learned bound: trained on a separate catalogue (seed + 2), 10^6 samples
    from cosmokdtree_b200.learned import LearnedBound
    t_tr = time.perf_counter()
    P_tr = make_points(name, seed_offset=2)
    tree_tr = kdtree.build_kdtree(torch.from_numpy(P_tr).cuda(), leaf=leaf, boxsize=box)
    rng_tr = np.random.default_rng(3)
    n_train = min(1_000_000, P_tr.shape[0])
    Q_tr = torch.from_numpy(P_tr[rng_tr.integers(0, P_tr.shape[0], n_train)]).cuda()
    lb = LearnedBound(seed=0)
    fit = lb.fit(tree_tr, Q_tr, k, epochs=30 if not args.profile else 4, batch=4096, lr=3e-3,
                 quantile=0.97)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t_tr
    tree_tr.close()
    del Q_tr

    # ---- plain search
    with ClockSampler(local) as clk:
        plain_total, plain_steps, plain_launches = timed(plain_step, args.steps, args.warmup)
        learned_total, learned_steps, launches = timed(learned_step, args.steps, args.warmup)
    fallback = int(nfb.value)
    plain_kernel_ms = kernel_ms(plain_step)
    learned_kernel_ms = kernel_ms(learned_step)
    exact = bool(torch.equal(idx_l, idx_t) and torch.equal(dist_l, dist_t))
    exact = allmax(0.0 if exact else 1.0) == 0.0
    plain_value = n_all * args.steps / (plain_total / 1e3)
    learned_value = n_all * args.steps / (learned_total / 1e3)
    # headline: the default exact path (knn_search / ckd_knn); the learned-bound
    # search is reported beside it with its ratio
    value = plain_value
    ms_per_step = plain_total / args.steps
    clocks = clk.summary()

    # ---- ball search over the same queries: r = half the mean interparticle spacing.
    # Inside the NFW cusps a query holds up to ~10^5 neighbours within r, so the
    # full result (about 10^12 ids) cannot be materialised: the count pass (phase 1
    # of the CSR protocol) runs over every query, the full count + scan + fill over
    # a random subset whose CSR holds about 1.5e9 results (24 GB).
    radius = 0.5 * n ** (-1.0 / 3.0)
    counts = torch.empty(nq, dtype=torch.int64, device="cuda")
    cp = ctypes.c_void_p(counts.data_ptr())

    def ball_count_step():
        _lib.check(L.ckd_ball_count(tree.handle, qp, nq, radius, cp, sp))

    ball_count_total, _, _ = timed(ball_count_step, args.steps, args.warmup)
    total_hits = int(counts.sum().item())
    mean_hits = total_hits / nq
    m_ball = int(min(nq, max(1024, 1.5e9 / max(mean_hits, 1.0))))
    bq = Q[torch.randperm(nq, device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))[:m_ball]].contiguous()
    bqp = ctypes.c_void_p(bq.data_ptr())
    bcounts = torch.empty(m_ball, dtype=torch.int64, device="cuda")
    boff = torch.zeros(m_ball + 1, dtype=torch.int64, device="cuda")
    _lib.check(L.ckd_ball_count(tree.handle, bqp, m_ball, radius, ctypes.c_void_p(bcounts.data_ptr()), sp))
    _lib.check(L.ckd_exclusive_scan(ctypes.c_void_p(bcounts.data_ptr()),
                                    ctypes.c_void_p(boff.data_ptr()), m_ball, sp))
    n_hits = int(boff[-1].item())
    bidx = torch.empty(max(1, n_hits), dtype=torch.int64, device="cuda")
    bdist = torch.empty(max(1, n_hits), dtype=torch.float64, device="cuda")

    def ball_step():
        _lib.check(L.ckd_ball_count(tree.handle, bqp, m_ball, radius,
                                    ctypes.c_void_p(bcounts.data_ptr()), sp))
        _lib.check(L.ckd_exclusive_scan(ctypes.c_void_p(bcounts.data_ptr()),
                                        ctypes.c_void_p(boff.data_ptr()), m_ball, sp))
        _lib.check(L.ckd_ball_fill(tree.handle, bqp, m_ball, radius, 0,
                                   ctypes.c_void_p(boff.data_ptr()),
                                   ctypes.c_void_p(bidx.data_ptr()),
                                   ctypes.c_void_p(bdist.data_ptr()), sp))

    ball_total, _, ball_launches = timed(ball_step, args.steps, args.warmup)
    stats = None
    if args.stats:
        names = ["node_tests", "gathered_leaves", "leaf_scans", "points_screened", "flushes",
                 "fp64_evals", "heap_inserts", "misses"]
        stats = {"plain_per_query": dict(zip(names, stats_of(plain_step))),
                 "learned_per_query": dict(zip(names, stats_of(learned_step)))}
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "workload": name, "variant": args.variant,
                              "tune": args.tune, "plain_ms": plain_total / args.steps,
                              "learned_ms": ms_per_step, "plain_kernel_ms": plain_kernel_ms,
                              "learned_kernel_ms": learned_kernel_ms, "fallback": fallback,
                              "exact": exact, "stats": stats, "build_ms": build_ms_v,
                              "depth": tree.depth, "n_nodes": tree.n_nodes}))
        tree.close()
        return 0

    # ---- end to end through the public API with host buffers (learned and plain)
    def e2e(fn):
        vals = []
        res = None
        for it in range(args.e2e_steps + 1):
            res = None  # return the previous result's pinned host buffers to the cache
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            if it > 0:
                vals.append(e0.elapsed_time(e1))
        return allmax(float(np.mean(vals))), res

    samp = np.random.default_rng(7).integers(0, nq, 20000)  # parity rows (of this shard)
    Ph = P[lo:hi]
    e2e_learned_ms, res = e2e(lambda: lb.knn(tree, Ph, k, sorted=True))
    hd, hi_l = res[0][samp], res[1][samp]
    del res
    e2e_ms_v, res = e2e(lambda: kdtree.knn_search(tree, Ph, k, sorted=True))
    hd0, hi0 = res[0][samp], res[1][samp]
    del res

    if rank == 0:
        import oracle
        peak, peak_kind = measured_peaks()
        threads = os.cpu_count() or 1
        # reference-algorithm tree on the host: algorithmic bytes, parity sample, CPU baseline
        t0 = time.perf_counter()
        otree = oracle.OracleTree(P, leaf, 1.0 if periodic else None, threads=threads)
        cpu_build_s = time.perf_counter() - t0
        od, oi = otree.knn(Ph[samp], k)
        parity = bool(np.array_equal(oi, hi_l) and np.array_equal(od, hd) and
                      np.array_equal(oi, hi0) and np.array_equal(od, hd0))
        # ball parity on a sample: the count pass against the oracle's CSR
        bo_o, _, _ = otree.ball_csr(Ph[samp[:5000]], radius)
        ball_parity = bool(np.array_equal(np.diff(bo_o), counts[torch.from_numpy(samp[:5000]).cuda()].cpu().numpy()))
        ab = otree.knn_algbytes(Ph[samp], k, od[:, -1] ** 2)
        bytes_per_q = ab["bytes"] / len(samp)

        def roof(ms, kernel, traffic_per_q=None):
            a = bytes_per_q * nq / (ms / 1e3) / 1e9
            return {"bound": "hbm", "achieved": a, "peak": peak, "unit": "GB/s", "frac": a / peak,
                    "traffic": None if traffic_per_q is None else traffic_per_q * nq,
                    "traffic_note": None if traffic_per_q is None else KNN_TRAFFIC_NOTE,
                    "kernel": kernel, "kernel_ms": ms,
                    "alg_bytes_per_query": bytes_per_q, "peak_kind": peak_kind}

        cpu = None
        if world == 1 and not args.no_cpu:
            rate, m, dt = cpu_knn_rate(otree, P, k, target_s=args.cpu_seconds)
            cpu = {"value": rate, "unit": "queries/s", "cores": threads, "kind": "port",
                   "sample": f"{m} random self-queries of the catalogue in {dt:.1f} s, "
                             "reference traversal, FP64"}
        out = {
            "metric": "knn_queries_per_s", "value": value, "unit": "queries/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(name, world),
            "roofline": roof(plain_kernel_ms, "k_knn_lane2", KNN_DRAM_BYTES_PER_QUERY),
            "cpu_baseline": cpu,
            "e2e": {"value": n_all / (e2e_ms_v / 1e3), "unit": "queries/s",
                    "h2d_bytes_per_step": n_all * 3 * 8, "d2h_bytes_per_step": n_all * k * 16,
                    "ms_per_step": e2e_ms_v},
            "gpu_launches": int(plain_launches),
            "clocks": clocks,
            "learned": {"method": "learned-bound kNN (MLP 12-64-64-1, BF16 weights)",
                        "value": learned_value, "speedup_vs_plain": learned_value / plain_value,
                        "ms_per_step": learned_total / args.steps,
                        "exact_vs_plain": exact, "fallback_queries": fallback,
                        "fallback_rate": fallback / nq, "kernel_ms": learned_kernel_ms,
                        "gpu_launches": int(launches),
                        "roofline": roof(learned_kernel_ms,
                                         "k_mlp_radius + k_knn_lane2 (bounded) + rerun"),
                        "e2e_queries_per_s": n_all / (e2e_learned_ms / 1e3),
                        "train_s": train_s, "train_samples": fit["n_train"],
                        "train_catalogue_seed_offset": 2, "margin_log2": fit["margin"],
                        "holdout_rms_log2": fit["holdout_rms_log2"],
                        "holdout_rerun_rate": fit["holdout_rerun_rate"],
                        "final_loss": fit["loss"][-1]},
            "plain": {"value": plain_value, "ms_per_step": plain_total / args.steps,
                      "kernel_ms": plain_kernel_ms, "method": "knn_search / ckd_knn (default)"},
            "ball": {"radius": radius, "unit": "queries/s",
                     "count_pass": {"queries": n_all, "value": n_all * args.steps /
                                    (ball_count_total / 1e3),
                                    "ms_per_step": ball_count_total / args.steps,
                                    "total_hits": total_hits, "mean_hits": mean_hits},
                     "count_scan_fill": {"queries": m_ball, "value": world * m_ball * args.steps /
                                         (ball_total / 1e3),
                                         "ms_per_step": ball_total / args.steps, "hits": n_hits,
                                         "output": "CSR, unsorted (reference default)",
                                         "gpu_launches": int(ball_launches)},
                     "count_parity_sample": ball_parity},
            "build": {"ms": build_ms_v, "mpts_per_s": n / (build_ms_v / 1e3) / 1e6,
                      "input_h2d_ms": build_h2d_ms, "roofline": build_roof,
                      "cpu_s": cpu_build_s, "cpu_mpts_per_s": n / cpu_build_s / 1e6,
                      "n_nodes": tree.n_nodes, "depth": tree.depth},
            "breakdown_ms": {"learned_step": float(np.mean(learned_steps)),
                             "plain_step": float(np.mean(plain_steps)),
                             "plain_search_kernel": plain_kernel_ms},
            "parity_sample": {"rows": int(len(samp)), "bit_exact": parity},
        }
        if stats:
            out["stats"] = stats
        print(json.dumps(out))
    tree.close()
    lb.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
