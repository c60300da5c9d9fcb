"""Autotuner of the search launch parameters.

Every kNN kernel variant returns the same exact result, so the choice is purely
about speed and depends on the data (dimension, clustering, periodicity), k and
the GPU.  ``Autotuner.tune`` times a grid of configurations on a sample of the
user's own points and queries -- leaf size (tree build), kernel variant (which
also fixes how a node is expanded: per-lane compact heaps descending by
bounding boxes or by child-pair records; the packet traversal and the caller's
output rows for k > 64 are the fallbacks the automatic choice keeps),
warps per block, a cap on resident blocks per SM, and whether queries are
ordered by leaf -- checks that every candidate returns the baseline's result
bit for bit, and caches the fastest per (d, k, dtype, periodic, size class, GPU)
in a JSON file.  ``apply`` installs a configuration through ``ckd_set_tuning``
(process-wide) and returns the leaf size to build with.

    tuner = Autotuner()
    cfg = tuner.tune(points, queries, k=32, boxsize=1.0)   # or tuner.lookup(...)
    leaf = tuner.apply(cfg)
    tree = build_kdtree(points, leaf=leaf, boxsize=1.0)
"""
from __future__ import annotations

import itertools
import json
import math
import os
import time

import numpy as np

from . import _lib

__all__ = ["Autotuner", "DEFAULT_GRID", "config_key"]

# ckd_set_tuning keys
_KEY_VARIANT, _KEY_BPS, _KEY_WPB, _KEY_ORDER = 0, 1, 2, 6

DEFAULT_GRID = {
    "leaf": (8, 16, 32),
    "variant": (7, 8),
    "warps_per_block": (1, 2, 4),
    "blocks_per_sm": (0,),
    "order": (0,),
}

DEFAULT_CONFIG = {"leaf": 16, "variant": 0, "warps_per_block": 2, "blocks_per_sm": 0, "order": 0}


def config_key(d: int, k: int, dtype: str, periodic: bool, n: int, device_name: str) -> str:
    """Cache key: problem shape class and GPU model (n bucketed by powers of 4)."""
    size_class = int(round(math.log(max(n, 1), 4)))
    return f"d{d}-k{k}-{dtype}-{'per' if periodic else 'open'}-n4^{size_class}-{device_name}"


def _default_cache_path() -> str:
    env = os.environ.get("CKD_AUTOTUNE_CACHE")
    if env:
        return env
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "cosmokdtree_b200", "autotune.json")


class Autotuner:
    """Grid search with a persistent cache.  ``timer(cfg) -> ms`` and ``runner`` may be
    injected (tests); by default candidates are timed on the GPU with CUDA events."""

    def __init__(self, cache_path: str | None = None):
        self.cache_path = cache_path or _default_cache_path()
        self.cache = self._load()

    # ------------------------------------------------------------ cache
    def _load(self) -> dict:
        try:
            with open(self.cache_path) as f:
                data = json.load(f)
            return data if isinstance(data, dict) else {}
        except (OSError, ValueError):
            return {}

    def save(self) -> None:
        os.makedirs(os.path.dirname(os.path.abspath(self.cache_path)), exist_ok=True)
        tmp = self.cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.cache, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)

    def lookup(self, key: str) -> dict | None:
        e = self.cache.get(key)
        return dict(e["config"]) if e else None

    # ------------------------------------------------------------ apply
    @staticmethod
    def apply(cfg: dict) -> int:
        """Install a configuration (process-wide) and return its leaf size."""
        L = _lib.load()
        c = dict(DEFAULT_CONFIG, **(cfg or {}))
        _lib.check(L.ckd_set_tuning(_KEY_VARIANT, int(c["variant"])))
        _lib.check(L.ckd_set_tuning(_KEY_WPB, int(c["warps_per_block"])))
        _lib.check(L.ckd_set_tuning(_KEY_BPS, int(c["blocks_per_sm"])))
        _lib.check(L.ckd_set_tuning(_KEY_ORDER, int(c["order"])))
        return int(c["leaf"])

    @staticmethod
    def candidates(grid: dict | None = None) -> list[dict]:
        g = dict(DEFAULT_GRID, **(grid or {}))
        names = ["leaf", "variant", "warps_per_block", "blocks_per_sm", "order"]
        return [dict(zip(names, vals)) for vals in itertools.product(*(g[n] for n in names))]

    # ------------------------------------------------------------ search
    def tune(self, points, queries, k: int, boxsize=None, grid: dict | None = None, reps: int = 3,
             timer=None, key: str | None = None, save: bool = True) -> dict:
        """Time every candidate; return (and cache) the fastest exact configuration.

        ``timer(cfg) -> (ms, result)`` replaces the GPU measurement when given; the
        result is compared with the first candidate's (bit-exact)."""
        pts = np.asarray(points.cpu() if hasattr(points, "cpu") else points)
        n, d = pts.shape
        if key is None:
            key = config_key(d, int(k), str(pts.dtype), boxsize is not None, n, _device_name())
        timer = timer or _GpuTimer(points, queries, int(k), boxsize, reps)
        results = []
        ref = None
        try:
            for cfg in self.candidates(grid):
                ms, res = timer(cfg)
                if ref is None:
                    ref = res
                exact = _same(res, ref)
                results.append({"config": cfg, "ms": float(ms), "exact": exact})
        finally:
            if hasattr(timer, "close"):
                timer.close()
            self.apply(DEFAULT_CONFIG)
        ok = [r for r in results if r["exact"]]
        if len(ok) != len(results):
            bad = [r["config"] for r in results if not r["exact"]]
            raise RuntimeError(f"autotune: candidates disagree with the baseline result: {bad}")
        best = min(ok, key=lambda r: r["ms"])
        self.cache[key] = {"config": best["config"], "ms": best["ms"],
                           "tried": len(results), "when": time.strftime("%Y-%m-%d %H:%M:%S")}
        if save:
            self.save()
        out = dict(best["config"])
        out["ms"] = best["ms"]
        out["key"] = key
        out["results"] = results
        return out


    # ------------------------------------------------- persistent forest
    def tune_forest_plan(self, points, offsets, queries, query_offsets, k: int, boxsize=None,
                         grid: dict | None = None, reps: int = 3, key: str | None = None,
                         save: bool = True) -> dict:
        """Queries per work item (``queries_per_block``: 32 lanes x 4 warps per CTA
        take 128 queries at a time, so 32..512 covers 1/4 to 4 queries per lane)
        and leaf size of the persistent forest launch, timed as whole build + kNN
        runs on the caller's forest; every candidate's rows must equal the first
        candidate's bit for bit.  Cached per (d, k, periodic, forest size class,
        GPU); returns the best config with ``key`` and ``candidates_ms``."""
        import torch
        from .forest import ForestPlan
        g = {"leaf": (16,), "queries_per_block": (32, 64, 128, 256, 512)}
        g.update(grid or {})
        n, d = int(points.shape[0]), int(points.shape[1])
        if key is None:
            key = "forest-plan-" + config_key(d, int(k), "float64", boxsize is not None, n,
                                              _device_name())
        hit = self.cache.get(key)
        if hit is not None:
            out = dict(hit["config"])
            out.update(key=key, candidates_ms=hit.get("candidates_ms"), cached=True)
            return out
        results, ref = [], None
        for leaf in g["leaf"]:
            for qb in g["queries_per_block"]:
                plan = ForestPlan(points, offsets, queries, query_offsets, k, leaf=leaf,
                                  boxsize=boxsize, queries_per_block=qb)
                try:
                    plan.run()
                    plan.check()
                    times = []
                    for _ in range(reps):
                        e0 = torch.cuda.Event(enable_timing=True)
                        e1 = torch.cuda.Event(enable_timing=True)
                        e0.record()
                        plan.run()
                        e1.record()
                        plan.check()
                        times.append(e0.elapsed_time(e1))
                    res = (plan.dist.clone(), plan.idx.clone())
                finally:
                    plan.close()
                if ref is None:
                    ref = res
                if not _same(res, ref):
                    raise RuntimeError(f"autotune: forest plan leaf={leaf} qblock={qb} differs")
                results.append({"config": {"leaf": leaf, "queries_per_block": qb},
                                "ms": float(np.median(times))})
        best = min(results, key=lambda r: r["ms"])
        cand = {f"{r['config']['leaf']}/{r['config']['queries_per_block']}": r["ms"]
                for r in results}
        self.cache[key] = {"config": best["config"], "ms": best["ms"], "tried": len(results),
                           "candidates_ms": cand, "when": time.strftime("%Y-%m-%d %H:%M:%S")}
        if save:
            self.save()
        out = dict(best["config"])
        out.update(key=key, ms=best["ms"], candidates_ms=cand, cached=False)
        return out


def _same(a, b) -> bool:
    if a is None or b is None:
        return a is b
    return all(bool((x == y).all()) for x, y in zip(a, b))


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name().replace(" ", "_")
    except Exception:
        return "unknown"


class _GpuTimer:
    """Builds one tree per leaf size (cached) and times ckd_knn per candidate with
    CUDA events on the launching stream (median of ``reps`` after one warm-up)."""

    def __init__(self, points, queries, k, boxsize, reps):
        import torch
        from . import kdtree
        self.torch = torch
        self.kdtree = kdtree
        self.P = points if isinstance(points, torch.Tensor) and points.is_cuda else \
            torch.from_numpy(np.ascontiguousarray(np.asarray(points, dtype=np.float64))).cuda()
        self.Q = queries if isinstance(queries, torch.Tensor) and queries.is_cuda else \
            torch.from_numpy(np.ascontiguousarray(np.asarray(queries, dtype=np.float64))).cuda()
        self.k, self.box, self.reps = k, boxsize, reps
        self.trees = {}

    def __call__(self, cfg):
        torch = self.torch
        leaf = Autotuner.apply(cfg)
        if leaf not in self.trees:
            self.trees[leaf] = self.kdtree.build_kdtree(self.P, leaf=leaf, boxsize=self.box)
        t = self.trees[leaf]
        res = self.kdtree.knn_search_batch(t, self.Q, self.k)
        times = []
        for _ in range(self.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            res = self.kdtree.knn_search_batch(t, self.Q, self.k)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        return float(np.median(times)), res

    def close(self):
        for t in self.trees.values():
            t.close()
        self.trees.clear()
