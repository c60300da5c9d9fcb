"""Multi-GPU execution: one process per GPU, queries and trees sharded across ranks.

The search path has no exchange step: queries are independent, so every rank
holds its own replica of the tree in its own HBM (built there from the same
points, or from points broadcast once by rank 0) and searches a contiguous
shard of the queries.  Forests are split by tree with a greedy
longest-processing-time assignment on the tree sizes, so each rank builds and
searches only the trees it owns.  Gathering results to every rank is optional
plumbing after the search (``torch.distributed.all_gather`` over NCCL, or gloo
on CPU), never inside it.

Launch with ``torchrun --nproc-per-node N`` (RANK / WORLD_SIZE / LOCAL_RANK from
the environment) and call ``torch.distributed.init_process_group("nccl")``.
"""
from __future__ import annotations

import heapq

import numpy as np
import torch

__all__ = ["rank_world", "shard_bounds", "lpt_partition", "broadcast_points", "knn_sharded",
           "gather_rows", "build_forest_sharded"]


def rank_world(group=None) -> tuple[int, int]:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced split of n items: rank r gets [lo, hi)."""
    base, extra = divmod(int(n), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def lpt_partition(costs, world: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment: items in decreasing cost, each to
    the currently lightest rank (ties to the lower rank).  Returns the item indices
    of every rank, each list ascending."""
    order = np.argsort(-np.asarray(costs, dtype=np.float64), kind="stable")
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(int(i))
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def broadcast_points(points: torch.Tensor | None, src: int = 0, group=None) -> torch.Tensor:
    """Send rank ``src``'s points to every rank (one collective before the build)."""
    import torch.distributed as dist
    rank, world = rank_world(group)
    if world == 1:
        return points
    dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() and \
        dist.get_backend(group) == "nccl" else torch.device("cpu")
    shape = torch.zeros(2, dtype=torch.int64, device=dev)
    if rank == src:
        shape[0], shape[1] = points.shape
    dist.broadcast(shape, src, group=group)
    buf = points.to(dev, torch.float64).contiguous() if rank == src else \
        torch.empty((int(shape[0]), int(shape[1])), dtype=torch.float64, device=dev)
    dist.broadcast(buf, src, group=group)
    return buf


def gather_rows(local: torch.Tensor, group=None) -> torch.Tensor:
    """All-gather row blocks of different lengths (rank order)."""
    import torch.distributed as dist
    rank, world = rank_world(group)
    if world == 1:
        return local
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=local.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    m = max(sizes)
    pad = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([b[:s] for b, s in zip(bufs, sizes)])


def knn_sharded(tree, queries, k, sorted=True, group=None, gather=False, search=None):
    """kNN of this rank's contiguous shard of ``queries`` against its local tree
    replica.  Returns (dist, idx, (lo, hi)) for the shard, or the full (dist, idx)
    on every rank with ``gather=True``.  ``search(tree, q, k, sorted)`` defaults to
    ``kdtree.knn_search_batch``."""
    if search is None:
        from .kdtree import knn_search_batch as search
    rank, world = rank_world(group)
    lo, hi = shard_bounds(len(queries), rank, world)
    dist, idx = search(tree, queries[lo:hi], k, sorted)
    if not gather:
        return dist, idx, (lo, hi)
    return gather_rows(dist, group), gather_rows(idx, group)


def build_forest_sharded(points_per_tree, group=None, leaf=16, boxsize=None, build=None):
    """Build the trees this rank owns (LPT on tree sizes).  Returns (forest or
    None, owned tree indices).  ``build(list_of_points, leaf, boxsize)`` defaults
    to ``forest.build_forest``."""
    if build is None:
        from .forest import build_forest as build
    rank, world = rank_world(group)
    owned = lpt_partition([len(p) for p in points_per_tree], world)[rank]
    if not owned:
        return None, owned
    return build([points_per_tree[i] for i in owned], leaf=leaf, boxsize=boxsize), owned
