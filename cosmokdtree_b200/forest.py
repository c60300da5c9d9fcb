"""Forests: thousands of independent trees of uneven sizes built and searched together.

Halo and subvolume catalogues come as many small, independent point sets.  The
reference builds one tree per call (src/cosmokdtree/kdtree.py:16-34) and keeps
the periodic box side in a module global (src/cosmokdtree.f90:87); here all
trees are built by one level-synchronous pass over every tree at once and all
trees' queries go through one ordering pass and one search launch
(``ckd_forest_*`` in include/ckd.h).  Every tree is exactly the tree
``build_kdtree`` would make from its own points, and every result equals the
single-tree result, with ids local to the tree.

    forest = build_forest(points, offsets, leaf=16, boxsize=1.0)
    dist, idx = forest.knn(queries, query_offsets, k=8)      # CUDA tensors
    offs, ids = forest.box_csr(boxes, box_offsets)

``ForestPlan`` does the build and the kNN of a whole forest in ONE persistent
launch driven by a device work queue of (tree, level) and (tree, query block)
items; ``run()`` allocates nothing and does not synchronise, so it can be captured
in a CUDA graph and replayed:

    plan = ForestPlan(points, offsets, queries, query_offsets, k=8, boxsize=1.0)
    plan.run(); plan.check()                    # or capture plan.run() in a graph
    dist, idx = plan.dist, plan.idx
    offs, ids = plan.forest().box_csr(boxes, box_offsets)
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import CKDArgumentError, check
from .kdtree import _check_k, _on_device, _ptr, _stream

__all__ = ["Forest", "ForestPlan", "build_forest"]


def _offsets(off, n_trees=None, total=None, what="offsets") -> np.ndarray:
    o = np.asarray(off.cpu() if isinstance(off, torch.Tensor) else off, dtype=np.int64).reshape(-1)
    if o.size < 2 or o[0] != 0 or np.any(np.diff(o) < 0):
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, f"{what} must start at 0 and not decrease")
    if n_trees is not None and o.size != n_trees + 1:
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, f"{what} must have n_trees + 1 entries")
    if total is not None and o[-1] != total:
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, f"{what}[-1] must equal the number of rows")
    return np.ascontiguousarray(o)


def _rows(x, d, device, name):
    if isinstance(x, (list, tuple)):
        x = np.concatenate([np.asarray(a, dtype=np.float64).reshape(-1, d) for a in x]) \
            if len(x) else np.zeros((0, d))
    t = x.to(device=f"cuda:{device}", dtype=torch.float64) if _on_device(x) else \
        torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.float64)))
    if t.dim() != 2 or t.shape[1] != d:
        raise CKDArgumentError(_lib.CKD_ERR_BAD_DIM, f"{name} must be (n, {d})")
    if not t.is_cuda:
        t = t.pin_memory().to(f"cuda:{device}", non_blocking=True)
    return t.contiguous()


class Forest:
    """Handle of a forest built on one GPU (owns all device buffers)."""

    def __init__(self, handle, offsets, d, leaf, boxsize, device):
        self._h = handle
        self.offsets = offsets
        self.n_trees = len(offsets) - 1
        self.n = int(offsets[-1])
        self.d = d
        self.leaf = leaf
        self.boxsize = boxsize
        self.periodic = boxsize is not None
        self.device = device
        info = [ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()]
        check(_lib.load().ckd_tree_info(self._h, None, None, None, None, ctypes.byref(info[0]),
                                        ctypes.byref(info[1]), ctypes.byref(info[2]), None))
        self.n_nodes, self.n_leaves, self.depth = (int(x.value) for x in info)

    @property
    def handle(self):
        if self._h is None:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "forest has been deallocated")
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.load().ckd_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _grouped(self, x, off, name, width):
        x = _rows(x, width, self.device, name)
        o = _offsets(off, self.n_trees, x.shape[0], f"{name} offsets")
        if name == "queries" and self.periodic and x.shape[0] > 0:
            half = torch.as_tensor(self.boxsize / 2.0, dtype=torch.float64, device=x.device)
            if bool(((x < -half) | (x > half) | torch.isnan(x)).any()):
                raise CKDArgumentError(_lib.CKD_ERR_OUT_OF_BOX,
                                       "periodic forest: query points must lie in [-L/2, L/2]")
        return x, torch.from_numpy(o).to(f"cuda:{self.device}")

    def knn(self, queries, query_offsets, k, sorted=True):
        """kNN of queries grouped by tree (rows query_offsets[t] .. [t+1]-1 search
        tree t).  Returns (dist, idx) CUDA tensors (nq, k); ids local to the tree."""
        k = _check_k(k)
        with torch.cuda.device(self.device):
            q, qo = self._grouped(queries, query_offsets, "queries", self.d)
            return self.knn_device(q, qo, k, sorted)

    def knn_device(self, q: torch.Tensor, q_offsets: torch.Tensor, k: int, sorted=True,
                   out=None):
        """As ``knn`` with inputs already on the device (float64 (nq, d) and int64
        offsets) and optional preallocated outputs; does not synchronise, so it can
        be captured in a CUDA graph."""
        nq = q.shape[0]
        if out is None:
            dist = torch.empty((nq, k), dtype=torch.float64, device=q.device)
            idx = torch.empty((nq, k), dtype=torch.int64, device=q.device)
        else:
            dist, idx = out
        if nq > 0:
            check(_lib.load().ckd_forest_knn(self.handle, _ptr(q), _ptr(q_offsets), nq, int(k),
                                             int(bool(sorted)), _ptr(dist), _ptr(idx), _stream()))
        return dist, idx

    def box_csr(self, boxes, box_offsets):
        """Points inside each box ([lo0, hi0, lo1, hi1, ...] rows, grouped by tree
        like the kNN queries), as CSR CUDA tensors (offsets (nb+1,), idx)."""
        L = _lib.load()
        with torch.cuda.device(self.device):
            b, bo = self._grouped(boxes, box_offsets, "boxes", 2 * self.d)
            nb = b.shape[0]
            counts = torch.empty(nb, dtype=torch.int64, device=b.device)
            offsets = torch.zeros(nb + 1, dtype=torch.int64, device=b.device)
            if nb > 0:
                check(L.ckd_forest_box_count(self.handle, _ptr(b), _ptr(bo), nb, _ptr(counts),
                                             _stream()))
                check(L.ckd_exclusive_scan(_ptr(counts), _ptr(offsets), nb, _stream()))
            total = int(offsets[-1].item())
            idx = torch.empty(total, dtype=torch.int64, device=b.device)
            if nb > 0 and total > 0:
                check(L.ckd_forest_box_fill(self.handle, _ptr(b), _ptr(bo), nb, _ptr(offsets),
                                            _ptr(idx), _stream()))
        return offsets, idx

    def ball_csr(self, queries, query_offsets, radius, sorted=False):
        """Points within ``radius`` of each query (rows grouped by tree like the kNN
        queries), as CSR CUDA tensors (offsets (nq+1,), idx local to the query's
        tree, dist); ``sorted`` orders each row by (distance, id)."""
        radius = float(radius)
        if not radius > 0:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "Radius must be a positive number")
        L = _lib.load()
        with torch.cuda.device(self.device):
            q, qo = self._grouped(queries, query_offsets, "queries", self.d)
            nq = q.shape[0]
            counts = torch.empty(nq, dtype=torch.int64, device=q.device)
            offsets = torch.zeros(nq + 1, dtype=torch.int64, device=q.device)
            if nq > 0:
                check(L.ckd_forest_ball_count(self.handle, _ptr(q), _ptr(qo), nq, radius,
                                              _ptr(counts), _stream()))
                check(L.ckd_exclusive_scan(_ptr(counts), _ptr(offsets), nq, _stream()))
            total = int(offsets[-1].item())
            idx = torch.empty(total, dtype=torch.int64, device=q.device)
            dist = torch.empty(total, dtype=torch.float64, device=q.device)
            if nq > 0 and total > 0:
                check(L.ckd_forest_ball_fill(self.handle, _ptr(q), _ptr(qo), nq, radius,
                                             int(bool(sorted)), _ptr(offsets), _ptr(idx),
                                             _ptr(dist), _stream()))
        return offsets, idx, dist


def build_forest(points, offsets=None, leaf=16, boxsize=None) -> Forest:
    """Build every tree of a forest in one pass.  ``points`` is an (N, d) array
    (numpy or CUDA tensor) with ``offsets`` (n_trees + 1 row offsets), or a list of
    per-tree (n_t, d) arrays.  All trees share ``leaf`` and ``boxsize`` (None: not
    periodic; otherwise coordinates in [-L/2, L/2])."""
    if leaf is None:
        leaf = 16
    if not (int(leaf) == leaf and leaf > 0):
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "Leaf size must be a positive integer")
    leaf = int(leaf)
    if isinstance(points, (list, tuple)):
        sizes = [len(a) for a in points]
        d = np.asarray(points[0]).shape[1]
        pts = torch.from_numpy(np.ascontiguousarray(
            np.concatenate([np.asarray(a, dtype=np.float64).reshape(-1, d) for a in points])))
        off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    else:
        pts = points if _on_device(points) else torch.from_numpy(
            np.ascontiguousarray(np.asarray(points, dtype=np.float64)))
        if offsets is None:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "offsets are required with an (N, d) array")
        off = _offsets(offsets, total=pts.shape[0])
    if pts.dim() != 2:
        raise CKDArgumentError(_lib.CKD_ERR_BAD_DIM, "points must be an (n, d) array")
    n, d = pts.shape
    if np.any(np.diff(off) <= 0):
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "every tree needs at least one point")
    box = None
    if boxsize is not None:
        box = np.full(d, float(boxsize)) if np.ndim(boxsize) == 0 else \
            np.array(boxsize, dtype=np.float64)
        if len(box) != d:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_DIM, "boxsize must have d entries")
    if pts.dtype not in (torch.float32, torch.float64):
        pts = pts.to(torch.float64)
    dtype = _lib.CKD_F32 if pts.dtype == torch.float32 else _lib.CKD_F64
    device = pts.device.index if pts.is_cuda else torch.cuda.current_device()
    with torch.cuda.device(device):
        if not pts.is_cuda:
            pts = pts.pin_memory().to(f"cuda:{device}", non_blocking=True)
        pts = pts.contiguous()
        h = ctypes.c_void_p()
        boxp = box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if box is not None else None
        check(_lib.load().ckd_forest_build(
            _ptr(pts), off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(off) - 1, d, dtype,
            leaf, boxp, 1, _stream(), ctypes.byref(h)))
    return Forest(h, off, d, leaf, box, device)


class _PlanForest(Forest):
    """The forest a ForestPlan built (its arrays belong to the plan)."""

    def close(self):
        self._h = None


class ForestPlan:
    """Build a forest and answer its kNN queries in one persistent launch.

    ``points`` (N, d) and ``queries`` (nq, d) are float64 CUDA tensors (kept by
    reference and read at every ``run``), rows grouped by tree with host offsets;
    results land in ``self.dist`` / ``self.idx`` (nq, k), ids local to the tree,
    exactly the rows ``build_forest(...).knn(...)`` returns."""

    def __init__(self, points, offsets, queries, query_offsets, k, leaf=16, boxsize=None,
                 sorted=True, node_factor=0.0, queries_per_block=128):
        k = _check_k(k)
        if not (_on_device(points) and _on_device(queries)):
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "points and queries must be CUDA tensors")
        if points.dim() != 2 or queries.dim() != 2 or queries.shape[1] != points.shape[1]:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_DIM, "points and queries must be (n, d)")
        self.device = points.device.index
        self.points = points.to(torch.float64).contiguous()
        self.queries = queries.to(device=points.device, dtype=torch.float64).contiguous()
        n, d = self.points.shape
        nq = self.queries.shape[0]
        self.offsets = _offsets(offsets, total=n)
        self.query_offsets = _offsets(query_offsets, len(self.offsets) - 1, nq, "query offsets")
        self.n_trees = len(self.offsets) - 1
        self.d, self.k, self.leaf = d, k, int(leaf)
        box = None
        if boxsize is not None:
            box = np.full(d, float(boxsize)) if np.ndim(boxsize) == 0 else \
                np.array(boxsize, dtype=np.float64)
        self.boxsize = box
        self.dist = torch.empty((nq, k), dtype=torch.float64, device=points.device)
        self.idx = torch.empty((nq, k), dtype=torch.int64, device=points.device)
        self._h = None
        h = ctypes.c_void_p()
        P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))  # noqa: E731
        with torch.cuda.device(self.device):
            boxp = box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if box is not None else None
            check(_lib.load().ckd_forest_plan_create(
                _ptr(self.points), P(self.offsets), self.n_trees, d, self.leaf, boxp,
                _ptr(self.queries), P(self.query_offsets), nq, k, int(bool(sorted)),
                _ptr(self.dist), _ptr(self.idx), float(node_factor), int(queries_per_block),
                ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        if self._h is None:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "plan has been freed")
        return self._h

    def run(self):
        """Enqueue the launch on the current stream (no allocation, no sync)."""
        with torch.cuda.device(self.device):
            check(_lib.load().ckd_forest_plan_run(self.handle, _stream()))

    def check(self):
        """Synchronise and raise if the last run failed (CKDTimeout, CKDOutOfMemory...)."""
        with torch.cuda.device(self.device):
            check(_lib.load().ckd_forest_plan_status(self.handle, _stream()))

    def forest(self) -> Forest:
        """The forest of the last successful run, for box and ball searches."""
        h = ctypes.c_void_p()
        check(_lib.load().ckd_forest_plan_forest(self.handle, ctypes.byref(h)))
        return _PlanForest(h, self.offsets, self.d, self.leaf, self.boxsize, self.device)

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.load().ckd_forest_plan_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
