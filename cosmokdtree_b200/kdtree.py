"""Drop-in replacement of cosmokdtree's Python API (src/cosmokdtree/kdtree.py:16-87).

Same functions, arguments, defaults and results as the reference:

* ``build_kdtree(points, leaf=None, boxsize=None)``      (kdtree.py:16-34)
* ``deallocate_kdtree(tree)``                              (kdtree.py:37-38)
* ``knn_search(tree, target, k, sorted=True)``             (kdtree.py:41-53)
* ``ball_search(tree, target, radius, sorted=False)``      (kdtree.py:56-79)
* ``box_search(tree, box)``                                (kdtree.py:82-87)

plus batched variants that keep results on the GPU:

* ``knn_search_batch``  -> (dist, idx) CUDA tensors of shape (nq, k)
* ``ball_search_csr``   -> (offsets, idx, dist) CSR CUDA tensors
* ``box_search_csr``    -> (offsets, idx) CSR CUDA tensors for many boxes

Every search runs on the B200 through libckd.so (include/ckd.h); there is no CPU
path.  Host (numpy) inputs are copied to the device and results copied back;
CUDA-tensor inputs stay on the device.  Ids are 0-based int64; a kNN slot with no
neighbour (k > n) holds id -2 and distance 1.8446743523953730e19 exactly as the
reference returns them.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib
from ._lib import CKDArgumentError, check

__all__ = [
    "KDTree", "build_kdtree", "deallocate_kdtree", "knn_search", "ball_search", "box_search",
    "knn_search_batch", "knn_search_multi_k", "ball_search_csr", "box_search_csr", "box_search_periodic_csr",
    "save_kdtree", "load_kdtree", "read_fortran_points", "release_cached_memory",
]


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


class KDTree:
    """Opaque handle of a tree built on the GPU (the reference returns an int64 address,
    src/cosmokdtree2py.f90:70-73)."""

    def __init__(self, handle, n, d, leaf, boxsize, device):
        self._h = handle
        self.n = n
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
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "tree has been deallocated")
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

    def export(self) -> dict:
        """Structure in preorder (left first): axis (-1 leaf), split, start, count,
        left/right preorder children, cell and tight box (n_nodes x 2d), ids (leaf order)."""
        m, d = self.n_nodes, self.d
        out = dict(axis=np.empty(m, np.int32), split=np.empty(m), start=np.empty(m, np.int64),
                   count=np.empty(m, np.int64), left=np.empty(m, np.int64),
                   right=np.empty(m, np.int64), cell=np.empty((m, 2 * d)),
                   box=np.empty((m, 2 * d)), ids=np.empty(self.n, np.int64))
        P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
        with torch.cuda.device(self.device):
            check(_lib.load().ckd_tree_export(
                self.handle, P(out["axis"], ctypes.c_int32), P(out["split"], ctypes.c_double),
                P(out["start"], ctypes.c_int64), P(out["count"], ctypes.c_int64),
                P(out["left"], ctypes.c_int64), P(out["right"], ctypes.c_int64),
                P(out["cell"], ctypes.c_double), P(out["box"], ctypes.c_double),
                P(out["ids"], ctypes.c_int64)))
        return out


# ---------------------------------------------------------------- helpers

def _on_device(x) -> bool:
    return isinstance(x, torch.Tensor) and x.is_cuda


def _queries(tree: KDTree, target) -> tuple[torch.Tensor, bool]:
    """(nq, d) contiguous FP64 CUDA tensor on the tree's device, and whether the
    caller passed device data.  A 1-D target is one point (kdtree.py:45-46)."""
    dev = _on_device(target)
    if dev:
        q = target.to(device=f"cuda:{tree.device}", dtype=torch.float64)
    else:
        q = torch.from_numpy(np.ascontiguousarray(np.atleast_1d(np.asarray(target,
                                                                           dtype=np.float64))))
    if q.dim() == 1:
        q = q.reshape(1, -1)
    if q.dim() != 2 or q.shape[1] != tree.d:
        raise CKDArgumentError(_lib.CKD_ERR_BAD_DIM,
                               "target dimensionality does not match the tree")
    if not dev:
        q = q.pin_memory().to(f"cuda:{tree.device}", non_blocking=True)
    if tree.periodic and q.shape[0] > 0:  # checked on the device
        half = torch.as_tensor(tree.boxsize / 2.0, dtype=torch.float64, device=q.device)
        bad = (q < -half) | (q > half) | torch.isnan(q)
        if bool(bad.any()):
            raise CKDArgumentError(_lib.CKD_ERR_OUT_OF_BOX,
                                   "periodic tree: query points must lie in [-L/2, L/2]")
    return q.contiguous(), dev


def _to_host(t: torch.Tensor) -> np.ndarray:
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    return h.numpy()


# ---------------------------------------------------------------- build

def build_kdtree(points, leaf=None, boxsize=None) -> KDTree:
    """Build a k-d tree (kdtree.py:16-34).  ``boxsize=None`` gives a non-periodic tree;
    otherwise the tree is periodic with box sides ``boxsize`` and every coordinate must
    lie in [-L/2, L/2] (cosmokdtree.f90:177-190).  FP32 input is kept FP32 on the copy
    and widened on the device."""
    if leaf is None:
        leaf = 16
    if not (int(leaf) == leaf and leaf > 0):
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "Leaf size must be a positive integer")
    leaf = int(leaf)
    dev_in = _on_device(points)
    if dev_in:
        pts = points
        if pts.dtype not in (torch.float32, torch.float64):
            pts = pts.to(torch.float64)
    else:
        arr = np.asarray(points)
        if arr.dtype != np.float32:
            arr = arr.astype(np.float64, copy=False)
        pts = torch.from_numpy(np.ascontiguousarray(arr))
    if pts.dim() != 2:
        raise CKDArgumentError(_lib.CKD_ERR_BAD_DIM, "points must be an (n, d) array")
    n, d = pts.shape
    box = None
    if boxsize is not None:
        if np.ndim(boxsize) == 0:  # a scalar side is broadcast to every axis
            boxsize = np.full(d, float(boxsize))
        box = np.array(boxsize, dtype=np.float64, ndmin=1)
        if len(box) != d:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_DIM,
                                   "Incorrect dimensions for boxsize var. Size must be [Lx, Ly, Lz, ...]")
        if np.all(box == -1.0):  # the reference's "not periodic" sentinel (cosmokdtree2py.f90:48-55)
            box = None
    dtype = _lib.CKD_F32 if pts.dtype == torch.float32 else _lib.CKD_F64
    if dev_in:
        device = pts.device.index if pts.device.index is not None else torch.cuda.current_device()
    else:
        device = torch.cuda.current_device()
    with torch.cuda.device(device):
        if not dev_in:
            pts = pts.pin_memory().to(f"cuda:{device}", non_blocking=True)
        pts = pts.contiguous()
        h = ctypes.c_void_p()
        boxp = box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if box is not None else None
        check(_lib.load().ckd_build(_ptr(pts), n, d, dtype, leaf, boxp, 1, _stream(),
                                    ctypes.byref(h)))
    return KDTree(h, n, d, leaf, box, device)


def deallocate_kdtree(tree: KDTree) -> None:
    """Free the tree's device memory (kdtree.py:37-38).  The memory returns to the
    library's device pool, where the next build reuses it."""
    tree.close()


def release_cached_memory(device: int | None = None) -> None:
    """Hand the memory cached in the library's pool on ``device`` (freed trees and
    build scratch) back to the driver, e.g. before a large PyTorch allocation."""
    dev = torch.cuda.current_device() if device is None else int(device)
    with torch.cuda.device(dev):
        check(_lib.load().ckd_release_cached_memory())


# ---------------------------------------------------------------- kNN

def _check_k(k):
    if type(k) not in (int, np.int32, np.int64):  # kdtree.py:42
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "k must be an integer")
    if k < 1:
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "k must be a positive integer")
    return int(k)


def knn_search_batch(tree: KDTree, target, k, sorted=True):
    """k nearest neighbours of every target point; (dist, idx) CUDA tensors (nq, k)."""
    k = _check_k(k)
    with torch.cuda.device(tree.device):
        q, _ = _queries(tree, target)
        nq = q.shape[0]
        dist = torch.empty((nq, k), dtype=torch.float64, device=q.device)
        idx = torch.empty((nq, k), dtype=torch.int64, device=q.device)
        check(_lib.load().ckd_knn(tree.handle, _ptr(q), nq, k, int(bool(sorted)), _ptr(dist),
                                  _ptr(idx), _stream()))
    return dist, idx


_PIPE_MIN_ROWS = 1 << 20  # host queries from which the search and the copy-back overlap
_PIPE_CHUNKS = 16


def _host_rows(tree: KDTree, target) -> np.ndarray:
    """Host target points as a C-contiguous (nq, d) FP64 array (a 1-D target is one
    point, kdtree.py:45-46); the dimensionality is checked against the tree."""
    q = np.ascontiguousarray(np.atleast_1d(np.asarray(target, dtype=np.float64)))
    if q.ndim == 1:
        q = q.reshape(1, -1)
    if q.ndim != 2 or q.shape[1] != tree.d:
        raise CKDArgumentError(_lib.CKD_ERR_BAD_DIM,
                               "target dimensionality does not match the tree")
    return q


def _knn_host_pipelined(tree: KDTree, target, k: int, sorted: bool, search=None,
                        chunks: int = _PIPE_CHUNKS):
    """Host queries, host results, in row chunks: each chunk's queries are copied
    into one of two pinned staging buffers by the host while the device works on
    the previous chunks, uploaded and searched on the current stream, and its
    results copied into the pinned host arrays by a second stream (two device
    result buffers in flight), so both transfers overlap the search.  The periodic
    range check runs on the device per chunk into one flag, read once at the end
    (an out-of-range query raises then, and no result is returned).  ``search(q,
    n, dist, idx, stream)`` runs one chunk (default: ckd_knn); a search with fixed
    costs per call takes fewer ``chunks``."""
    L = _lib.load()
    if search is None:
        def search(qc, n, db, ib, st):
            check(L.ckd_knn(tree.handle, _ptr(qc), n, k, int(bool(sorted)), _ptr(db), _ptr(ib),
                            st))
    qh = _host_rows(tree, target)
    nq, d = qh.shape
    dev = torch.device(f"cuda:{tree.device}")
    rows = -(-nq // max(1, int(chunks)))
    q = torch.empty((nq, d), dtype=torch.float64, device=dev)
    stage = [torch.empty((rows, d), dtype=torch.float64, pin_memory=True) for _ in range(2)]
    uploaded = [None, None]
    bad = None
    if tree.periodic:
        half = torch.as_tensor(tree.boxsize / 2.0, dtype=torch.float64, device=dev)
        bad = torch.zeros((), dtype=torch.bool, device=dev)
    dist_h = torch.empty((nq, k), dtype=torch.float64, pin_memory=True)
    idx_h = torch.empty((nq, k), dtype=torch.int64, pin_memory=True)
    comp = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    bufs = [(torch.empty((rows, k), dtype=torch.float64, device=dev),
             torch.empty((rows, k), dtype=torch.int64, device=dev)) for _ in range(2)]
    done = [None, None]
    for c, r0 in enumerate(range(0, nq, rows)):
        r1 = min(nq, r0 + rows)
        b = c % 2
        if uploaded[b] is not None:
            uploaded[b].synchronize()  # the staging buffer's previous upload has finished
        stage[b][: r1 - r0].copy_(torch.from_numpy(qh[r0:r1]))
        qc = q[r0:r1]
        qc.copy_(stage[b][: r1 - r0], non_blocking=True)
        uploaded[b] = torch.cuda.Event()
        uploaded[b].record(comp)
        if bad is not None:
            bad |= ((qc < -half) | (qc > half) | torch.isnan(qc)).any()
        if done[b] is not None:
            comp.wait_event(done[b])  # the buffer's previous copy has finished
        db, ib = bufs[b]
        search(qc, r1 - r0, db, ib, ctypes.c_void_p(comp.cuda_stream))
        ready = torch.cuda.Event()
        ready.record(comp)
        copy.wait_event(ready)
        with torch.cuda.stream(copy):
            dist_h[r0:r1].copy_(db[: r1 - r0], non_blocking=True)
            idx_h[r0:r1].copy_(ib[: r1 - r0], non_blocking=True)
        done[b] = torch.cuda.Event()
        done[b].record(copy)
    copy.synchronize()
    comp.wait_stream(copy)
    if bad is not None and bool(bad):
        raise CKDArgumentError(_lib.CKD_ERR_OUT_OF_BOX,
                               "periodic tree: query points must lie in [-L/2, L/2]")
    return dist_h.numpy(), idx_h.numpy()


def knn_search(tree: KDTree, target, k, sorted=True):
    """k nearest neighbours (kdtree.py:41-53).  Returns (dist, idx), each (ntar, k):
    numpy arrays for host input, CUDA tensors for CUDA-tensor input."""
    if not _on_device(target):
        k = _check_k(k)
        nq = np.shape(target)[0] if np.ndim(target) == 2 else 1
        if nq >= _PIPE_MIN_ROWS:
            with torch.cuda.device(tree.device):
                return _knn_host_pipelined(tree, target, k, sorted)
    dist, idx = knn_search_batch(tree, target, k, sorted)
    if _on_device(target):
        return dist, idx
    with torch.cuda.device(tree.device):
        return _to_host(dist), _to_host(idx)


def knn_search_multi_k(tree: KDTree, target, ks, sorted=True):
    """k nearest neighbours with a k per target point, in one call.  ``ks`` holds
    one positive integer per target row.  Returns (dist, idx) of shape
    (ntar, max(ks)); a row's slots past its own k hold id -2 and distance
    1.8446743523953730e19 (the k > n marker).  numpy for host input, CUDA tensors
    for CUDA-tensor input."""
    with torch.cuda.device(tree.device):
        q, _ = _queries(tree, target)
        nq = q.shape[0]
        kt = torch.as_tensor(np.asarray(ks) if not isinstance(ks, torch.Tensor) else ks)
        if kt.dim() != 1 or kt.shape[0] != nq:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "ks must hold one k per target row")
        if kt.dtype.is_floating_point or kt.dtype == torch.bool:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "k must be an integer")
        kt = kt.to(device=q.device, dtype=torch.int32).contiguous()
        kmax = int(kt.max().item()) if nq > 0 else 1
        if nq > 0 and int(kt.min().item()) < 1:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "k must be a positive integer")
        dist = torch.empty((nq, kmax), dtype=torch.float64, device=q.device)
        idx = torch.empty((nq, kmax), dtype=torch.int64, device=q.device)
        if nq > 0:
            check(_lib.load().ckd_knn_multi_k(tree.handle, _ptr(q), nq, _ptr(kt), kmax,
                                              int(bool(sorted)), _ptr(dist), _ptr(idx), _stream()))
        if _on_device(target):
            return dist, idx
        return _to_host(dist), _to_host(idx)


# ---------------------------------------------------------------- ball

def _check_radius(radius):
    if not radius > 0.0:  # kdtree.py:57
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "Radius must be a positive number")
    return float(radius)


def ball_search_csr(tree: KDTree, target, radius, sorted=False):
    """All points within ``radius`` of every target, as CSR CUDA tensors
    (offsets (nq+1,), idx, dist)."""
    radius = _check_radius(radius)
    L = _lib.load()
    with torch.cuda.device(tree.device):
        q, _ = _queries(tree, target)
        nq = q.shape[0]
        counts = torch.empty(nq, dtype=torch.int64, device=q.device)
        offsets = torch.zeros(nq + 1, dtype=torch.int64, device=q.device)
        if nq > 0:
            check(L.ckd_ball_count(tree.handle, _ptr(q), nq, radius, _ptr(counts), _stream()))
            check(L.ckd_exclusive_scan(_ptr(counts), _ptr(offsets), nq, _stream()))
        total = int(offsets[-1].item())
        idx = torch.empty(total, dtype=torch.int64, device=q.device)
        dist = torch.empty(total, dtype=torch.float64, device=q.device)
        if nq > 0 and total > 0:
            check(L.ckd_ball_fill(tree.handle, _ptr(q), nq, radius, int(bool(sorted)),
                                  _ptr(offsets), _ptr(idx), _ptr(dist), _stream()))
    return offsets, idx, dist


def ball_search(tree: KDTree, target, radius, sorted=False):
    """Ball search (kdtree.py:56-79): per target lists of distances and 0-based ids."""
    offsets, idx, dist = ball_search_csr(tree, target, radius, sorted)
    with torch.cuda.device(tree.device):
        off, i, d = _to_host(offsets), _to_host(idx), _to_host(dist)
    n = len(off) - 1
    return ([d[off[j]:off[j + 1]] for j in range(n)], [i[off[j]:off[j + 1]] for j in range(n)])


# ---------------------------------------------------------------- box

def box_search_csr(tree: KDTree, boxes):
    """Points inside each of many axis-aligned boxes ([lo0, hi0, lo1, hi1, ...] rows),
    CSR CUDA tensors (offsets (nb+1,), idx)."""
    L = _lib.load()
    with torch.cuda.device(tree.device):
        if _on_device(boxes):
            b = boxes.to(device=f"cuda:{tree.device}", dtype=torch.float64)
        else:
            b = torch.from_numpy(np.array(boxes, dtype=np.float64, copy=True, ndmin=1))
        if b.dim() == 1:
            b = b.reshape(1, -1)
        if b.shape[-1] != 2 * tree.d:  # cosmokdtree2py.f90:275-277
            raise CKDArgumentError(_lib.CKD_ERR_BAD_DIM,
                                   "Error: box size does not match tree dimensionality.")
        b = b.to(f"cuda:{tree.device}").contiguous()
        nb = b.shape[0]
        counts = torch.empty(nb, dtype=torch.int64, device=b.device)
        offsets = torch.zeros(nb + 1, dtype=torch.int64, device=b.device)
        if nb > 0:
            check(L.ckd_box_count(tree.handle, _ptr(b), nb, _ptr(counts), _stream()))
            check(L.ckd_exclusive_scan(_ptr(counts), _ptr(offsets), nb, _stream()))
        total = int(offsets[-1].item())
        idx = torch.empty(total, dtype=torch.int64, device=b.device)
        if nb > 0 and total > 0:
            check(L.ckd_box_fill(tree.handle, _ptr(b), nb, _ptr(offsets), _ptr(idx), _stream()))
    return offsets, idx


def box_search(tree: KDTree, box):
    """Ids of the points inside one box [xmin, xmax, ymin, ymax, ...] (kdtree.py:82-87)."""
    b = np.array(box, dtype=np.float64, ndmin=1).reshape(-1)
    offsets, idx = box_search_csr(tree, b.reshape(1, -1))
    with torch.cuda.device(tree.device):
        return _to_host(idx)


def _wrap_pieces(lo, hi, L):
    """Pieces of [lo, hi] on a periodic axis of side L, each inside [-L/2, L/2]."""
    if hi - lo >= L:
        return [(-L / 2, L / 2)]
    a = ((lo + L / 2) % L) - L / 2
    b = a + (hi - lo)
    if b <= L / 2:
        return [(a, b)]
    return [(a, L / 2), (-L / 2, b - L)]


def box_search_periodic_csr(tree: KDTree, boxes):
    """Box search that wraps boxes across the faces of a periodic tree (opt-in).

    The reference's box_search never wraps (src/cosmokdtree.f90:1258-1328): a box
    that crosses a face of the periodic box silently misses the points on the far
    side, and ``box_search`` / ``box_search_csr`` keep that behaviour.  Here each box
    [lo0, hi0, lo1, hi1, ...] (coordinates in any image; a side >= L covers the whole
    axis) is split on every axis into at most two pieces inside [-L/2, L/2], the
    pieces are searched with the reference's descent rule, and each box's ids are
    returned sorted.  Returns CSR CUDA tensors (offsets (nb+1,), idx)."""
    if not tree.periodic:
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "periodic box search needs a periodic tree")
    b = boxes.detach().cpu().numpy() if _on_device(boxes) else np.asarray(boxes, dtype=np.float64)
    b = np.array(b, dtype=np.float64, ndmin=2)
    d = tree.d
    if b.shape[-1] != 2 * d:
        raise CKDArgumentError(_lib.CKD_ERR_BAD_DIM,
                               "Error: box size does not match tree dimensionality.")
    if not np.all(np.isfinite(b)):
        raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "box coordinates must be finite")
    L = tree.boxsize
    pieces, owner = [], []
    for i, row in enumerate(b):
        axes = [_wrap_pieces(row[2 * j], row[2 * j + 1], L[j]) for j in range(d)]
        combos = [[]]
        for ax in axes:
            combos = [c + [p] for c in combos for p in ax]
        for c in combos:
            pieces.append([v for lohi in c for v in lohi])
            owner.append(i)
    nb = b.shape[0]
    with torch.cuda.device(tree.device):
        if not pieces:
            return (torch.zeros(nb + 1, dtype=torch.int64, device=f"cuda:{tree.device}"),
                    torch.empty(0, dtype=torch.int64, device=f"cuda:{tree.device}"))
        off, idx = box_search_csr(tree, np.array(pieces))
        dev = off.device
        own = torch.as_tensor(owner, dtype=torch.int64, device=dev)
        rows = torch.repeat_interleave(own, off[1:] - off[:-1])
        key = torch.unique(rows * max(1, tree.n) + idx)  # sorted; drops repeats
        rows, idx = key // max(1, tree.n), key % max(1, tree.n)
        counts = torch.bincount(rows, minlength=nb)
        offsets = torch.zeros(nb + 1, dtype=torch.int64, device=dev)
        offsets[1:] = torch.cumsum(counts, 0)
    return offsets, idx


# ---------------------------------------------------------------- files

def save_kdtree(tree, path: str) -> None:
    """Write a built tree (or forest) to ``path``; ``load_kdtree`` restores it without
    rebuilding and with bit-identical results."""
    with torch.cuda.device(tree.device):
        check(_lib.load().ckd_tree_save(tree.handle, os.fsencode(path)))


def load_kdtree(path: str, device=None):
    """Load a tree saved by ``save_kdtree`` onto ``device`` (default: current).
    Returns a KDTree, or a Forest when the file holds several trees."""
    device = torch.cuda.current_device() if device is None else int(device)
    L = _lib.load()
    with torch.cuda.device(device):
        h = ctypes.c_void_p()
        check(L.ckd_tree_load(os.fsencode(path), ctypes.byref(h)))
        n, d, leaf, per = ctypes.c_int64(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(L.ckd_tree_info(h, ctypes.byref(n), ctypes.byref(d), ctypes.byref(leaf),
                              ctypes.byref(per), None, None, None, None))
        nt = ctypes.c_int64()
        check(L.ckd_forest_info(h, ctypes.byref(nt), None))
        off = np.empty(nt.value + 1, np.int64)
        check(L.ckd_forest_info(h, None, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        box = None
        if per.value:
            box = _saved_boxsize(path, d.value)
    if nt.value > 1:
        from .forest import Forest
        return Forest(h, off, d.value, leaf.value, box, device)
    return KDTree(h, int(n.value), d.value, leaf.value, box, device)


def _saved_boxsize(path: str, d: int) -> np.ndarray:
    # header after the 8-byte magic: 2 int64, 8 int32, then 8 float64 box sides
    with open(path, "rb") as f:
        f.seek(8 + 16 + 32)
        return np.frombuffer(f.read(8 * d), dtype=np.float64).copy()


def read_fortran_points(path: str, dtype=np.float32) -> np.ndarray:
    """Read a point file in the reference's Fortran unformatted sequential layout
    (build/inhomogeneous/tree_test.f90:72-81, generate_inhomogeneous_distribution.py:61-65):
    a record holding the int32 point count n, then one record per coordinate axis
    holding n values (float32 by default).  Each record is framed by 4-byte length
    markers.  Returns an (n, d) array (d = number of coordinate records)."""
    raw = np.fromfile(path, dtype=np.uint8)
    pos, recs = 0, []
    while pos < raw.size:
        if pos + 4 > raw.size:
            raise ValueError(f"{path}: truncated record marker")
        ln = int(raw[pos:pos + 4].view(np.int32)[0])
        body = raw[pos + 4:pos + 4 + ln]
        end = pos + 4 + ln
        if ln < 0 or end + 4 > raw.size or int(raw[end:end + 4].view(np.int32)[0]) != ln:
            raise ValueError(f"{path}: inconsistent record markers")
        recs.append(body)
        pos = end + 4
    if not recs or recs[0].size != 4:
        raise ValueError(f"{path}: first record must hold the int32 point count")
    n = int(recs[0].view(np.int32)[0])
    axes = [r.view(dtype) for r in recs[1:]]
    if not axes or any(a.size != n for a in axes):
        raise ValueError(f"{path}: coordinate records must each hold {n} values")
    return np.ascontiguousarray(np.stack(axes, axis=1))
