"""CPU oracle for the cosmokdtree build / kNN / ball / box path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py``.  The product package ``cosmokdtree_b200`` never
imports it.

The heavy lifting is ``libckd_oracle.so`` (``ckd_oracle.cpp``, a C++17/OpenMP
restatement of ``src/cosmokdtree.f90``); this module is a thin ctypes wrapper that
mirrors the reference Python API (``src/cosmokdtree/kdtree.py:16-87``).

Parity pinning: the reference ships no golden vectors and cannot be compiled here
(it is Fortran and there is no Fortran compiler in the image).  The oracle is pinned
against the reference's own brute-force demo checks, re-run seeded and asserted
(tests/test_oracle.py), against committed brute-force golden fixtures
(tests/golden/), and cross-checked against scipy's cKDTree.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libckd_oracle.so")
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_i32 = ctypes.POINTER(ctypes.c_int32)
_u8 = ctypes.POINTER(ctypes.c_uint8)


def build_library(force: bool = False) -> str:
    """Compile libckd_oracle.so with the Makefile beside this file."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "ckd_oracle.cpp"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build_library()
        L = ctypes.CDLL(_LIB_PATH)
        L.ora_build.argtypes = [_d, ctypes.c_int64, ctypes.c_int, ctypes.c_int, _d, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_void_p)]
        L.ora_build.restype = ctypes.c_int
        L.ora_free.argtypes = [ctypes.c_void_p]
        L.ora_n_nodes.argtypes = [ctypes.c_void_p]
        L.ora_n_nodes.restype = ctypes.c_int64
        L.ora_depth.argtypes = [ctypes.c_void_p]
        L.ora_depth.restype = ctypes.c_int
        L.ora_export.argtypes = [ctypes.c_void_p, _i32, _d, _i64, _i64, _u8, _i64, _i64, _d, _i64, _d]
        L.ora_knn.argtypes = [ctypes.c_void_p, _d, ctypes.c_int64, ctypes.c_int, ctypes.c_int, _d,
                              _i64, ctypes.c_int]
        L.ora_ball_count.argtypes = [ctypes.c_void_p, _d, ctypes.c_int64, ctypes.c_double, _i64,
                                     ctypes.c_int]
        L.ora_ball_fill.argtypes = [ctypes.c_void_p, _d, ctypes.c_int64, ctypes.c_double,
                                    ctypes.c_int, _i64, _i64, _d, ctypes.c_int]
        L.ora_box_count.argtypes = [ctypes.c_void_p, _d, ctypes.c_int64, _i64, ctypes.c_int]
        L.ora_box_fill.argtypes = [ctypes.c_void_p, _d, ctypes.c_int64, _i64, _i64, ctypes.c_int]
        L.ora_knn_algbytes.argtypes = [ctypes.c_void_p, _d, ctypes.c_int64, ctypes.c_int, _d, _d,
                                       ctypes.c_int]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


class OracleTree:
    """A k-d tree built by the CPU oracle.  ``threads=0`` uses every OpenMP thread."""

    def __init__(self, points, leaf=16, boxsize=None, threads=0):
        pts = np.ascontiguousarray(points, dtype=np.float64)
        if pts.ndim != 2:
            raise ValueError("points must be (n, d)")
        self.n, self.d = pts.shape
        self.leaf = int(leaf)
        self.periodic = boxsize is not None
        self.threads = threads
        box = None
        if boxsize is not None:
            box = np.ascontiguousarray(np.broadcast_to(np.asarray(boxsize, np.float64), (self.d,)))
        h = ctypes.c_void_p()
        rc = lib().ora_build(_p(pts, _d), self.n, self.d, self.leaf,
                             _p(box, _d) if box is not None else None, threads, ctypes.byref(h))
        if rc == 2:
            raise ValueError("Points outside (-L/2, L/2) range")
        if rc != 0:
            raise ValueError("oracle build: bad arguments")
        self._h = h
        self.boxsize = box

    def close(self):
        if getattr(self, "_h", None):
            lib().ora_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_nodes(self) -> int:
        return int(lib().ora_n_nodes(self._h))

    @property
    def depth(self) -> int:
        return int(lib().ora_depth(self._h))

    def export(self) -> dict:
        """Preorder node arrays plus the leaf-ordered ids and points."""
        m, d = self.n_nodes, self.d
        out = dict(axis=np.empty(m, np.int32), split=np.empty(m), start=np.empty(m, np.int64),
                   count=np.empty(m, np.int64), is_leaf=np.empty(m, np.uint8),
                   left=np.empty(m, np.int64), right=np.empty(m, np.int64),
                   cell=np.empty((m, 2 * d)), ids=np.empty(self.n, np.int64),
                   pts=np.empty((self.n, d)))
        lib().ora_export(self._h, _p(out["axis"], _i32), _p(out["split"], _d),
                         _p(out["start"], _i64), _p(out["count"], _i64), _p(out["is_leaf"], _u8),
                         _p(out["left"], _i64), _p(out["right"], _i64), _p(out["cell"], _d),
                         _p(out["ids"], _i64), _p(out["pts"], _d))
        return out

    def _q(self, target):
        q = np.ascontiguousarray(np.asarray(target, np.float64))
        if q.ndim == 1:
            q = q.reshape(1, -1)
        if q.shape[1] != self.d:
            raise ValueError("target dimensionality does not match the tree")
        return q

    def knn(self, target, k, sorted=True):
        q = self._q(target)
        nq = q.shape[0]
        dist = np.empty((nq, k))
        idx = np.empty((nq, k), np.int64)
        lib().ora_knn(self._h, _p(q, _d), nq, int(k), int(bool(sorted)), _p(dist, _d),
                      _p(idx, _i64), self.threads)
        return dist, idx

    def ball_csr(self, target, radius, sorted=False):
        q = self._q(target)
        nq = q.shape[0]
        counts = np.empty(nq, np.int64)
        lib().ora_ball_count(self._h, _p(q, _d), nq, float(radius), _p(counts, _i64), self.threads)
        offsets = np.zeros(nq + 1, np.int64)
        np.cumsum(counts, out=offsets[1:])
        m = int(offsets[-1])
        idx = np.empty(m, np.int64)
        dist = np.empty(m)
        lib().ora_ball_fill(self._h, _p(q, _d), nq, float(radius), int(bool(sorted)),
                            _p(offsets, _i64), _p(idx, _i64), _p(dist, _d), self.threads)
        return offsets, idx, dist

    def box_csr(self, boxes):
        b = np.ascontiguousarray(np.asarray(boxes, np.float64))
        if b.ndim == 1:
            b = b.reshape(1, -1)
        if b.shape[1] != 2 * self.d:
            raise ValueError("box size does not match tree dimensionality")
        nb = b.shape[0]
        counts = np.empty(nb, np.int64)
        lib().ora_box_count(self._h, _p(b, _d), nb, _p(counts, _i64), self.threads)
        offsets = np.zeros(nb + 1, np.int64)
        np.cumsum(counts, out=offsets[1:])
        idx = np.empty(int(offsets[-1]), np.int64)
        lib().ora_box_fill(self._h, _p(b, _d), nb, _p(offsets, _i64), _p(idx, _i64), self.threads)
        return offsets, idx

    def knn_algbytes(self, target, k, kth_d2):
        """Algorithmic bytes (and leaves / nodes / points) of an exact cell-pruned
        kNN search for these queries, given each query's exact k-th squared distance."""
        q = self._q(target)
        kd = np.ascontiguousarray(kth_d2, np.float64)
        out = np.zeros(4)
        lib().ora_knn_algbytes(self._h, _p(q, _d), q.shape[0], int(k), _p(kd, _d), _p(out, _d),
                               self.threads)
        return dict(bytes=out[0], leaves=out[1], nodes=out[2], points=out[3])


# --------------------------------------------------------------------------
# Reference-shaped functional API (src/cosmokdtree/kdtree.py:16-87)
def build_kdtree(points, leaf=None, boxsize=None, threads=0):
    return OracleTree(points, leaf=16 if leaf is None else leaf, boxsize=boxsize, threads=threads)


def knn_search(tree, target, k, sorted=True):
    return tree.knn(target, k, sorted)


def ball_search(tree, target, radius, sorted=False):
    off, idx, dist = tree.ball_csr(target, radius, sorted)
    return ([dist[off[i]:off[i + 1]] for i in range(len(off) - 1)],
            [idx[off[i]:off[i + 1]] for i in range(len(off) - 1)])


def box_search(tree, box):
    off, idx = tree.box_csr(box)
    return idx[off[0]:off[1]]


# --------------------------------------------------------------------------
# Brute-force definitions (the reference demos' checks, asserted)
def brute_d2(points, q, boxsize=None):
    """Squared distances with the reference's evaluation order (axis by axis,
    separately rounded), minimum image when periodic (cosmokdtree.f90:1441-1465)."""
    P = np.asarray(points, np.float64)
    q = np.asarray(q, np.float64)
    s = np.zeros(P.shape[0])
    for j in range(P.shape[1]):
        dx = P[:, j] - q[j]
        if boxsize is not None:
            a = np.abs(dx)
            L = float(np.broadcast_to(np.asarray(boxsize, np.float64), (P.shape[1],))[j])
            dx = np.minimum(a, L - a)
        s = s + dx * dx
    return s


def brute_knn(points, q, k, boxsize=None):
    d2 = brute_d2(points, q, boxsize)
    order = np.lexsort((np.arange(len(d2)), d2))[:k]
    return d2[order], order
