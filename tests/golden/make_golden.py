"""Generate the golden fixtures in this directory (``golden_*.npz``).

The reference (Fortran) cannot run here and ships no golden vectors, so the
fixtures are the brute-force definitions its demo programs check by hand
(demos/cosmokdtree/periodic/tree_test.f90:79-139 for periodic kNN and ball,
demos/cosmokdtree/box_search/tree_test.f90:85-97 for box), computed with plain
numpy from seeded inputs -- independent of both the CPU oracle and the GPU code:

* kNN: the k smallest (d2, id), d2 summed axis by axis with separately rounded
  FP64 operations, minimum image when periodic; dist = sqrt(d2).  Missing slots
  (k > n) are id -2, dist sqrt(FLT_MAX).
* ball: every id with d2 <= r*r, ordered by (d2, id).
* box: every id with lo <= x <= hi on all axes, ascending id.  Boxes are drawn at
  random coordinates, so no box face coincides with a split plane and the
  reference's descent rule returns exactly this set.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FLT_MAX = float(np.finfo(np.float32).max)


def d2_all(P, q, L):
    s = np.zeros(P.shape[0])
    for j in range(P.shape[1]):
        dx = P[:, j] - q[j]
        if L is not None:
            a = np.abs(dx)
            dx = np.minimum(a, L[j] - a)
        s = s + dx * dx
    return s


def knn(P, Q, k, L):
    nq = Q.shape[0]
    dist = np.full((nq, k), np.sqrt(FLT_MAX))
    idx = np.full((nq, k), -2, np.int64)
    for i in range(nq):
        d2 = d2_all(P, Q[i], L)
        o = np.lexsort((np.arange(len(d2)), d2))[:k]
        o = o[d2[o] < FLT_MAX]
        dist[i, :len(o)] = np.sqrt(d2[o])
        idx[i, :len(o)] = o
    return dist, idx


def ball(P, Q, r, L):
    offs, ids, ds = [0], [], []
    for i in range(Q.shape[0]):
        d2 = d2_all(P, Q[i], L)
        sel = np.nonzero(d2 <= r * r)[0]
        sel = sel[np.lexsort((sel, d2[sel]))]
        ids.append(sel)
        ds.append(np.sqrt(d2[sel]))
        offs.append(offs[-1] + len(sel))
    return np.array(offs, np.int64), np.concatenate(ids).astype(np.int64), np.concatenate(ds)


def box(P, B):
    offs, ids = [0], []
    for b in B:
        m = np.all((P >= b[0::2]) & (P <= b[1::2]), axis=1)
        sel = np.nonzero(m)[0]
        ids.append(sel)
        offs.append(offs[-1] + len(sel))
    return np.array(offs, np.int64), np.concatenate(ids).astype(np.int64)


CASES = [
    # name, seed, n, d, periodic L, leaf, k, radius, nq, nb
    ("uniform3d", 10, 4000, 3, None, 16, 16, 0.08, 64, 16),
    ("periodic3d", 11, 4000, 3, 1.0, 16, 16, 0.08, 64, 16),
    ("periodic_demo", 12, 20000, 3, 100.0, 16, 100, 10.0, 4, 4),
    ("uniform6d", 13, 3000, 6, None, 32, 8, 0.35, 32, 8),
    ("clustered2d", 14, 3000, 2, None, 4, 7, 0.02, 48, 12),
    ("tiny_k_gt_n", 15, 11, 3, None, 16, 20, 0.5, 8, 4),
]


def points_for(name, rng, n, d, L):
    if name == "clustered2d":
        c = rng.random((6, d))
        P = c[rng.integers(0, 6, n)] + 0.01 * rng.standard_normal((n, d))
        P[:40] = P[0]  # exact duplicates
        return P
    if L is not None:
        return (rng.random((n, d)) - 0.5) * L
    return rng.random((n, d))


def main():
    for name, seed, n, d, L, leaf, k, r, nq, nb in CASES:
        rng = np.random.default_rng(seed)
        P = points_for(name, rng, n, d, L)
        Lv = None if L is None else np.full(d, float(L))
        if name == "periodic_demo":
            # the periodic demo's targets (periodic/tree_test.f90:81, :121)
            Q = np.array([[-49.6, 1.0, 43.0], [-44.6, 1.0, 43.0],
                          [49.9, -49.9, 0.0], [0.0, 0.0, 0.0]])
        elif L is not None:
            Q = (rng.random((nq, d)) - 0.5) * L
        else:
            Q = rng.random((nq, d))
            Q[: nq // 4] = P[: nq // 4]  # self queries (distance 0, ties)
        lo = rng.random((nb, d)) * (0.8 if L is None else 0.8 * L) - (0 if L is None else 0.4 * L)
        side = (0.2 if d <= 3 else 0.7) * (1.0 if L is None else L)
        B = np.empty((nb, 2 * d))
        B[:, 0::2] = lo
        B[:, 1::2] = lo + side * rng.random((nb, d))
        if name == "periodic_demo":
            B[0] = [-20, 10, -5, 20, -10, 10]  # box_search/tree_test.f90:77
        kd, ki = knn(P, Q, k, Lv)
        bo, bi, bd = ball(P, Q, r, Lv)
        xo, xi = box(P, B)
        np.savez_compressed(
            os.path.join(HERE, f"golden_{name}.npz"), points=P, queries=Q, boxes=B,
            boxsize=np.array([] if L is None else Lv), leaf=leaf, k=k, radius=r, knn_dist=kd,
            knn_idx=ki, ball_off=bo, ball_idx=bi, ball_dist=bd, box_off=xo, box_idx=xi)
        print(name, "points", P.shape, "ball hits", len(bi), "box hits", len(xi))


if __name__ == "__main__":
    main()
