"""Forests on the GPU: every tree of a forest gives exactly the results of the
same points built alone (kNN and box, bit-exact, ids local to the tree), checked
against the single-tree path and the CPU oracle; CUDA-graph capture of the
forest kNN; argument errors."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _forest_points(n_trees, seed, periodic):
    from cosmokdtree_b200 import synth
    rng = np.random.default_rng(seed)
    sizes = np.floor(10 ** rng.uniform(1.0, 4.3, n_trees)).astype(int)
    sizes[0] = 1          # a tree with one point
    sizes[1] = 16         # a tree that is a single leaf
    pts = []
    for t, m in enumerate(sizes):
        P = synth.nfw_cluster(int(m), seed * 1000 + t)
        pts.append(P if periodic else P * 0.9)
    return pts


def _queries_per_tree(pts, rng, frac=0.1):
    qs = []
    for P in pts:
        m = max(1, int(frac * len(P)))
        q = P[rng.integers(0, len(P), m)].copy()
        q[: m // 2] = rng.random((m // 2, 3)) - 0.5
        qs.append(q)
    return qs


@pytest.mark.parametrize("periodic", [True, False])
def test_forest_knn_matches_single_trees(gpu, oracle, periodic):
    from cosmokdtree_b200 import kdtree, build_forest
    rng = np.random.default_rng(61)
    pts = _forest_points(48, 61 + periodic, periodic)
    box = 1.0 if periodic else None
    f = build_forest(pts, leaf=16, boxsize=box)
    assert f.n_trees == 48 and f.n == sum(len(p) for p in pts)
    qs = _queries_per_tree(pts, rng)
    qoff = np.concatenate([[0], np.cumsum([len(q) for q in qs])])
    for k in (8, 20):
        d, i = f.knn(qs, qoff, k)
        d, i = d.cpu().numpy(), i.cpu().numpy()
        for t, (P, Q) in enumerate(zip(pts, qs)):
            tr = kdtree.build_kdtree(P, leaf=16, boxsize=box)
            d1, i1 = kdtree.knn_search(tr, Q, k)
            np.testing.assert_array_equal(i[qoff[t]:qoff[t + 1]], i1)
            np.testing.assert_array_equal(d[qoff[t]:qoff[t + 1]], d1)
            if t % 12 == 2:
                ot = oracle.OracleTree(P, 16, [1.0] * 3 if periodic else None)
                od, oi = ot.knn(Q, k)
                np.testing.assert_array_equal(i1, oi)
                np.testing.assert_array_equal(d1, od)
    f.close()


def test_forest_box_matches_single_trees(gpu):
    from cosmokdtree_b200 import kdtree, build_forest
    rng = np.random.default_rng(62)
    pts = _forest_points(40, 62, True)
    f = build_forest(pts, leaf=16, boxsize=1.0)
    boxes = []
    for P in pts:
        lo = rng.random((9, 3)) * 0.6 - 0.35
        b = np.empty((9, 6))
        b[:, 0::2] = lo
        b[:, 1::2] = lo + 0.05 + 0.2 * rng.random((9, 3))
        boxes.append(b)
    boff = np.arange(0, 9 * 41, 9)
    off, idx = f.box_csr(np.concatenate(boxes), boff)
    off, idx = off.cpu().numpy(), idx.cpu().numpy()
    for t, P in enumerate(pts):
        tr = kdtree.build_kdtree(P, leaf=16, boxsize=1.0)
        o1, i1 = kdtree.box_search_csr(tr, boxes[t])
        o1, i1 = o1.cpu().numpy(), i1.cpu().numpy()
        for r in range(9):
            a = idx[off[9 * t + r]:off[9 * t + r + 1]]
            b = i1[o1[r]:o1[r + 1]]
            np.testing.assert_array_equal(a, b)  # same traversal order too
            m = np.all((P >= boxes[t][r, 0::2]) & (P <= boxes[t][r, 1::2]), axis=1)
            np.testing.assert_array_equal(np.sort(a), np.nonzero(m)[0])


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("sorted_", [False, True])
def test_forest_ball_matches_single_trees(gpu, oracle, periodic, sorted_):
    """Forest ball search: each tree's rows equal the single-tree search of the same
    points (same order), and the oracle's on a few trees.  Enough queries to take
    the leaf-ordered path, warps spanning several trees, and rows past 256 results
    (the warp-per-row fill)."""
    from cosmokdtree_b200 import kdtree, build_forest
    rng = np.random.default_rng(64 + periodic)
    pts = _forest_points(44, 64 + periodic, periodic)
    box = 1.0 if periodic else None
    f = build_forest(pts, leaf=16, boxsize=box)
    qs = _queries_per_tree(pts, rng, 0.3)
    qoff = np.concatenate([[0], np.cumsum([len(q) for q in qs])])
    r = 0.06
    off, idx, dist = (x.cpu().numpy() for x in f.ball_csr(qs, qoff, r, sorted=sorted_))
    assert np.diff(off).max() >= 256
    for t, (P, Q) in enumerate(zip(pts, qs)):
        tr = kdtree.build_kdtree(P, leaf=16, boxsize=box)
        o1, i1, d1 = (x.cpu().numpy() for x in kdtree.ball_search_csr(tr, Q, r, sorted=sorted_))
        rows = slice(qoff[t], qoff[t + 1] + 1)
        np.testing.assert_array_equal(off[rows] - off[qoff[t]], o1)
        lo, hi = off[qoff[t]], off[qoff[t + 1]]
        np.testing.assert_array_equal(idx[lo:hi], i1)
        np.testing.assert_array_equal(dist[lo:hi], d1)
        if t % 11 == 3:
            ot = oracle.OracleTree(P, 16, [1.0] * 3 if periodic else None)
            oo, oi, od = ot.ball_csr(Q, r, sorted=sorted_)
            np.testing.assert_array_equal(o1, oo)
            if sorted_ or not periodic:
                np.testing.assert_array_equal(i1, oi)
                np.testing.assert_array_equal(d1, od)
    f.close()


def test_forest_knn_cuda_graph(gpu):
    import torch
    from cosmokdtree_b200 import build_forest
    rng = np.random.default_rng(63)
    pts = _forest_points(30, 63, True)
    f = build_forest(pts, leaf=16, boxsize=1.0)
    qs = _queries_per_tree(pts, rng, 0.2)
    qoff = torch.tensor(np.concatenate([[0], np.cumsum([len(q) for q in qs])]), device="cuda")
    q_static = torch.from_numpy(np.concatenate(qs)).cuda()
    out = (torch.empty((q_static.shape[0], 8), dtype=torch.float64, device="cuda"),
           torch.empty((q_static.shape[0], 8), dtype=torch.int64, device="cuda"))
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        f.knn_device(q_static, qoff, 8, out=out)  # first call outside capture
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        f.knn_device(q_static, qoff, 8, out=out)
    for trial in range(2):
        qs2 = _queries_per_tree(pts, np.random.default_rng(100 + trial), 0.2)
        q_new = torch.from_numpy(np.concatenate([q[: len(a)] for q, a in zip(qs2, qs)]))
        q_static.copy_(q_new)
        g.replay()
        torch.cuda.synchronize()
        d_ref, i_ref = f.knn(q_new.numpy(), qoff.cpu().numpy(), 8)
        assert torch.equal(out[1], i_ref) and torch.equal(out[0], d_ref)
    del g


def test_forest_errors(gpu):
    import torch
    from cosmokdtree_b200 import kdtree, build_forest, _lib
    pts = [np.random.default_rng(1).random((50, 3)) - 0.5, np.zeros((0, 3))]
    with pytest.raises(AssertionError):
        build_forest(pts, boxsize=1.0)  # empty tree
    f = build_forest([np.random.default_rng(2).random((70, 3)) - 0.5] * 3, boxsize=1.0)
    with pytest.raises(AssertionError):
        f.knn(np.zeros((4, 3)), [0, 2, 4], 3)  # wrong offset count
    with pytest.raises(AssertionError):
        f.knn(np.full((3, 3), 0.7), [0, 1, 2, 3], 3)  # outside the periodic box
    L = _lib.load()
    q = torch.zeros((2, 3), dtype=torch.float64, device="cuda")
    dd = torch.empty((2, 2), dtype=torch.float64, device="cuda")
    ii = torch.empty((2, 2), dtype=torch.int64, device="cuda")
    import ctypes
    st = L.ckd_knn(f.handle, ctypes.c_void_p(q.data_ptr()), 2, 2, 1, ctypes.c_void_p(dd.data_ptr()),
                   ctypes.c_void_p(ii.data_ptr()), None)
    assert st == _lib.CKD_ERR_BAD_ARG and "forest" in _lib.last_error()
    with pytest.raises(AssertionError):
        f.knn(np.zeros((3, 3)), [0, 1, 2, 3], 65)  # k above the forest limit
    d, i = f.knn(np.zeros((3, 3)), [0, 1, 2, 3], 3)  # the library still works
    assert d.shape == (3, 3)
    del kdtree
