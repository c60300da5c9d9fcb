"""GPU parity: the CUDA path (libckd.so through the reference-shaped API) against the
golden fixtures and the CPU oracle.  Bar: bit-exact ids, FP64 distances equal to
the last bit (both sides use separately rounded FP64 arithmetic), identical tree
structure, identical sorted order."""
import zlib

import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu


def _rows(off, idx):
    return [idx[off[i]:off[i + 1]] for i in range(len(off) - 1)]


def _np(t):
    return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)


def clustered(rng, n, d=3, periodic=False, dup=0):
    c = rng.random((12, d)) - 0.5
    w = rng.integers(0, 12, n)
    P = c[w] + 0.02 * rng.standard_normal((n, d)) * rng.random((n, 1)) ** 2
    P[: n // 4] = rng.random((n // 4, d)) - 0.5
    if dup:
        P[n // 2: n // 2 + dup] = P[n // 2]
    if periodic:
        P = (P + 0.5) % 1.0 - 0.5
    return P


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_gpu_golden(gpu, oracle, name):
    g = load_golden(name)
    kd = gpu.kdtree
    t = kd.build_kdtree(g["points"], leaf=g["leaf"], boxsize=g["boxsize"])
    d, i = kd.knn_search(t, g["queries"], g["k"], sorted=True)
    np.testing.assert_array_equal(i, g["knn_idx"])
    np.testing.assert_array_equal(d, g["knn_dist"])
    off, bi, bd = (_np(x) for x in kd.ball_search_csr(t, g["queries"], g["radius"], sorted=True))
    np.testing.assert_array_equal(off, g["ball_off"])
    np.testing.assert_array_equal(bi, g["ball_idx"])
    np.testing.assert_array_equal(bd, g["ball_dist"])
    xo, xi = (_np(x) for x in kd.box_search_csr(t, g["boxes"]))
    ot = oracle.OracleTree(g["points"], g["leaf"], g["boxsize"])
    oxo, oxi = ot.box_csr(g["boxes"])
    np.testing.assert_array_equal(xo, oxo)
    np.testing.assert_array_equal(xi, oxi)  # same ids in the same (reference) order
    kd.deallocate_kdtree(t)


STRUCT_CASES = [
    ("uniform3d", 20000, 3, False, 16),
    ("periodic3d", 20000, 3, True, 16),
    ("clustered_dup", 30000, 3, False, 16),
    ("periodic_clustered", 30000, 3, True, 8),
    ("d1", 5000, 1, False, 16),
    ("d2_leaf1", 3000, 2, False, 1),
    ("d6", 20000, 6, False, 32),
    ("d8_periodic", 8000, 8, True, 16),
    ("tiny", 7, 3, False, 16),
    ("root_split", 17, 3, False, 16),
    # odd n: the build's scalar (non-vector, unstaged) paths at every level
    ("uniform3d_odd", 20001, 3, False, 16),
    ("periodic_clustered_odd", 30001, 3, True, 8),
    ("d4_odd", 12345, 4, True, 4),
]


def make_points(name, n, d, periodic, seed=0):
    rng = np.random.default_rng(seed + zlib.crc32(name.encode()) % 1000)  # same data every run
    if "clustered" in name:
        P = clustered(rng, n, d, periodic, dup=200 if "dup" in name else 0)
    elif "lattice" in name:  # many exactly equal distances (ties broken by id)
        P = rng.integers(-8, 8, (n, d)).astype(np.float64) / 16.0
    else:
        P = rng.random((n, d)) - (0.5 if periodic else 0.0)
    return P


@pytest.mark.parametrize("name,n,d,periodic,leaf", STRUCT_CASES)
def test_gpu_structure_matches_oracle(gpu, oracle, name, n, d, periodic, leaf):
    P = make_points(name, n, d, periodic)
    box = 1.0 if periodic else None
    t = gpu.kdtree.build_kdtree(P, leaf=leaf, boxsize=box)
    ot = oracle.OracleTree(P, leaf, box)
    assert t.n_nodes == ot.n_nodes
    g, o = t.export(), ot.export()
    for key in ("axis", "start", "count", "left", "right"):
        np.testing.assert_array_equal(g[key], o[key], err_msg=key)
    internal = g["axis"] >= 0
    np.testing.assert_array_equal(g["split"][internal], o["split"][internal])
    np.testing.assert_array_equal(g["cell"], o["cell"])
    np.testing.assert_array_equal(g["ids"], o["ids"])
    # tight boxes contain their points
    pts = o["pts"]
    for a in np.nonzero(~internal)[0][:500]:
        s, c = g["start"][a], g["count"][a]
        seg = pts[s:s + c]
        np.testing.assert_array_equal(seg.min(0), g["box"][a][0::2])
        np.testing.assert_array_equal(seg.max(0), g["box"][a][1::2])


KNN_CASES = [
    # name, n, d, periodic, leaf, nq, k
    ("uniform3d", 50000, 3, False, 16, 6000, 16),
    ("periodic3d", 50000, 3, True, 16, 6000, 32),
    ("clustered_dup", 40000, 3, False, 16, 5000, 32),
    ("periodic_clustered", 40000, 3, True, 16, 5000, 64),
    ("d6", 30000, 6, False, 32, 3000, 64),
    ("d2", 20000, 2, True, 4, 3000, 7),
    ("uniform3d", 20000, 3, False, 16, 500, 100),
    ("lattice", 30000, 3, False, 16, 3000, 24),
    ("lattice_periodic", 30000, 3, True, 16, 3000, 40),
]


@pytest.fixture(params=[1, 7, 8, 0],
                ids=["fp64", "lane_compact", "lane_compact_pair", "auto"])
def knn_variant(request, gpu):
    """Every kNN kernel of the product (tuning key 0)."""
    from cosmokdtree_b200 import _lib
    L = _lib.load()
    _lib.check(L.ckd_set_knn_variant(request.param))
    yield request.param
    L.ckd_set_knn_variant(0)


@pytest.mark.parametrize("name,n,d,periodic,leaf,nq,k", KNN_CASES)
def test_gpu_knn_matches_oracle(gpu, oracle, knn_variant, name, n, d, periodic, leaf, nq, k):
    P = make_points(name, n, d, periodic)
    rng = np.random.default_rng(99)
    Q = np.concatenate([P[rng.integers(0, n, nq // 2)],
                        rng.random((nq - nq // 2, d)) - (0.5 if periodic else 0.0)])
    box = 1.0 if periodic else None
    t = gpu.kdtree.build_kdtree(P, leaf=leaf, boxsize=box)
    ot = oracle.OracleTree(P, leaf, box)
    od, oi = ot.knn(Q, k)
    gd, gi = gpu.kdtree.knn_search(t, Q, k)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd, od)
    ud, ui = gpu.kdtree.knn_search(t, Q, k, sorted=False)
    np.testing.assert_array_equal(np.sort(ui, 1), np.sort(oi, 1))


def test_gpu_knn_k_greater_than_n(gpu):
    P = np.random.default_rng(1).random((5, 3))
    t = gpu.kdtree.build_kdtree(P)
    d, i = gpu.kdtree.knn_search(t, P[0], 8)
    assert d.shape == (1, 8) and i.shape == (1, 8)
    assert list(i[0, 5:]) == [-2, -2, -2]
    assert np.all(d[0, 5:] == 1.8446743523953730e19)
    assert i[0, 0] == 0 and d[0, 0] == 0.0


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("sorted_", [False, True])
def test_gpu_ball_matches_oracle(gpu, oracle, periodic, sorted_):
    P = make_points("clustered_dup", 40000, 3, periodic)
    rng = np.random.default_rng(5)
    Q = np.concatenate([P[rng.integers(0, len(P), 3000)], rng.random((3000, 3)) - 0.5])
    if not periodic:
        Q = np.clip(Q, -0.7, 0.7)
    box = 1.0 if periodic else None
    t = gpu.kdtree.build_kdtree(P, boxsize=box)
    ot = oracle.OracleTree(P, 16, box)
    r = 0.03
    off, idx, dist = (_np(x) for x in gpu.kdtree.ball_search_csr(t, Q, r, sorted=sorted_))
    ooff, oidx, odist = ot.ball_csr(Q, r, sorted=sorted_)
    np.testing.assert_array_equal(off, ooff)
    if sorted_ or not periodic:
        # sorted rows, and non-periodic traversal order, equal the oracle's exactly
        np.testing.assert_array_equal(idx, oidx)
        np.testing.assert_array_equal(dist, odist)
    else:
        for a, b in zip(_rows(off, idx), _rows(ooff, oidx)):
            np.testing.assert_array_equal(np.sort(a), np.sort(b))
    dl, il = gpu.kdtree.ball_search(t, Q[:10], r, sorted=sorted_)  # list API (kdtree.py:56-79)
    for j in range(10):
        ref = oidx[ooff[j]:ooff[j + 1]]
        if sorted_:
            np.testing.assert_array_equal(il[j], ref)
            np.testing.assert_array_equal(dl[j], odist[ooff[j]:ooff[j + 1]])
        else:
            np.testing.assert_array_equal(np.sort(il[j]), np.sort(ref))


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("sorted_", [False, True])
def test_gpu_ball_heavy_rows_match_oracle(gpu, oracle, periodic, sorted_):
    """Rows of tens of thousands of results: whole subtrees go through the
    emission tasks, sorted rows through the block merge sort."""
    P = make_points("clustered", 120000, 3, periodic, seed=3)
    rng = np.random.default_rng(8)
    Q = np.concatenate([P[rng.integers(0, len(P), 40)], rng.random((10, 3)) - 0.5])
    box = 1.0 if periodic else None
    t = gpu.kdtree.build_kdtree(P, boxsize=box)
    ot = oracle.OracleTree(P, 16, box)
    r = 0.25
    off, idx, dist = (_np(x) for x in gpu.kdtree.ball_search_csr(t, Q, r, sorted=sorted_))
    ooff, oidx, odist = ot.ball_csr(Q, r, sorted=sorted_)
    np.testing.assert_array_equal(off, ooff)
    assert np.diff(off).max() > 8192  # several shared-memory tiles per long row
    if sorted_ or not periodic:
        np.testing.assert_array_equal(idx, oidx)
        np.testing.assert_array_equal(dist, odist)
    else:
        for a, b in zip(_rows(off, idx), _rows(ooff, oidx)):
            np.testing.assert_array_equal(np.sort(a), np.sort(b))


def test_gpu_box_matches_oracle(gpu, oracle):
    P = make_points("clustered_dup", 50000, 3, False)
    rng = np.random.default_rng(6)
    lo = rng.random((1000, 3)) - 0.6
    B = np.empty((1000, 6))
    B[:, 0::2] = lo
    B[:, 1::2] = lo + 0.1 * rng.random((1000, 3))
    B[0] = [-20, 10, -5, 20, -10, 10]
    t = gpu.kdtree.build_kdtree(P)
    ot = oracle.OracleTree(P, 16, None)
    xo, xi = (_np(x) for x in gpu.kdtree.box_search_csr(t, B))
    oo, oi = ot.box_csr(B)
    np.testing.assert_array_equal(xo, oo)
    np.testing.assert_array_equal(xi, oi)
    one = gpu.kdtree.box_search(t, B[1])
    np.testing.assert_array_equal(one, oi[oo[1]:oo[2]])


@pytest.mark.parametrize("warp", [0, 1])
def test_gpu_box_kernels_match_oracle(gpu, oracle, warp):
    """Both box kernels (a lane per box; a warp per box with the level-wise
    frontier and its depth-first fallback for boxes over many leaves), on a
    forest-free tree, small and large batches (the warp kernel serves up to 32768
    boxes per call)."""
    from cosmokdtree_b200 import _lib
    P = make_points("clustered_dup", 60000, 3, True)
    rng = np.random.default_rng(16)
    nb = 40000 if warp == 0 else 3000
    lo = rng.random((nb, 3)) - 0.55
    B = np.empty((nb, 6))
    B[:, 0::2] = lo
    B[:, 1::2] = lo + rng.choice([0.01, 0.05, 0.3], (nb, 1)) * rng.random((nb, 3))
    B[:5] = [-0.5, 0.5, -0.5, 0.5, -0.5, 0.5]  # every leaf: frontier overflow
    t = gpu.kdtree.build_kdtree(P, boxsize=1.0)
    ot = oracle.OracleTree(P, 16, 1.0)
    L = _lib.load()
    _lib.check(L.ckd_set_tuning(8, warp))
    try:
        xo, xi = (_np(x) for x in gpu.kdtree.box_search_csr(t, B))
    finally:
        _lib.check(L.ckd_set_tuning(8, 1))
    oo, oi = ot.box_csr(B)
    np.testing.assert_array_equal(xo, oo)
    np.testing.assert_array_equal(xi, oi)


def test_gpu_box_on_split_plane_quirk(gpu, oracle):
    """A point lying exactly on a split plane is missed when box_hi == split
    (strict descent, cosmokdtree.f90:1296-1300); the GPU reproduces the rule."""
    rng = np.random.default_rng(2)
    P = rng.random((2000, 3))
    ot = oracle.OracleTree(P, 16, None)
    e = ot.export()
    a = int(np.nonzero(e["axis"] >= 0)[0][3])
    ax, sp = int(e["axis"][a]), float(e["split"][a])
    B = np.array([[0.0, 1.0] * 3])
    B[0, 2 * ax + 1] = sp
    t = gpu.kdtree.build_kdtree(P)
    xo, xi = (_np(x) for x in gpu.kdtree.box_search_csr(t, B))
    oo, oi = ot.box_csr(B)
    np.testing.assert_array_equal(xi, oi)


def test_gpu_float32_input(gpu, oracle):
    rng = np.random.default_rng(11)
    P32 = (rng.random((30000, 6)) - 0.5).astype(np.float32)
    P = P32.astype(np.float64)
    t = gpu.kdtree.build_kdtree(P32, leaf=32)
    ot = oracle.OracleTree(P, 32, None)
    Q = P[:2000]
    gd, gi = gpu.kdtree.knn_search(t, Q, 64)
    od, oi = ot.knn(Q, 64)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd, od)


def test_gpu_device_tensor_path(gpu, oracle):
    import torch
    rng = np.random.default_rng(12)
    P = rng.random((20000, 3))
    Pt = torch.from_numpy(P).cuda()
    t = gpu.kdtree.build_kdtree(Pt)
    Qt = Pt[:5000]
    d, i = gpu.kdtree.knn_search(t, Qt, 32)
    assert d.is_cuda and i.is_cuda
    od, oi = oracle.OracleTree(P, 16, None).knn(P[:5000], 32)
    np.testing.assert_array_equal(i.cpu().numpy(), oi)
    np.testing.assert_array_equal(d.cpu().numpy(), od)


def test_gpu_errors_and_recovery(gpu):
    kd = gpu.kdtree
    from cosmokdtree_b200 import _lib
    P = np.random.default_rng(0).random((1000, 3)) - 0.5
    with pytest.raises(_lib.CKDArgumentError):
        kd.build_kdtree(P + 0.6, boxsize=[1.0, 1.0, 1.0])  # outside [-L/2, L/2]
    bad = P.copy()
    bad[10, 1] = np.nan
    with pytest.raises(_lib.CKDArgumentError):
        kd.build_kdtree(bad)
    t = kd.build_kdtree(P, boxsize=[1.0, 1.0, 1.0])
    with pytest.raises(AssertionError):
        kd.knn_search(t, P[:3], 0)
    with pytest.raises(AssertionError):
        kd.ball_search(t, P[:3], -1.0)
    with pytest.raises(AssertionError):
        kd.knn_search(t, np.zeros((3, 2)), 4)
    with pytest.raises(AssertionError):
        kd.knn_search(t, np.full((1, 3), 0.75), 4)  # query outside the periodic box
    with pytest.raises(AssertionError):
        kd.box_search(t, [0, 1, 0, 1])
    d, i = kd.knn_search(t, P[:3], 4)  # the library keeps working after errors
    assert i[0, 0] == 0
    kd.deallocate_kdtree(t)
    with pytest.raises(AssertionError):
        kd.knn_search(t, P[:3], 4)


def test_gpu_periodic_box_wraps(gpu):
    """Opt-in wrapped box search on a periodic tree: every point whose minimum-image
    offset from the box's low corner lies within the box's sides, for boxes that
    cross faces, lie in other images or span whole axes."""
    kd = gpu.kdtree
    rng = np.random.default_rng(71)
    P = rng.random((30000, 3)) - 0.5
    t = kd.build_kdtree(P, leaf=16, boxsize=1.0)
    lo = rng.random((40, 3)) * 2.0 - 1.0          # any image
    side = 0.05 + 0.3 * rng.random((40, 3))
    side[0] = [1.2, 0.1, 0.1]                      # whole first axis
    B = np.empty((40, 6))
    B[:, 0::2] = lo
    B[:, 1::2] = lo + side
    off, idx = (x.cpu().numpy() for x in kd.box_search_periodic_csr(t, B))
    for r in range(40):
        dlt = np.mod(P - lo[r], 1.0)
        inside = np.all((dlt <= side[r]) | (side[r] >= 1.0), axis=1)
        np.testing.assert_array_equal(idx[off[r]:off[r + 1]], np.nonzero(inside)[0])
    # boxes inside the box give the reference's (non-wrapping) answer as a set
    inner = np.array([[-0.2, 0.1, -0.05, 0.2, -0.1, 0.1]])
    o2, i2 = (x.cpu().numpy() for x in kd.box_search_periodic_csr(t, inner))
    np.testing.assert_array_equal(i2, np.sort(kd.box_search(t, inner[0])))
    with pytest.raises(AssertionError):
        kd.box_search_periodic_csr(kd.build_kdtree(P), inner)


@pytest.mark.gpu
def test_gpu_pool_reuse_and_release(gpu):
    """Freed trees return to the library pool; rebuilding from reused memory and
    after handing the cache back to the driver gives identical trees."""
    import torch
    kd = gpu.kdtree
    P = np.random.default_rng(5).random((300_000, 3)) - 0.5
    ref = kd.build_kdtree(P, boxsize=[1.0, 1.0, 1.0]).export()
    for _ in range(2):
        t = kd.build_kdtree(P, boxsize=[1.0, 1.0, 1.0])
        e = t.export()
        kd.deallocate_kdtree(t)
        for key in ref:
            np.testing.assert_array_equal(e[key], ref[key])
    free0 = torch.cuda.mem_get_info()[0]
    kd.release_cached_memory()
    assert torch.cuda.mem_get_info()[0] >= free0
    t = kd.build_kdtree(P, boxsize=[1.0, 1.0, 1.0])
    e = t.export()
    for key in ref:
        np.testing.assert_array_equal(e[key], ref[key])
    d, i = kd.knn_search(t, P[:5], 3)
    assert (i[:, 0] == np.arange(5)).all()


def test_gpu_host_csr_entry_points(gpu, oracle):
    """The host-buffer two-phase ball and box entry points (used by the Fortran
    front end) give the device path's CSR."""
    import ctypes
    from cosmokdtree_b200 import _lib
    L = _lib.load()
    P = make_points("clustered", 30000, 3, True, seed=4)
    rng = np.random.default_rng(21)
    Q = np.ascontiguousarray(np.concatenate([P[:200], rng.random((100, 3)) - 0.5]))
    t = gpu.kdtree.build_kdtree(P, boxsize=1.0)
    ot = oracle.OracleTree(P, 16, 1.0)
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)
    for sorted_ in (0, 1):
        off = np.empty(len(Q) + 1, np.int64)
        _lib.check(L.ckd_ball_count_host(t.handle, vp(Q), len(Q), 0.02, vp(off), None))
        idx = np.empty(max(off[-1], 1), np.int64)
        dist = np.empty(max(off[-1], 1), np.float64)
        _lib.check(L.ckd_ball_fill_host(t.handle, vp(Q), len(Q), 0.02, sorted_, vp(off), vp(idx),
                                        vp(dist), None))
        ooff, oidx, odist = ot.ball_csr(Q, 0.02, sorted=bool(sorted_))
        np.testing.assert_array_equal(off, ooff)
        if sorted_:
            np.testing.assert_array_equal(idx[:off[-1]], oidx)
            np.testing.assert_array_equal(dist[:off[-1]], odist)
        else:
            for a, b in zip(_rows(off, idx), _rows(ooff, oidx)):
                np.testing.assert_array_equal(np.sort(a), np.sort(b))
    lo = rng.random((500, 3)) - 0.55
    B = np.empty((500, 6))
    B[:, 0::2] = lo
    B[:, 1::2] = lo + 0.08 * rng.random((500, 3))
    off = np.empty(len(B) + 1, np.int64)
    _lib.check(L.ckd_box_count_host(t.handle, vp(B), len(B), vp(off), None))
    idx = np.empty(max(off[-1], 1), np.int64)
    _lib.check(L.ckd_box_fill_host(t.handle, vp(B), len(B), vp(off), vp(idx), None))
    oo, oi = ot.box_csr(B)
    np.testing.assert_array_equal(off, oo)
    np.testing.assert_array_equal(idx[:off[-1]], oi)
    empty = np.zeros(1, np.int64)
    _lib.check(L.ckd_box_count_host(t.handle, vp(B), 0, vp(empty), None))
    assert empty[0] == 0


def test_gpu_knn_multi_k(gpu, oracle):
    """One call with a k per query: each row equals the single-k search (and the
    oracle) for its k, padded past its k with the missing-neighbour marker."""
    import torch
    P = make_points("clustered", 40000, 3, True, seed=7)
    rng = np.random.default_rng(31)
    Q = np.concatenate([P[rng.integers(0, len(P), 6000)], rng.random((3000, 3)) - 0.5])
    ks = rng.choice([1, 5, 8, 32, 64, 100], len(Q))
    t = gpu.kdtree.build_kdtree(P, boxsize=1.0)
    d, i = gpu.kdtree.knn_search_multi_k(t, Q, ks)
    assert d.shape == (len(Q), 100) and i.shape == (len(Q), 100)
    ot = oracle.OracleTree(P, 16, 1.0)
    for k in np.unique(ks):
        rows = np.nonzero(ks == k)[0]
        d1, i1 = gpu.kdtree.knn_search(t, Q[rows], int(k))
        np.testing.assert_array_equal(i[rows, :k], i1)
        np.testing.assert_array_equal(d[rows, :k], d1)
        assert (i[rows, k:] == -2).all() and (d[rows, k:] == 1.8446743523953730e19).all()
        od, oi = ot.knn(Q[rows[:200]], int(k))
        np.testing.assert_array_equal(i1[:200], oi)
    dt, it = gpu.kdtree.knn_search_multi_k(t, torch.from_numpy(Q).cuda(),
                                           torch.from_numpy(ks).cuda(), sorted=False)
    np.testing.assert_array_equal(np.sort(it.cpu().numpy(), 1), np.sort(i, 1))
    with pytest.raises(AssertionError):
        gpu.kdtree.knn_search_multi_k(t, Q[:3], [1, 0, 2])


def test_gpu_knn_host_pipeline(gpu):
    """Host queries from 2^20 rows take the chunked path (search and copy-back
    overlapped on two streams); results equal the device path's."""
    import torch
    kd = gpu.kdtree
    rng = np.random.default_rng(41)
    P = rng.random((300_000, 3)) - 0.5
    Q = rng.random(((1 << 20) + 77, 3)) - 0.5
    t = kd.build_kdtree(P, boxsize=1.0)
    d, i = kd.knn_search(t, Q, 8)
    assert isinstance(d, np.ndarray) and d.shape == (len(Q), 8)
    dd, ii = kd.knn_search_batch(t, torch.from_numpy(Q).cuda(), 8)
    np.testing.assert_array_equal(i, ii.cpu().numpy())
    np.testing.assert_array_equal(d, dd.cpu().numpy())
    with pytest.raises(AssertionError):
        kd.knn_search(t, np.full((1 << 20, 3), 0.75), 4)  # outside the periodic box
