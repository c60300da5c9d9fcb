"""Parity at the sizes of the benchmark configurations, against the CPU oracle.

Each test builds the configuration's catalogue with the same seeded generators the
benchmark uses (cosmokdtree_b200/synth.py) and compares the GPU results with the
oracle's restatement of the reference (src/cosmokdtree.f90:504-540 kNN, :1015-1072
ball, :1220-1253 box): ids exactly, distances to the last bit, CSR rows in the
reference's order.  Where the oracle would take minutes for every row, a seeded
random sample of rows is compared; the GPU still computes every row.

  C1  2^20 uniform, 10^5 queries: kNN k=16 sorted, ball r=0.01 sorted, 10^3 boxes
      of side 0.02 -- every row.
  C2  2^24 clustered periodic self-queries: kNN k=32 on 50k sampled rows of the
      full search, ball counts at half the mean spacing on 5k rows, the sorted CSR
      fill on 1k rows and the unsorted fill (as sets) on 200.
  C3  200 NFW trees (the forest workload's generator): kNN k=8 of 10% of each
      tree's points and 64 boxes per tree, every 10th tree against its own oracle.
  C4  2^22 clustered periodic, mixed queries (half particles, half uniform), k per
      query in {8, 32, 64} in one call, and the learned-bound search per k.
  C5  2^22 6-D phase space, float32 input, leaf 32, k=64.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_gpu_config_c1_uniform_2p20_every_row(gpu, oracle):
    kd = gpu.kdtree
    rng = np.random.default_rng(0)
    P = rng.random((1 << 20, 3))
    Q = rng.random((100_000, 3))
    cen = rng.random((1000, 3))
    B = np.empty((1000, 6))
    B[:, 0::2] = cen - 0.01
    B[:, 1::2] = cen + 0.01
    t = kd.build_kdtree(P, leaf=16)
    ot = oracle.OracleTree(P, 16, None)
    d, i = kd.knn_search(t, Q, 16, sorted=True)
    od, oi = ot.knn(Q, 16)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(d, od)
    off, bi, bd = (x.cpu().numpy() for x in kd.ball_search_csr(t, Q, 0.01, sorted=True))
    ooff, obi, obd = ot.ball_csr(Q, 0.01, sorted=True)
    np.testing.assert_array_equal(off, ooff)
    np.testing.assert_array_equal(bi, obi)
    np.testing.assert_array_equal(bd, obd)
    xo, xi = (x.cpu().numpy() for x in kd.box_search_csr(t, B))
    oxo, oxi = ot.box_csr(B)
    np.testing.assert_array_equal(xo, oxo)
    np.testing.assert_array_equal(xi, oxi)
    kd.deallocate_kdtree(t)


def test_gpu_config_c2_clustered_2p24_sampled(gpu, oracle):
    import torch
    from cosmokdtree_b200 import synth
    kd = gpu.kdtree
    n, k = 1 << 24, 32
    P = synth.clustered_periodic(n, seed=1)
    Pd = torch.from_numpy(P).cuda()
    t = kd.build_kdtree(Pd, leaf=16, boxsize=1.0)
    ot = oracle.OracleTree(P, 16, [1.0, 1.0, 1.0])
    d, i = kd.knn_search_batch(t, Pd, k, sorted=True)  # every point queried
    rng = np.random.default_rng(17)
    sel = np.sort(rng.choice(n, 50_000, replace=False))
    seld = torch.from_numpy(sel).cuda()
    od, oi = ot.knn(P[sel], k)
    np.testing.assert_array_equal(i[seld].cpu().numpy(), oi)
    np.testing.assert_array_equal(d[seld].cpu().numpy(), od)
    del d, i
    r = 0.5 * n ** (-1.0 / 3.0)
    # counts (CSR phase 1) on 5k rows, the unsorted fill (reference order) on 1k
    s5 = sel[:5000]
    import ctypes
    from cosmokdtree_b200 import _lib
    L = _lib.load()
    Qs = torch.from_numpy(P[s5]).cuda()
    cnt = torch.empty(len(s5), dtype=torch.int64, device="cuda")
    _lib.check(L.ckd_ball_count(t.handle, ctypes.c_void_p(Qs.data_ptr()), len(s5), r,
                                ctypes.c_void_p(cnt.data_ptr()),
                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    ooff, _, _ = ot.ball_csr(P[s5], r)
    np.testing.assert_array_equal(cnt.cpu().numpy(), np.diff(ooff))
    # sorted rows equal the oracle's exactly; unsorted periodic rows hold the same
    # points in another traversal order (the reference visits the near side of
    # each split first, cosmokdtree.f90:1143-1212; the GPU fill goes left first)
    s1 = sel[5000:6000]
    off, bi, bd = (x.cpu().numpy() for x in kd.ball_search_csr(t, P[s1], r, sorted=True))
    ooff, obi, obd = ot.ball_csr(P[s1], r, sorted=True)
    np.testing.assert_array_equal(off, ooff)
    np.testing.assert_array_equal(bi, obi)
    np.testing.assert_array_equal(bd, obd)
    s2 = sel[6000:6200]
    off, bi, _ = (x.cpu().numpy() for x in kd.ball_search_csr(t, P[s2], r, sorted=False))
    ooff, obi, _ = ot.ball_csr(P[s2], r, sorted=False)
    np.testing.assert_array_equal(off, ooff)
    for j in range(len(s2)):
        np.testing.assert_array_equal(np.sort(bi[off[j]:off[j + 1]]),
                                      np.sort(obi[ooff[j]:ooff[j + 1]]))
    kd.deallocate_kdtree(t)


def test_gpu_config_c3_forest_200_trees(gpu, oracle):
    import torch
    from cosmokdtree_b200 import build_forest, synth
    Pd, off = synth.forest_catalogue(200, seed=2)
    sizes = np.diff(off)
    f = build_forest(Pd, off, leaf=16, boxsize=1.0)
    rng = np.random.default_rng(12)
    qsz = np.maximum(1, sizes // 10)
    qidx = np.concatenate([o + rng.integers(0, m, q) for o, m, q in zip(off[:-1], sizes, qsz)])
    qoff = np.concatenate([[0], np.cumsum(qsz)]).astype(np.int64)
    Q = Pd[torch.from_numpy(qidx).cuda()].contiguous()
    d, i = f.knn_device(Q, torch.from_numpy(qoff).cuda(), 8)
    d, i = d.cpu().numpy(), i.cpu().numpy()
    boxes = np.empty((200 * 64, 6))
    lo = rng.random((200 * 64, 3)) - 0.5
    boxes[:, 0::2] = lo - 0.025
    boxes[:, 1::2] = lo + 0.025
    boff = np.arange(0, 200 * 64 + 1, 64, dtype=np.int64)
    xo, xi = (x.cpu().numpy() for x in f.box_csr(boxes, boff))
    Ph = Pd.cpu().numpy()
    for tr in range(0, 200, 10):
        Pt = Ph[off[tr]:off[tr + 1]]
        ot = oracle.OracleTree(Pt, 16, [1.0, 1.0, 1.0])
        qs = slice(qoff[tr], qoff[tr + 1])
        od, oi = ot.knn(Q[qs].cpu().numpy(), 8)
        np.testing.assert_array_equal(i[qs], oi)
        np.testing.assert_array_equal(d[qs], od)
        oxo, oxi = ot.box_csr(boxes[tr * 64:(tr + 1) * 64])
        a, b = xo[tr * 64], xo[(tr + 1) * 64]
        np.testing.assert_array_equal(xo[tr * 64:(tr + 1) * 64 + 1] - a, oxo)
        np.testing.assert_array_equal(xi[a:b], oxi)
    f.close()


def test_gpu_config_c4_mixed_k_and_learned(gpu, oracle):
    import torch
    from cosmokdtree_b200 import synth
    from cosmokdtree_b200.learned import LearnedBound
    kd = gpu.kdtree
    n, nq = 1 << 22, 200_000
    P = synth.clustered_periodic(n, seed=1)
    Q = synth.mixed_queries(P, nq, seed=4)
    rng = np.random.default_rng(8)
    ks = rng.choice([8, 32, 64], nq).astype(np.int32)
    t = kd.build_kdtree(torch.from_numpy(P).cuda(), leaf=16, boxsize=1.0)
    ot = oracle.OracleTree(P, 16, [1.0, 1.0, 1.0])
    d, i = kd.knn_search_multi_k(t, Q, ks)  # host input: numpy results
    sel = rng.choice(nq, 6000, replace=False)
    for kk in (8, 32, 64):
        rows = sel[ks[sel] == kk]
        od, oi = ot.knn(Q[rows], kk)
        np.testing.assert_array_equal(i[rows, :kk], oi)
        np.testing.assert_array_equal(d[rows, :kk], od)
        assert np.all(i[rows, kk:] == -2)
    # the learned-bound search, trained on a separate smaller catalogue
    Ptr = synth.clustered_periodic(1 << 20, seed=3)
    ttr = kd.build_kdtree(torch.from_numpy(Ptr).cuda(), leaf=16, boxsize=1.0)
    lb = LearnedBound(seed=0)
    lb.fit(ttr, synth.mixed_queries(Ptr, 60_000, seed=5), [8, 32, 64], epochs=4, batch=4096)
    # the whole mixed batch in one learned-bound call equals the plain mixed-k call
    md, mi = lb.knn_multi_k(t, Q, ks)
    np.testing.assert_array_equal(mi, i)
    np.testing.assert_array_equal(md, d)
    assert 0 <= lb.last_fallback < nq
    for kk in (8, 32, 64):
        rows = np.nonzero(ks == kk)[0]
        ld, li = lb.knn(t, Q[rows], kk)
        pd_, pi = kd.knn_search(t, Q[rows], kk)
        np.testing.assert_array_equal(li, pi)
        np.testing.assert_array_equal(ld, pd_)
        sub = rows[:2000]
        od, oi = ot.knn(Q[sub], kk)
        np.testing.assert_array_equal(li[:2000], oi)
        np.testing.assert_array_equal(ld[:2000], od)
    lb.close()
    kd.deallocate_kdtree(ttr)
    kd.deallocate_kdtree(t)


def test_gpu_config_c5_phase_space_6d(gpu, oracle):
    import torch
    from cosmokdtree_b200 import synth
    kd = gpu.kdtree
    n = 1 << 22
    P = synth.phase_space(n, seed=5, dtype=np.float32)
    t = kd.build_kdtree(torch.from_numpy(P).cuda(), leaf=32)
    P64 = P.astype(np.float64)
    ot = oracle.OracleTree(P64, 32, None)
    rng = np.random.default_rng(7)
    Q = P64[rng.integers(0, n, 100_000)]
    d, i = kd.knn_search(t, Q, 64)
    sel = rng.choice(len(Q), 4000, replace=False)
    od, oi = ot.knn(Q[sel], 64)
    np.testing.assert_array_equal(i[sel], oi)
    np.testing.assert_array_equal(d[sel], od)
    kd.deallocate_kdtree(t)
