"""The learned k-th-distance bound on the GPU: the training kernels' gradient and
the inference kernel against the FP64 CPU reference (oracle/mlp_ref.py), the
features against a NumPy restatement, exactness of the bounded search against
the plain search (every prediction is judged by it), and the work the trained
network saves."""
import ctypes

import numpy as np
import pytest

from oracle import mlp_ref as M

pytestmark = pytest.mark.gpu


def _catalogue(n, seed, periodic=True):
    from cosmokdtree_b200 import synth
    P = synth.clustered_periodic(n, seed, n_clusters=max(8, n // 4096))
    return P if periodic else P * 0.999


@pytest.fixture(scope="module")
def trained(gpu):
    from cosmokdtree_b200 import kdtree
    from cosmokdtree_b200.learned import LearnedBound
    P = _catalogue(200_000, 41)
    t = kdtree.build_kdtree(P, leaf=16, boxsize=1.0)
    rng = np.random.default_rng(42)
    Qtr = np.concatenate([P[rng.integers(0, len(P), 45_000)], rng.random((15_000, 3)) - 0.5])
    lb = LearnedBound(seed=5)
    info = lb.fit(t, Qtr, 32, epochs=25, batch=2048, lr=3e-3, quantile=0.97)
    return t, P, lb, info


def test_gradient_matches_cpu_reference(gpu):
    import torch
    from cosmokdtree_b200 import kdtree
    from cosmokdtree_b200.learned import LearnedBound
    P = _catalogue(30_000, 43)
    t = kdtree.build_kdtree(P, leaf=16, boxsize=1.0)
    Q = _catalogue(3000, 44)
    lb = LearnedBound(seed=9)
    feat = lb.features(t, Q, 16)
    targ = LearnedBound.targets(t, Q, 16)
    g, loss = lb.grad(feat, targ)  # first use sets the normalisation from these samples
    sd = lb.state_dict()
    X, T = feat.cpu().numpy(), targ.cpu().numpy()
    lref, gref = M.loss_and_grad(sd["params"], sd["norm"], X, T)
    assert np.isclose(loss, lref, rtol=1e-4)
    scale = np.abs(gref).max()
    np.testing.assert_allclose(g, gref, rtol=2e-3, atol=1e-4 * scale)
    # one more point after some training: weights no longer at initialisation
    lb.train(feat, targ, epochs=3, batch=512, lr=1e-3)
    g2, loss2 = lb.grad(feat, targ)
    sd2 = lb.state_dict()
    lref2, gref2 = M.loss_and_grad(sd2["params"], sd2["norm"], X, T)
    assert loss2 < loss
    assert np.isclose(loss2, lref2, rtol=1e-4)
    np.testing.assert_allclose(g2, gref2, rtol=2e-3, atol=1e-4 * np.abs(gref2).max())
    # FP32 inference kernel against the FP64 forward pass
    from cosmokdtree_b200 import _lib
    _lib.check(_lib.load().ckd_set_tuning(7, 0))
    try:
        y = lb.predict(feat).cpu().numpy()
    finally:
        _lib.check(_lib.load().ckd_set_tuning(7, 1))
    np.testing.assert_allclose(y, M.predict(sd2["params"], sd2["norm"], X), rtol=0, atol=2e-4)
    del torch


def test_features_match_numpy(gpu):
    from cosmokdtree_b200 import kdtree
    from cosmokdtree_b200.learned import LearnedBound
    rng = np.random.default_rng(45)
    P = _catalogue(20_000, 45, periodic=False)
    t = kdtree.build_kdtree(P, leaf=16)
    Q = rng.random((300, 3)) * 0.9 - 0.45
    lb = LearnedBound(seed=1)
    f = lb.features(t, Q, 24).cpu().numpy()
    e = t.export()
    parent = -np.ones(t.n_nodes, np.int64)
    for a in range(t.n_nodes):
        if e["axis"][a] >= 0:
            parent[e["left"][a]] = a
            parent[e["right"][a]] = a
    e["parent"] = parent
    ref = np.stack([M.features_np(e, q, 24) for q in Q])
    np.testing.assert_allclose(f, ref, rtol=0, atol=2e-4)


@pytest.fixture(params=[0, 3],
                ids=["bounded_lane_compact", "bounded_lane_pair"])
def learned_kernel(request, gpu):
    from cosmokdtree_b200 import _lib
    _lib.check(_lib.load().ckd_set_tuning(4, request.param))
    yield request.param
    _lib.load().ckd_set_tuning(4, 3)


@pytest.mark.parametrize("k", [8, 32])
@pytest.mark.parametrize("margin_shift", [-1.0, 0.0, 3.0])
def test_learned_knn_is_exact(trained, learned_kernel, k, margin_shift):
    from cosmokdtree_b200 import kdtree
    t, P, lb, info = trained
    rng = np.random.default_rng(46)
    Q = np.concatenate([P[rng.integers(0, len(P), 6000)], rng.random((6000, 3)) - 0.5])
    m0 = lb.margin
    try:
        lb.set_margin(m0 + margin_shift)
        d1, i1 = lb.knn(t, Q, k)
        nfb = lb.last_fallback
        d0, i0 = kdtree.knn_search(t, Q, k)
    finally:
        lb.set_margin(m0)
    np.testing.assert_array_equal(i1, i0)
    np.testing.assert_array_equal(d1, d0)
    assert 0 <= nfb <= len(Q)
    if margin_shift <= -1.0:
        assert nfb > 0  # a too-tight bound exercises the rerun path
    # unsorted output is the same set
    d2, i2 = lb.knn(t, Q[:2000], k, sorted=False)
    np.testing.assert_array_equal(np.sort(i2, 1), np.sort(i0[:2000], 1))


def test_learned_knn_periodic_and_plain_trees(gpu):
    from cosmokdtree_b200 import kdtree
    from cosmokdtree_b200.learned import LearnedBound
    rng = np.random.default_rng(47)
    P = rng.random((50_000, 3)) - 0.5
    for box in (None, 1.0):
        t = kdtree.build_kdtree(P, leaf=16, boxsize=box)
        lb = LearnedBound(seed=3)
        lb.fit(t, rng.random((20_000, 3)) - 0.5, [8, 16], epochs=6, batch=1024)
        Q = rng.random((5000, 3)) - 0.5
        for k in (8, 16, 40):
            d1, i1 = lb.knn(t, Q, k)
            d0, i0 = kdtree.knn_search(t, Q, k)
            np.testing.assert_array_equal(i1, i0)
            np.testing.assert_array_equal(d1, d0)


def test_training_converges(trained):
    _, _, _, info = trained
    loss = info["loss"]
    assert loss[-1] < 0.25 * loss[0]
    assert info["holdout_rms_log2"] < 0.6
    assert info["holdout_rerun_rate"] < 0.06


def test_learned_bound_saves_work(trained):
    """What the trained network gains over the plain per-lane search on the same
    queries: fewer node expansions, heap insertions and FP64 distance checks
    (traversal counters), at a small rerun rate."""
    from cosmokdtree_b200 import _lib, kdtree
    t, P, lb, _ = trained
    L = _lib.load()
    rng = np.random.default_rng(48)
    Q = P[rng.integers(0, len(P), 40_000)]

    def stats(fn):
        out = (ctypes.c_int64 * 8)()
        _lib.check(L.ckd_knn_stats(1, None))
        fn()
        _lib.check(L.ckd_knn_stats(0, out))
        return np.array(out[:])

    # per-lane kernels: the plain search against the bounded one
    _lib.check(L.ckd_set_knn_variant(7))
    _lib.check(L.ckd_set_tuning(4, 3))
    try:
        plain = stats(lambda: kdtree.knn_search(t, Q, 32))
        learned = stats(lambda: lb.knn(t, Q, 32))
    finally:
        _lib.check(L.ckd_set_knn_variant(0))
    nfb = lb.last_fallback
    assert nfb < 0.06 * len(Q)
    # counters: 0 node expansions, 2 leaf scans, 5 FP64 evaluations, 6 heap inserts
    assert learned[6] < 0.8 * plain[6], (learned, plain)
    assert learned[0] < 0.9 * plain[0], (learned, plain)
    assert learned[5] < plain[5], (learned, plain)
    # child-pair-record kernels (the defaults): fewer inserts and FP64 evaluations
    _lib.check(L.ckd_set_knn_variant(8))
    try:
        pplain = stats(lambda: kdtree.knn_search(t, Q, 32))
        plearned = stats(lambda: lb.knn(t, Q, 32))
    finally:
        _lib.check(L.ckd_set_knn_variant(0))
    assert plearned[6] < pplain[6], (plearned, pplain)
    assert plearned[5] < pplain[5], (plearned, pplain)


def test_tensor_core_inference_matches_reference(gpu):
    """The tcgen05 inference kernel against the FP64 reference with BF16
    activations, and the learned search through it stays exact."""
    from cosmokdtree_b200 import _lib, kdtree
    from cosmokdtree_b200.learned import LearnedBound
    L = _lib.load()
    P = _catalogue(60_000, 49)
    t = kdtree.build_kdtree(P, leaf=16, boxsize=1.0)
    rng = np.random.default_rng(50)
    lb = LearnedBound(seed=11)
    lb.fit(t, P[rng.integers(0, len(P), 20_000)], [8, 32], epochs=4, batch=1024)
    Q = np.concatenate([P[rng.integers(0, len(P), 3000)], rng.random((333, 3)) - 0.5])
    feat = lb.features(t, Q, 16)
    sd = lb.state_dict()
    X = feat.cpu().numpy()
    _lib.check(L.ckd_set_tuning(7, 0))
    y_simt = lb.predict(feat).cpu().numpy()
    _lib.check(L.ckd_set_tuning(7, 1))
    try:
        y_tc = lb.predict(feat).cpu().numpy()
        ref = M.predict_bf16_activations(sd["params"], sd["norm"], X)
        np.testing.assert_allclose(y_tc, ref, rtol=0, atol=2e-2)
        assert np.median(np.abs(y_tc - ref)) < 1e-3
        assert np.abs(y_tc - y_simt).max() < 0.1  # BF16 activations move predictions slightly
        for k in (8, 32):
            d1, i1 = lb.knn(t, Q, k)
            d0, i0 = kdtree.knn_search(t, Q, k)
            np.testing.assert_array_equal(i1, i0)
            np.testing.assert_array_equal(d1, d0)
    finally:
        _lib.check(L.ckd_set_tuning(7, 1))


def test_learned_host_pipeline_is_exact(trained):
    """Host queries from 2^20 rows on take the chunked pipeline (each chunk a learned
    call with its own reruns); rows equal the plain search's and the rerun count is
    summed over the chunks."""
    from cosmokdtree_b200 import kdtree
    t, P, lb, _ = trained
    rng = np.random.default_rng(77)
    nq = kdtree._PIPE_MIN_ROWS + 321
    Q = np.concatenate([P[rng.integers(0, len(P), nq // 2)],
                        rng.random((nq - nq // 2, 3)) - 0.5])
    ld, li = lb.knn(t, Q, 32)
    assert isinstance(li, np.ndarray) and li.shape == (nq, 32)
    assert 0 <= lb.last_fallback < 0.2 * nq
    pd, pi = kdtree.knn_search(t, Q, 32)
    np.testing.assert_array_equal(li, pi)
    np.testing.assert_array_equal(ld, pd)
