"""The persistent forest launch (ForestPlan / ckd_forest_plan_*): a whole forest
built and its kNN queries answered by one launch over a device work queue.

Results must equal the level-synchronous forest build + forest kNN (which the
other forest tests tie to single trees and to the oracle) row for row, also when
the launch is captured in a CUDA graph and replayed, and the built forest must
answer box searches like the ordinary one.  Failures come from the host: a point
outside the periodic box, NaN, too small a node capacity, and a withheld work
item (ckd_set_tuning key 11) that the bounded queue wait turns into
CKD_ERR_TIMEOUT; after each the plan runs again exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _forest_points(rng, n_trees, d, periodic, lo=30, hi=40000):
    sizes = np.floor(10 ** rng.uniform(np.log10(lo), np.log10(hi), n_trees)).astype(np.int64)
    sizes[:3] = [1, 16, 17]  # a one-point tree, a single leaf, one split
    parts = []
    for m in sizes:
        c = rng.random(d) - 0.5
        x = c + 0.05 * rng.standard_normal((m, d)) * rng.uniform(0.2, 2.0)
        if periodic:
            x = np.mod(x + 0.5, 1.0) - 0.5
        parts.append(x)
    P = np.concatenate(parts)
    if periodic:
        P[P >= 0.5] = -0.5
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    return P, off


def _queries(rng, P, off, frac=0.1):
    sizes = np.diff(off)
    qsz = np.maximum(0, sizes // int(1 / frac))
    qsz[5] = 0  # a tree without queries
    qidx = np.concatenate([o + rng.integers(0, max(m, 1), q) for o, m, q in
                           zip(off[:-1], sizes, qsz)]).astype(np.int64)
    qoff = np.concatenate([[0], np.cumsum(qsz)]).astype(np.int64)
    return P[qidx], qoff


@pytest.mark.parametrize("d,periodic,k", [(3, True, 8), (3, False, 32), (2, True, 16),
                                          (6, False, 64)])
def test_gpu_forest_plan_matches_forest(gpu, d, periodic, k):
    import torch
    from cosmokdtree_b200 import ForestPlan, build_forest
    rng = np.random.default_rng(40 + d + k)
    P, off = _forest_points(rng, 60, d, periodic)
    Q, qoff = _queries(rng, P, off)
    box = 1.0 if periodic else None
    Pd, Qd = torch.from_numpy(P).cuda(), torch.from_numpy(Q).cuda()
    f = build_forest(Pd, off, leaf=16, boxsize=box)
    rd, ri = f.knn_device(Qd, torch.from_numpy(qoff).cuda(), k)
    plan = ForestPlan(Pd, off, Qd, qoff, k, leaf=16, boxsize=box)
    plan.run()
    plan.check()
    assert torch.equal(plan.idx, ri)
    assert torch.equal(plan.dist, rd)
    pf = plan.forest()
    assert pf.n_leaves == f.n_leaves and pf.n_nodes == f.n_nodes and pf.depth == f.depth
    # the built forest answers box searches like the ordinary one
    B = np.empty((60 * 8, 2 * d))
    lo = rng.random((60 * 8, d)) - 0.5
    B[:, 0::2], B[:, 1::2] = lo - 0.08, lo + 0.08
    boff = np.arange(0, 60 * 8 + 1, 8, dtype=np.int64)
    xo, xi = f.box_csr(B, boff)
    yo, yi = pf.box_csr(B, boff)
    assert torch.equal(xo, yo) and torch.equal(xi, yi)
    # a second run over the same buffers
    plan.dist.fill_(-1.0)
    plan.idx.fill_(-7)
    plan.run()
    plan.check()
    assert torch.equal(plan.idx, ri) and torch.equal(plan.dist, rd)
    plan.close()
    f.close()


def test_gpu_forest_plan_graph_replay(gpu, oracle):
    import torch
    from cosmokdtree_b200 import ForestPlan
    rng = np.random.default_rng(77)
    P, off = _forest_points(rng, 120, 3, True, lo=100, hi=60000)
    Q, qoff = _queries(rng, P, off)
    Pd, Qd = torch.from_numpy(P).cuda(), torch.from_numpy(Q).cuda()
    plan = ForestPlan(Pd, off, Qd, qoff, 8, leaf=16, boxsize=1.0, queries_per_block=64)
    plan.run()  # the first, uncaptured run sets the kernel attributes
    plan.check()
    ref_i, ref_d = plan.idx.clone(), plan.dist.clone()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            plan.run()
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(2):
        plan.idx.fill_(-7)
        g.replay()
        plan.check()
        assert torch.equal(plan.idx, ref_i) and torch.equal(plan.dist, ref_d)
    del g
    # against the oracle, tree by tree (every 15th)
    for t in range(0, 120, 15):
        Pt = P[off[t]:off[t + 1]]
        qs = slice(qoff[t], qoff[t + 1])
        if qoff[t + 1] == qoff[t]:
            continue
        ot = oracle.OracleTree(Pt, 16, [1.0, 1.0, 1.0])
        od, oi = ot.knn(Q[qs], 8)
        np.testing.assert_array_equal(ref_i[qs].cpu().numpy(), oi)
        np.testing.assert_array_equal(ref_d[qs].cpu().numpy(), od)
    plan.close()


def test_gpu_forest_plan_failures_from_the_host(gpu):
    import torch
    from cosmokdtree_b200 import ForestPlan, _lib
    L = _lib.load()
    rng = np.random.default_rng(5)
    P, off = _forest_points(rng, 40, 3, True)
    Q, qoff = _queries(rng, P, off)
    Pd, Qd = torch.from_numpy(P).cuda(), torch.from_numpy(Q).cuda()
    plan = ForestPlan(Pd, off, Qd, qoff, 8, boxsize=1.0)
    plan.run()
    plan.check()
    ref_i = plan.idx.clone()
    # a work item the host never pushes: the queue cannot drain, the bounded wait
    # of the idle CTAs ends the launch with CKD_ERR_TIMEOUT
    try:
        _lib.check(L.ckd_set_tuning(10, 300))
        _lib.check(L.ckd_set_tuning(11, 1))
        plan.run()
        with pytest.raises(_lib.CKDTimeout):
            plan.check()
    finally:
        _lib.check(L.ckd_set_tuning(11, 0))
        _lib.check(L.ckd_set_tuning(10, 20000))
    plan.run()
    plan.check()
    assert torch.equal(plan.idx, ref_i)
    # a point outside the periodic box, then NaN: argument errors, then a clean run
    saved = Pd[7].clone()
    Pd[7, 0] = 0.75
    plan.run()
    with pytest.raises(_lib.CKDArgumentError):
        plan.check()
    Pd[7, 0] = float("nan")
    plan.run()
    with pytest.raises(_lib.CKDArgumentError):
        plan.check()
    Pd[7] = saved
    plan.run()
    plan.check()
    assert torch.equal(plan.idx, ref_i)
    plan.close()
    # too small a node capacity is reported, a default plan works
    small = ForestPlan(Pd, off, Qd, qoff, 8, boxsize=1.0, node_factor=0.002)
    small.run()
    with pytest.raises(MemoryError):
        small.check()
    small.close()
    with pytest.raises(AssertionError):
        ForestPlan(Pd, off, Qd, qoff, 65, boxsize=1.0)  # k > 64


def test_gpu_forest_plan_autotuned_equals_default(gpu, tmp_path):
    """The autotuner times the persistent launch over queries per work item, checks
    every candidate's rows against the first, caches the winner; the tuned plan's
    results equal the default plan's."""
    import torch
    from cosmokdtree_b200 import ForestPlan
    from cosmokdtree_b200.autotune import Autotuner
    rng = np.random.default_rng(9)
    P, off = _forest_points(rng, 50, 3, True)
    Q, qoff = _queries(rng, P, off)
    Pd, Qd = torch.from_numpy(P).cuda(), torch.from_numpy(Q).cuda()
    tuner = Autotuner(cache_path=str(tmp_path / "tune.json"))
    cfg = tuner.tune_forest_plan(Pd, off, Qd, qoff, 8, boxsize=1.0, reps=1,
                                 grid={"queries_per_block": (32, 128, 512)})
    assert cfg["queries_per_block"] in (32, 128, 512) and not cfg["cached"]
    again = Autotuner(cache_path=str(tmp_path / "tune.json")).tune_forest_plan(
        Pd, off, Qd, qoff, 8, boxsize=1.0)
    assert again["cached"] and again["queries_per_block"] == cfg["queries_per_block"]
    tuned = ForestPlan(Pd, off, Qd, qoff, 8, leaf=cfg["leaf"], boxsize=1.0,
                       queries_per_block=cfg["queries_per_block"])
    default = ForestPlan(Pd, off, Qd, qoff, 8, boxsize=1.0)
    for p in (tuned, default):
        p.run()
        p.check()
    assert torch.equal(tuned.idx, default.idx) and torch.equal(tuned.dist, default.dist)
    tuned.close()
    default.close()
