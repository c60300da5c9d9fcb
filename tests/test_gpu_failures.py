"""Failure paths driven from the host, each followed by a working call.

The reference stops the whole process on these conditions (``STOP`` at
src/cosmokdtree.f90:161, :170 and :190, src/cosmokdtree2py.f90:58 and :276); here
every failure is a status code, the call returns what it took from the device
pool, and the library keeps working.  Nothing here makes a GPU fault or hang: the
depth failure is a host-side level cap reached by a degenerate input, and the
allocation failure comes from a cap on the library's own pool.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MIB = 1 << 20


def _pool_used():
    import torch
    from cosmokdtree_b200 import _lib
    L = _lib.load()
    torch.cuda.synchronize()
    used, res = ctypes.c_int64(), ctypes.c_int64()
    _lib.check(L.ckd_pool_usage(ctypes.byref(used), ctypes.byref(res)))
    return used.value


def test_gpu_depth_cap_reported(gpu, oracle):
    """9000 copies of one point with leaf 1: every sliding-midpoint split peels one
    point off (cosmokdtree.f90:372-410), so the tree would be 8999 levels deep,
    past the build's 8192-level cap.  The build fails with CKD_ERR_DEPTH, returns
    its scratch, and the next build and search are exact."""
    from cosmokdtree_b200 import _lib
    kd = gpu.kdtree
    used0 = _pool_used()
    P = np.full((9000, 3), 0.125)
    with pytest.raises(_lib.CKDError) as ei:
        kd.build_kdtree(P, leaf=1)
    assert ei.value.status == _lib.CKD_ERR_DEPTH
    assert "8192" in str(ei.value)
    assert _pool_used() == used0, "the failed build kept pool memory"
    # fewer copies stay within the cap and give the lowest ids first
    P2 = np.full((300, 3), 0.125)
    t = kd.build_kdtree(P2, leaf=1)
    d, i = kd.knn_search(t, P2[:4], 5)
    np.testing.assert_array_equal(i, np.tile(np.arange(5), (4, 1)))
    np.testing.assert_array_equal(d, np.zeros((4, 5)))
    kd.deallocate_kdtree(t)
    # an ordinary tree afterwards
    rng = np.random.default_rng(5)
    P3 = rng.random((20000, 3))
    t = kd.build_kdtree(P3)
    ot = oracle.OracleTree(P3, 16)
    d, i = kd.knn_search(t, P3[:500], 8)
    od, oi = ot.knn(P3[:500], 8)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(d, od)
    kd.deallocate_kdtree(t)


def test_gpu_allocation_failure_capped_pool(gpu, oracle):
    """With the pool capped just above the tree's own memory, the searches' scratch
    cannot be allocated: kNN, ball and box searches and a build fail with
    CKD_ERR_OOM (MemoryError), the pool's in-use bytes return to the tree's, and
    with the cap lifted the same calls are exact."""
    from cosmokdtree_b200 import _lib
    kd = gpu.kdtree
    L = _lib.load()
    rng = np.random.default_rng(11)
    P = rng.random((200000, 3)) - 0.5
    Q = rng.random((300000, 3)) - 0.5
    t = kd.build_kdtree(P, leaf=16, boxsize=1.0)
    used0 = _pool_used()
    cap_mib = (used0 + MIB - 1) // MIB + 1
    try:
        _lib.check(L.ckd_set_tuning(9, int(cap_mib)))
        with pytest.raises(MemoryError):
            kd.knn_search(t, Q, 16)
        assert _pool_used() == used0, "kNN kept pool memory after failing"
        with pytest.raises(MemoryError):
            kd.ball_search_csr(t, Q, 0.01)
        assert _pool_used() == used0, "ball search kept pool memory after failing"
        with pytest.raises(MemoryError):
            kd.build_kdtree(P, leaf=16, boxsize=1.0)
        assert _pool_used() == used0, "the failed build kept pool memory"
    finally:
        _lib.check(L.ckd_set_tuning(9, 0))
    ot = oracle.OracleTree(P, 16, [1.0, 1.0, 1.0])
    d, i = kd.knn_search(t, Q[:2000], 16)
    od, oi = ot.knn(Q[:2000], 16)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(d, od)
    off, bi, bd = (x.cpu().numpy() for x in kd.ball_search_csr(t, Q[:2000], 0.01, sorted=True))
    ooff, obi, obd = ot.ball_csr(Q[:2000], 0.01, sorted=True)
    np.testing.assert_array_equal(off, ooff)
    np.testing.assert_array_equal(bi, obi)
    kd.deallocate_kdtree(t)
    assert _pool_used() <= used0


def test_gpu_pool_cap_rejects_negative(gpu):
    from cosmokdtree_b200 import _lib
    L = _lib.load()
    assert L.ckd_set_tuning(9, -1) == _lib.CKD_ERR_BAD_ARG
