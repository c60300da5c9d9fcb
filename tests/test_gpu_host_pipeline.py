"""Host-array kNN at sizes that take the chunked pipeline (queries staged through
pinned buffers chunk by chunk, results copied back while later chunks are
searched): rows equal the device-array path, the ragged last chunk included, and
an out-of-range query of a periodic tree still raises."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_gpu_host_pipeline_matches_device_path(gpu):
    import torch
    kd = gpu.kdtree
    rng = np.random.default_rng(31)
    P = rng.random((1 << 17, 3)) - 0.5
    nq = kd._PIPE_MIN_ROWS + 12345  # a ragged last chunk
    Q = rng.random((nq, 3)) - 0.5
    for box in (None, [1.0, 1.0, 1.0]):
        t = kd.build_kdtree(P, leaf=16, boxsize=box)
        hd, hi = kd.knn_search(t, Q, 6)
        assert isinstance(hd, np.ndarray) and hd.shape == (nq, 6)
        dd, di = kd.knn_search(t, torch.from_numpy(Q).cuda(), 6)
        np.testing.assert_array_equal(hi, di.cpu().numpy())
        np.testing.assert_array_equal(hd, dd.cpu().numpy())
        t.close()


def test_gpu_host_pipeline_rejects_out_of_box_queries(gpu):
    kd = gpu.kdtree
    rng = np.random.default_rng(32)
    P = rng.random((1 << 14, 3)) - 0.5
    t = kd.build_kdtree(P, leaf=16, boxsize=[1.0, 1.0, 1.0])
    Q = rng.random((kd._PIPE_MIN_ROWS + 7, 3)) - 0.5
    Q[kd._PIPE_MIN_ROWS + 3, 1] = 0.75  # in the last chunk
    with pytest.raises(gpu.kdtree.CKDArgumentError):
        kd.knn_search(t, Q, 4)
    Q[kd._PIPE_MIN_ROWS + 3, 1] = 0.25
    Q[5, 0] = np.nan  # in the first chunk
    with pytest.raises(gpu.kdtree.CKDArgumentError):
        kd.knn_search(t, Q, 4)
    # the tree is still usable
    Q[5, 0] = 0.0
    d, i = kd.knn_search(t, Q[:1000], 4)
    assert (i >= 0).all()
    t.close()


def test_gpu_c_abi_host_pipeline(gpu):
    """ckd_knn_host from 2^20 queries on runs chunked with the copy-back overlapped:
    pageable (numpy) and pinned output buffers both give the device path's rows."""
    import ctypes

    import torch
    from cosmokdtree_b200 import _lib
    kd = gpu.kdtree
    L = _lib.load()
    rng = np.random.default_rng(33)
    P = rng.random((1 << 16, 3)) - 0.5
    t = kd.build_kdtree(P, leaf=16, boxsize=[1.0, 1.0, 1.0])
    nq, k = (1 << 20) + 777, 5
    Q = np.ascontiguousarray(rng.random((nq, 3)) - 0.5)
    dd, di = kd.knn_search(t, torch.from_numpy(Q).cuda(), k)
    dd, di = dd.cpu().numpy(), di.cpu().numpy()
    vp = ctypes.c_void_p
    hd = np.empty((nq, k))
    hi = np.empty((nq, k), dtype=np.int64)
    _lib.check(L.ckd_knn_host(t.handle, vp(Q.ctypes.data), nq, k, 1, vp(hd.ctypes.data),
                              vp(hi.ctypes.data), None))
    np.testing.assert_array_equal(hi, di)
    np.testing.assert_array_equal(hd, dd)
    pdist = torch.empty((nq, k), dtype=torch.float64, pin_memory=True)
    pidx = torch.empty((nq, k), dtype=torch.int64, pin_memory=True)
    _lib.check(L.ckd_knn_host(t.handle, vp(Q.ctypes.data), nq, k, 1, vp(pdist.data_ptr()),
                              vp(pidx.data_ptr()), None))
    np.testing.assert_array_equal(pidx.numpy(), di)
    np.testing.assert_array_equal(pdist.numpy(), dd)
    t.close()
