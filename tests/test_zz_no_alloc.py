"""ckd_knn_noalloc: the kNN entry point that allocates no device memory.

Callers that cannot allocate during a search (memory reserved up front by the
host application, or loops that cannot afford an allocation's synchronisation)
use it instead of ckd_knn.  It must return exactly what ckd_knn returns.  The
test calls both through the C ABI on the same tree and queries, twice in a row
(the shared scratch array keeps the previous call's contents, so the second call
checks that nothing stale leaks into its result), and checks the documented size
limit.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


# "far": coordinates near 1e18, beyond the range where the FP32 screen is used,
# so the entry point takes its FP64 packet kernel instead of the per-lane one
@pytest.mark.parametrize("case", ["open", "periodic", "far"])
def test_knn_noalloc_matches_knn(gpu, oracle, case):
    import torch
    from cosmokdtree_b200 import _lib, kdtree
    L = _lib.load()
    rng = np.random.default_rng(31)
    n = 60000
    P = rng.random((n, 3)) - 0.5
    P[:20000] = P[:20000] * 0.05  # a dense core
    box = [1.0, 1.0, 1.0] if case == "periodic" else None
    shift, scale = (1e18, 1e17) if case == "far" else (0.0, 1.0)
    P = shift + scale * P
    tree = kdtree.build_kdtree(P, leaf=16, boxsize=box)
    ot = oracle.OracleTree(P, 16, box)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, (nq, k) in enumerate([(20000, 32), (7000, 16)]):
        Q = np.concatenate([P[rng.integers(0, n, nq // 2)],
                            shift + scale * (rng.random((nq - nq // 2, 3)) - 0.5)])
        Qd = torch.from_numpy(Q).cuda()
        d_ref = torch.empty((nq, k), dtype=torch.float64, device="cuda")
        i_ref = torch.empty((nq, k), dtype=torch.int64, device="cuda")
        d_na = torch.full((nq, k), -1.0, dtype=torch.float64, device="cuda")
        i_na = torch.full((nq, k), -7, dtype=torch.int64, device="cuda")
        _lib.check(L.ckd_knn(tree.handle, _p(Qd), nq, k, 1, _p(d_ref), _p(i_ref), stream))
        _lib.check(L.ckd_knn_noalloc(tree.handle, _p(Qd), nq, k, 1, _p(d_na), _p(i_na), stream))
        torch.cuda.synchronize()
        assert torch.equal(i_na, i_ref), f"ids differ on call {call}"
        assert torch.equal(d_na, d_ref), f"distances differ on call {call}"
        # and both equal the CPU oracle (ids exactly, distances to the last bit)
        sel = rng.integers(0, nq, 2000)
        od, oi = ot.knn(Q[sel], k)
        np.testing.assert_array_equal(i_na.cpu().numpy()[sel], oi)
        np.testing.assert_array_equal(d_na.cpu().numpy()[sel], od)
    # the documented limit is enforced with a clear error
    big = 2097152 + 1
    st = L.ckd_knn_noalloc(tree.handle, _p(Qd), big, 8, 1, _p(d_na), _p(i_na), stream)
    assert st == _lib.CKD_ERR_BAD_ARG and "2097152" in _lib.last_error()
    tree.close()
