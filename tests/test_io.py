"""Point-file reader for the reference's Fortran unformatted layout (CPU) and tree
save/load round trips (GPU)."""
import numpy as np
import pytest


def _write_fortran(path, arrays):
    with open(path, "wb") as f:
        for a in arrays:
            b = np.ascontiguousarray(a).tobytes()
            m = np.array([len(b)], np.int32).tobytes()
            f.write(m + b + m)


def test_read_fortran_points(tmp_path):
    from cosmokdtree_b200.kdtree import read_fortran_points
    rng = np.random.default_rng(0)
    P = rng.random((1000, 3)).astype(np.float32)
    p = tmp_path / "points.dat"
    _write_fortran(p, [np.array([1000], np.int32), P[:, 0], P[:, 1], P[:, 2]])
    np.testing.assert_array_equal(read_fortran_points(str(p)), P)
    bad = tmp_path / "bad.dat"
    _write_fortran(bad, [np.array([1000], np.int32), P[:999, 0]])
    with pytest.raises(ValueError):
        read_fortran_points(str(bad))
    raw = p.read_bytes()
    trunc = tmp_path / "trunc.dat"
    trunc.write_bytes(raw[:-3])
    with pytest.raises(ValueError):
        read_fortran_points(str(trunc))


@pytest.mark.gpu
def test_save_load_tree_and_forest(gpu, tmp_path):
    from cosmokdtree_b200 import kdtree, build_forest
    rng = np.random.default_rng(1)
    P = rng.random((50000, 3)) - 0.5
    Q = rng.random((3000, 3)) - 0.5
    for box in (None, 1.0):
        t = kdtree.build_kdtree(P, leaf=16, boxsize=box)
        path = str(tmp_path / f"tree_{box}.ckd")
        kdtree.save_kdtree(t, path)
        t2 = kdtree.load_kdtree(path)
        assert (t2.n, t2.d, t2.leaf, t2.periodic, t2.n_nodes, t2.depth) == \
            (t.n, t.d, t.leaf, t.periodic, t.n_nodes, t.depth)
        d0, i0 = kdtree.knn_search(t, Q, 12)
        d1, i1 = kdtree.knn_search(t2, Q, 12)
        np.testing.assert_array_equal(i0, i1)
        np.testing.assert_array_equal(d0, d1)
        o0, b0, _ = (x.cpu().numpy() for x in kdtree.ball_search_csr(t, Q, 0.02))
        o1, b1, _ = (x.cpu().numpy() for x in kdtree.ball_search_csr(t2, Q, 0.02))
        np.testing.assert_array_equal(o0, o1)
        np.testing.assert_array_equal(b0, b1)
    f = build_forest([P[:20000], P[20000:]], leaf=16, boxsize=1.0)
    fp = str(tmp_path / "forest.ckd")
    kdtree.save_kdtree(f, fp)
    f2 = kdtree.load_kdtree(fp)
    assert f2.n_trees == 2
    qoff = [0, 1500, 3000]
    a = f.knn(Q, qoff, 8)
    b = f2.knn(Q, qoff, 8)
    assert all(np.array_equal(x.cpu().numpy(), y.cpu().numpy()) for x, y in zip(a, b))
    junk = tmp_path / "junk.ckd"
    junk.write_bytes(b"not a tree at all")
    with pytest.raises(AssertionError):
        kdtree.load_kdtree(str(junk))
