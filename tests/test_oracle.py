"""The CPU oracle against the golden fixtures, brute force, the reference demos'
checks (seeded and asserted) and scipy's cKDTree (third-party cross-check)."""
import numpy as np
import pytest
from hypothesis import given, settings, strategies as st

from conftest import GOLDEN_CASES, load_golden


def _sorted_rows(off, idx):
    return [np.sort(idx[off[i]:off[i + 1]]) for i in range(len(off) - 1)]


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_golden(oracle, name):
    g = load_golden(name)
    t = oracle.OracleTree(g["points"], g["leaf"], g["boxsize"])
    d, i = t.knn(g["queries"], g["k"], sorted=True)
    np.testing.assert_array_equal(i, g["knn_idx"])
    np.testing.assert_array_equal(d, g["knn_dist"])  # bit-exact FP64
    off, bi, bd = t.ball_csr(g["queries"], g["radius"], sorted=True)
    np.testing.assert_array_equal(off, g["ball_off"])
    np.testing.assert_array_equal(bi, g["ball_idx"])
    np.testing.assert_array_equal(bd, g["ball_dist"])
    xo, xi = t.box_csr(g["boxes"])
    np.testing.assert_array_equal(xo, g["box_off"])
    for a, b in zip(_sorted_rows(xo, xi), _sorted_rows(g["box_off"], g["box_idx"])):
        np.testing.assert_array_equal(a, b)


def test_oracle_unsorted_is_permutation(oracle):
    g = load_golden("uniform3d")
    t = oracle.OracleTree(g["points"], g["leaf"], None)
    d, i = t.knn(g["queries"], g["k"], sorted=False)
    for r in range(len(i)):
        assert sorted(i[r]) == sorted(g["knn_idx"][r])
    off, bi, _ = t.ball_csr(g["queries"], g["radius"], sorted=False)
    for a, b in zip(_sorted_rows(off, bi), _sorted_rows(g["ball_off"], g["ball_idx"])):
        np.testing.assert_array_equal(a, b)


def test_reference_periodic_demo_checks(oracle):
    """demos/cosmokdtree/periodic/tree_test.f90:79-139, seeded and asserted
    (n scaled from 1e7 to 2e5): periodic kNN k=100 at (-49.6, 1, 43) against a
    brute-force minimum-image ranking, and the ball r=10 count at (-44.6, 1, 43)."""
    rng = np.random.default_rng(7)
    L = 100.0
    P = (rng.random((200_000, 3)) - 0.5) * L
    t = oracle.OracleTree(P, 16, [L, L, L])
    q = np.array([-49.6, 1.0, 43.0])
    d, i = t.knn(q, 100)
    bd2, bi = oracle.brute_knn(P, q, 100, L)
    np.testing.assert_array_equal(i[0], bi)
    np.testing.assert_array_equal(d[0], np.sqrt(bd2))
    q2 = np.array([-44.6, 1.0, 43.0])
    off, _, _ = t.ball_csr(q2, 10.0)
    assert off[1] == np.count_nonzero(oracle.brute_d2(P, q2, L) <= 100.0)


def test_reference_box_demo_check(oracle):
    """demos/cosmokdtree/box_search/tree_test.f90:70-97 (n scaled to 2e5)."""
    rng = np.random.default_rng(8)
    P = (rng.random((200_000, 3)) - 0.5) * 100.0
    t = oracle.OracleTree(P, 16, None)
    box = np.array([-20., 10., -5., 20., -10., 10.])
    off, idx = t.box_csr(box)
    m = np.all((P >= box[0::2]) & (P <= box[1::2]), axis=1)
    np.testing.assert_array_equal(np.sort(idx), np.nonzero(m)[0])


def test_oracle_tree_invariants(oracle):
    rng = np.random.default_rng(3)
    P = np.concatenate([rng.random((3000, 3)), np.full((50, 3), 0.25),
                        rng.random((200, 3)) * 1e-6 + 0.7])
    t = oracle.OracleTree(P, 8, None)
    e = t.export()
    assert sorted(e["ids"]) == list(range(len(P)))
    for a in range(t.n_nodes):
        s, c = e["start"][a], e["count"][a]
        pts = e["pts"][s:s + c]
        cell = e["cell"][a]
        assert np.all(pts >= cell[0::2]) and np.all(pts <= cell[1::2])
        if e["is_leaf"][a]:
            assert c <= 8
            # stable partition: each leaf holds its points in ascending original id
            assert np.all(np.diff(e["ids"][s:s + c]) > 0)
            continue
        ax, sp = e["axis"][a], e["split"][a]
        L, R = e["left"][a], e["right"][a]
        assert e["count"][L] + e["count"][R] == c and e["count"][L] > 0 and e["count"][R] > 0
        lp = e["pts"][e["start"][L]:e["start"][L] + e["count"][L], ax]
        rp = e["pts"][e["start"][R]:e["start"][R] + e["count"][R], ax]
        assert np.all(lp <= sp) and np.all(rp >= sp)


@settings(max_examples=40, deadline=None)
@given(n=st.integers(1, 300), k=st.integers(1, 40), leaf=st.integers(1, 20),
       periodic=st.booleans(), lattice=st.booleans(), seed=st.integers(0, 2**31 - 1))
def test_oracle_knn_brute_force_property(oracle, n, k, leaf, periodic, lattice, seed):
    rng = np.random.default_rng(seed)
    if lattice:  # many exact ties in distance
        P = rng.integers(-3, 4, (n, 3)).astype(np.float64) / 8.0
    else:
        P = rng.random((n, 3)) - 0.5
    L = 1.0 if periodic else None
    t = oracle.OracleTree(P, leaf, L)
    Q = np.concatenate([P[: min(n, 5)], rng.random((5, 3)) - 0.5])
    d, i = t.knn(Q, k)
    for r in range(len(Q)):
        bd2, bi = oracle.brute_knn(P, Q[r], k, L)
        m = len(bi)
        np.testing.assert_array_equal(i[r, :m], bi)
        np.testing.assert_array_equal(d[r, :m], np.sqrt(bd2))
        assert np.all(i[r, m:] == -2)
        assert np.all(d[r, m:] == np.float64(np.sqrt(np.float64(np.finfo(np.float32).max))))
    off, bidx, _ = t.ball_csr(Q, 0.2)
    for r in range(len(Q)):
        d2 = oracle.brute_d2(P, Q[r], L)
        assert sorted(bidx[off[r]:off[r + 1]]) == sorted(np.nonzero(d2 <= 0.2 * 0.2)[0])


def test_oracle_vs_scipy(oracle):
    cKDTree = pytest.importorskip("scipy.spatial").cKDTree
    rng = np.random.default_rng(4)
    P = rng.random((20000, 3)) - 0.5
    Q = rng.random((500, 3)) - 0.5
    for L in (None, 1.0):
        t = oracle.OracleTree(P, 16, L)
        d, i = t.knn(Q, 12)
        if L is None:
            sd, si = cKDTree(P).query(Q, 12)
        else:  # scipy wants [0, L)
            sd, si = cKDTree(P + 0.5, boxsize=1.0).query(Q + 0.5, 12)
        np.testing.assert_allclose(d, sd, rtol=1e-12, atol=1e-15)
        assert np.mean(i == si) > 0.999  # ids differ only at (near-)ties


def test_oracle_rejects_out_of_box(oracle):
    P = np.array([[0.0, 0.0, 0.0], [0.6, 0.0, 0.0]])
    with pytest.raises(ValueError):
        oracle.OracleTree(P, 16, 1.0)
