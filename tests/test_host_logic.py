"""Host-side logic that needs no GPU: the split of a box into in-box pieces used by
the opt-in periodic-wrapping box search."""
import numpy as np

from cosmokdtree_b200.kdtree import _wrap_pieces


def _covered(x, pieces):
    return any(a <= x <= b for a, b in pieces)


def test_wrap_pieces_cover_the_interval_modulo_L():
    rng = np.random.default_rng(12)
    for L in (1.0, 2.5):
        for _ in range(400):
            lo = rng.uniform(-2 * L, 2 * L)
            hi = lo + rng.choice([rng.uniform(0, 0.2 * L), rng.uniform(0, L), rng.uniform(L, 2 * L)])
            pieces = _wrap_pieces(lo, hi, L)
            assert 1 <= len(pieces) <= 2
            for a, b in pieces:
                assert -L / 2 <= a <= b <= L / 2
            total = sum(b - a for a, b in pieces)
            assert abs(total - min(hi - lo, L)) <= 1e-9 * L
            xs = rng.uniform(-L / 2, L / 2, 200)
            for x in xs:
                # x is in the periodic interval iff some image x + jL lies in [lo, hi]
                j = np.ceil((lo - x) / L)
                inside = x + j * L <= hi or hi - lo >= L
                on_edge = any(abs(x + i * L - e) <= 1e-9 for i in range(-4, 5) for e in (lo, hi))
                if not on_edge:  # images within rounding of an end are ambiguous
                    assert _covered(x, pieces) == inside, (lo, hi, x, pieces)


def test_wrap_pieces_inside_box_unchanged():
    assert _wrap_pieces(-0.2, 0.3, 1.0) == [(-0.2, 0.3)]
    assert _wrap_pieces(0.4, 0.7, 1.0)[0][0] == 0.4
    assert _wrap_pieces(-3.0, 5.0, 1.0) == [(-0.5, 0.5)]
