"""The CPU reference of the learned-bound network: its gradient against finite
differences and its BF16 rounding against torch's."""
import numpy as np
import torch

from oracle import mlp_ref as M


def _setup(n=64, seed=0):
    rng = np.random.default_rng(seed)
    w = np.concatenate([rng.standard_normal(M.B3 - 0) * 0.3, [0.1]]).astype(np.float64)
    norm = np.concatenate([rng.standard_normal(M.F), 0.5 + rng.random(M.F), [-7.0, 1.5]])
    X = rng.standard_normal((n, M.F)) * 2 + norm[:M.F]
    T = -7.0 + 1.5 * rng.standard_normal(n)
    return w, norm.astype(np.float32), X.astype(np.float32), T.astype(np.float32)


def test_layout():
    assert M.N_PARAMS == 5057 and M.N_NORM == 26
    assert (M.W1, M.B1, M.W2, M.B2, M.W3, M.B3) == (0, 768, 832, 4928, 4992, 5056)


def test_gradient_matches_finite_differences():
    w, norm, X, T = _setup()
    loss, g = M.loss_and_grad(w, norm, X, T, rounded=False)
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(M.N_PARAMS, 60, replace=False), [M.B3, M.W1, M.W3]])
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (M.loss_and_grad(wp, norm, X, T, rounded=False)[0] -
              M.loss_and_grad(wm, norm, X, T, rounded=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g).max()), (i, fd, g[i])


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(2)
    x = (rng.standard_normal(100000) * 10.0 ** rng.uniform(-6, 6, 100000)).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(M.bf16_round(x), ref)


def test_loss_is_mean_squared_normalised_error():
    w, norm, X, T = _setup(n=10)
    z, _ = M.forward(w, norm, X)
    tn = (T - norm[24]) / norm[25]
    loss, _ = M.loss_and_grad(w, norm, X, T)
    assert np.isclose(loss, np.mean((z - tn) ** 2), rtol=1e-6)
