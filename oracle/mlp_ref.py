"""CPU reference of the learned-bound network (test infrastructure only).

FP64 restatement of the forward pass and of the gradient of the training loss
of ``cosmokdtree_b200/csrc/mlp.cu`` (k_mlp_forward / k_mlp_grad), used to check
the GPU training kernels.  The network has no counterpart in the reference
implementation; this file defines its mathematics independently of the CUDA code:

  xh = (x - mu) * inv_sigma                       (FP32, as the kernels do)
  h1 = relu(W1 xh + b1),  h2 = relu(W2 h1 + b2),  z = W3 . h2 + b3
  loss = mean_s (z_s - (t_s - t_mu) / t_sigma)^2

The forward pass uses the BF16-rounded weights (round to nearest even); the
gradient is taken with respect to the weights at those rounded values.
"""
from __future__ import annotations

import numpy as np

F, H = 12, 64
W1, B1 = 0, H * F
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
N_PARAMS = B3 + 1
N_NORM = 2 * F + 2


def bf16_round(x) -> np.ndarray:
    """FP32 -> BF16 -> FP32 with round-to-nearest-even (finite inputs)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return (w[W1:B1].reshape(H, F), w[B1:W2], w[W2:B2].reshape(H, H), w[B2:W3], w[W3:B3],
            w[B3])


def normalise(norm, X, T=None):
    norm = np.asarray(norm, dtype=np.float32)
    mu, isg = norm[:F], norm[F:2 * F]
    xh = ((np.asarray(X, np.float32) - mu) * isg).astype(np.float64)
    if T is None:
        return xh, None
    tn = ((np.asarray(T, np.float32) - norm[2 * F]) / norm[2 * F + 1]).astype(np.float64)
    return xh, tn


def forward(w, norm, X, rounded=True):
    """Normalised network output z for every row of X, and the activations."""
    wr = bf16_round(w) if rounded else np.asarray(w, np.float64)
    w1, b1, w2, b2, w3, b3 = unpack(wr)
    xh, _ = normalise(norm, X)
    a1 = xh @ w1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ w2.T + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ w3 + b3
    return z, (xh, a1, h1, a2, h2)


def predict_bf16_activations(w, norm, X):
    """Prediction with BF16 inputs to both hidden layers' products (the tensor-core
    inference path): standardised features and first-layer activations rounded to
    BF16, products accumulated exactly, biases / ReLU / output layer in FP64."""
    norm = np.asarray(norm, dtype=np.float32)
    w1, b1, w2, b2, w3, b3 = unpack(bf16_round(w))
    xh = bf16_round(((np.asarray(X, np.float32) - norm[:F]) * norm[F:2 * F]).astype(np.float32))
    h1 = np.maximum(xh.astype(np.float64) @ w1.T + b1, 0.0)
    h1b = bf16_round(h1.astype(np.float32)).astype(np.float64)
    h2 = np.maximum(h1b @ w2.T + b2, 0.0)
    z = h2 @ w3 + b3
    return float(norm[2 * F]) + float(norm[2 * F + 1]) * z


def predict(w, norm, X):
    """log2 k-th distance prediction y = t_mu + t_sigma * z (FP64)."""
    norm = np.asarray(norm, dtype=np.float32)
    z, _ = forward(w, norm, X)
    return float(norm[2 * F]) + float(norm[2 * F + 1]) * z


def loss_and_grad(w, norm, X, T, rounded=True):
    """(loss, gradient[N_PARAMS]) in FP64 at the BF16-rounded weights (or at the
    weights themselves with rounded=False)."""
    wr = bf16_round(w) if rounded else np.asarray(w, np.float64)
    w1, b1, w2, b2, w3, b3 = unpack(wr)
    z, (xh, a1, h1, a2, h2) = forward(w, norm, X, rounded)
    _, tn = normalise(norm, X, T)
    n = len(z)
    e = z - tn
    loss = float(np.mean(e * e))
    dz = 2.0 * e / n
    g = np.zeros(N_PARAMS)
    g[W3:B3] = h2.T @ dz
    g[B3] = dz.sum()
    d2 = np.outer(dz, w3) * (a2 > 0)
    g[W2:B2] = (d2.T @ h1).reshape(-1)
    g[B2:W3] = d2.sum(0)
    d1 = (d2 @ w2) * (a1 > 0)
    g[W1:B1] = (d1.T @ xh).reshape(-1)
    g[B1:W2] = d1.sum(0)
    return loss, g


def features_np(export: dict, q: np.ndarray, k: int) -> np.ndarray:
    """Features of one query from an exported tree (preorder arrays of
    ``KDTree.export`` / ``OracleTree.export`` plus a 'parent' array), following the
    definition in csrc/mlp.cu (leaf_features)."""
    axis, split, left, right = export["axis"], export["split"], export["left"], export["right"]
    count, cell, box, parent = export["count"], export["cell"], export["box"], export["parent"]
    node, depth = 0, 0
    while axis[node] >= 0:
        node = left[node] if q[axis[node]] < split[node] else right[node]
        depth += 1

    def mls(b, a):
        w = (b[a, 1::2] - b[a, 0::2]).astype(np.float32)
        return np.float32(np.mean(np.log2(np.maximum(w, np.float32(1e-30)))))

    par = parent[node] if parent[node] >= 0 else node
    sib = (right[par] if left[par] == node else left[par]) if parent[node] >= 0 else node
    gp = parent[par] if parent[par] >= 0 else par
    ggp = parent[gp] if parent[gp] >= 0 else gp
    f = np.empty(F, np.float32)
    f[0] = np.log2(max(count[node], 1))
    f[1] = mls(cell, node)
    f[2] = max(mls(box, node), f[1] - 20)
    f[3] = np.log2(max(count[sib], 1))
    f[4] = mls(cell, sib)
    f[5] = np.log2(max(count[gp], 1))
    f[6] = mls(cell, gp)
    f[7] = np.log2(max(count[ggp], 1))
    f[8] = mls(cell, ggp)
    f[9] = depth
    f[10] = np.log2(k)
    lo, hi = cell[node, 0::2], cell[node, 1::2]
    w = hi - lo
    u = np.where(w > 0, (q - 0.5 * (lo + hi)) / np.where(w > 0, w, 1), 0).astype(np.float32)
    f[11] = 0.5 * np.log2(np.float32(np.sum(u * u)) + np.float32(9.5367431640625e-07))
    return f
