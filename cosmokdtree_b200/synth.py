"""Seeded synthetic catalogues with the shapes of the benchmark configurations.

The reference's own point files (benchmark/examples/points_*.dat / .npy, read by
demos/cosmokdtree/build/inhomogeneous/tree_test.f90:72) are not shipped, so these
generators stand in for them:

* ``uniform``: i.i.d. uniform points in [0, 1)^d (config "plain method, small").
* ``clustered_periodic``: a periodic unit box stored in [-0.5, 0.5)^3; 70% of the
  points in 4096 NFW-like clusters (centres uniform, concentration c ~ U(5, 15),
  virial radius log-uniform in [0.002, 0.02], masses power law dN/dM ~ M^-1.9 on
  [1, 1e4] sampled by inverse CDF, points allotted multinomially by mass, radii from
  the NFW enclosed-mass CDF inverted by bisection, isotropic directions, wrapped
  periodically) plus 30% uniform background.
* ``nfw_cluster``: one NFW-like cluster centred in its own periodic box (batched
  trees configuration); ``forest_catalogue`` draws a whole forest of them (tree
  sizes log-uniform, concentration U(4, 20) per tree) on the GPU.
* ``phase_space``: positions as in ``clustered_periodic`` but non-periodic, with
  velocities per cluster ~ N(v_bulk, sigma^2), sigma ~ U(0.05, 0.3),
  v_bulk ~ N(0, 0.1^2); background velocities N(0, 0.1^2).
"""
from __future__ import annotations

import numpy as np


def uniform(n, d=3, seed=0):
    return np.random.default_rng(seed).random((n, d))


def _nfw_mu(y):
    return np.log1p(y) - y / (1.0 + y)


def nfw_radii(rng, c, iters=40):
    """x = r / r_vir in (0, 1] with enclosed-mass CDF mu(c x) / mu(c), per-point c."""
    u = rng.random(c.shape[0])
    target = u * _nfw_mu(c)
    lo = np.zeros_like(c)
    hi = np.ones_like(c)
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        below = _nfw_mu(c * mid) < target
        lo = np.where(below, mid, lo)
        hi = np.where(below, hi, mid)
    return 0.5 * (lo + hi)


def _directions(rng, m):
    v = rng.standard_normal((m, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v


def _power_law_masses(rng, m, lo=1.0, hi=1e4, slope=-1.9):
    a = 1.0 + slope
    u = rng.random(m)
    return (lo ** a + u * (hi ** a - lo ** a)) ** (1.0 / a)


def clustered_periodic(n, seed=1, n_clusters=4096, frac=0.7, c_range=(5.0, 15.0),
                       rvir_range=(0.002, 0.02), box=1.0, return_labels=False):
    """Clustered catalogue in a periodic box of side ``box`` stored in [-box/2, box/2)."""
    rng = np.random.default_rng(seed)
    centres = (rng.random((n_clusters, 3)) - 0.5) * box
    conc = rng.uniform(*c_range, n_clusters)
    rvir = np.exp(rng.uniform(np.log(rvir_range[0]), np.log(rvir_range[1]), n_clusters)) * box
    mass = _power_law_masses(rng, n_clusters)
    n_cl = int(round(frac * n))
    counts = rng.multinomial(n_cl, mass / mass.sum())
    lab = np.repeat(np.arange(n_clusters), counts)
    x = nfw_radii(rng, conc[lab])
    pos = centres[lab] + (x * rvir[lab])[:, None] * _directions(rng, n_cl)
    pos = np.mod(pos + 0.5 * box, box) - 0.5 * box
    bg = (rng.random((n - n_cl, 3)) - 0.5) * box
    P = np.concatenate([pos, bg])
    labels = np.concatenate([lab, np.full(n - n_cl, -1)])
    perm = rng.permutation(n)
    P = np.ascontiguousarray(P[perm])
    # guard against rounding onto +box/2 by the wrap
    P[P >= 0.5 * box] = -0.5 * box
    if return_labels:
        return P, labels[perm]
    return P


def nfw_cluster(n, seed, c_range=(4.0, 20.0), rvir=0.25, box=1.0):
    """One NFW-like cluster centred in its own periodic box [-box/2, box/2)^3."""
    rng = np.random.default_rng(seed)
    c = np.full(n, rng.uniform(*c_range))
    x = nfw_radii(rng, c)
    pos = (x * rvir * box)[:, None] * _directions(rng, n)
    pos = np.mod(pos + 0.5 * box, box) - 0.5 * box
    pos[pos >= 0.5 * box] = -0.5 * box
    return pos


def phase_space(n, seed=5, dtype=np.float32):
    """6-D (position, velocity) catalogue, non-periodic."""
    P, lab = clustered_periodic(n, seed=seed, return_labels=True)
    rng = np.random.default_rng(seed + 1000)
    ncl = int(lab.max()) + 1
    sigma = rng.uniform(0.05, 0.3, ncl)
    bulk = rng.normal(0.0, 0.1, (ncl, 3))
    V = rng.standard_normal((n, 3))
    inc = lab >= 0
    V[inc] = bulk[lab[inc]] + V[inc] * sigma[lab[inc], None]
    V[~inc] *= 0.1
    return np.ascontiguousarray(np.concatenate([P, V], axis=1).astype(dtype))


def mixed_queries(P, nq, seed, box=1.0):
    """Half drawn from the particle distribution, half uniform in the box."""
    rng = np.random.default_rng(seed)
    h = nq // 2
    q1 = P[rng.integers(0, P.shape[0], h)]
    q2 = (rng.random((nq - h, P.shape[1])) - 0.5) * box
    Q = np.concatenate([q1, q2])
    return np.ascontiguousarray(Q[rng.permutation(nq)])


def forest_catalogue(n_trees, seed=2, n_range=(1e3, 1e6), c_range=(4.0, 20.0), rvir=0.25,
                     box=1.0, device="cuda"):
    """Forest of independent NFW-like clusters, each centred in its own periodic box
    [-box/2, box/2)^3: tree sizes n = floor(10^U(log10 lo, log10 hi)), concentration
    c ~ U(c_range) per tree, radii from the NFW enclosed-mass CDF (bisection),
    isotropic directions.  Generated with torch on ``device`` (hundreds of millions
    of points); returns (points (N, 3) float64 tensor, offsets int64 numpy array)."""
    import torch
    rng = np.random.default_rng(seed)
    lo, hi = np.log10(n_range[0]), np.log10(n_range[1])
    sizes = np.floor(10.0 ** rng.uniform(lo, hi, n_trees)).astype(np.int64)
    conc = rng.uniform(*c_range, n_trees)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    c = torch.repeat_interleave(torch.from_numpy(conc).to(device),
                                torch.from_numpy(sizes).to(device))
    mu = lambda y: torch.log1p(y) - y / (1.0 + y)  # noqa: E731
    target = torch.rand(c.shape[0], generator=g, device=device, dtype=torch.float64) * mu(c)
    a = torch.zeros_like(c)
    b = torch.ones_like(c)
    for _ in range(40):
        m = 0.5 * (a + b)
        below = mu(c * m) < target
        a = torch.where(below, m, a)
        b = torch.where(below, b, m)
    r = 0.5 * (a + b) * rvir * box
    del a, b, target
    v = torch.randn((c.shape[0], 3), generator=g, device=device, dtype=torch.float64)
    v /= torch.linalg.norm(v, dim=1, keepdim=True)
    pos = torch.remainder(r[:, None] * v + 0.5 * box, box) - 0.5 * box
    pos[pos >= 0.5 * box] = -0.5 * box
    return pos.contiguous(), off
