"""Learned k-th-neighbour distance bound for exact kNN search.

A 12 -> 64 -> 64 -> 1 ReLU network (BF16 weights, FP32 arithmetic; kernels in
``csrc/mlp.cu``) predicts ``log2`` of each query's k-th-neighbour distance from
features of the query's leaf and its ancestors (occupancy and cell size of the
leaf, its sibling, grandparent and great-grandparent, the leaf's tight-box size,
depth, ``log2 k`` and the query's offset in the leaf cell).  ``knn`` seeds every
query's heap with the bound ``2**(y + margin)`` so the traversal prunes from the
root; a query with fewer than k points inside its bound is searched again
without a bound, so results are exactly those of ``kdtree.knn_search``.  The
margin sets the trade-off between tight bounds and reruns; ``fit`` calibrates it
as a quantile of the prediction residuals on held-out samples.

Training runs on the GPU with the project's own forward, backward and Adam
kernels, on exact k-th distances produced by the plain search.  The reference
has no counterpart; it only changes how fast ``knn_search`` runs.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._lib import MLP_FEATURES, MLP_NORM, MLP_PARAMS, CKDArgumentError, check
from .kdtree import (_PIPE_MIN_ROWS, KDTree, _check_k, _knn_host_pipelined, _ptr, _queries,
                     _stream, _to_host, knn_search_batch)

__all__ = ["LearnedBound"]

_MIN_LOG2 = -60.0  # floor of log2 distance targets (duplicate points give d_k = 0)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class LearnedBound:
    """A trainable k-th-distance predictor living on one GPU."""

    def __init__(self, seed: int = 0, device: int | None = None):
        self.device = torch.cuda.current_device() if device is None else int(device)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(_lib.load().ckd_mlp_create(ctypes.c_uint64(seed & (2**64 - 1)), ctypes.byref(h)))
        self._h = h
        self.last_fallback = None  # fallback count of the last knn call
        self.history: list[float] = []

    # ------------------------------------------------------------ handle
    @property
    def handle(self):
        if self._h is None:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "network has been freed")
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.load().ckd_mlp_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ state
    def state_dict(self) -> dict:
        params = np.empty(MLP_PARAMS, np.float32)
        norm = np.empty(MLP_NORM, np.float32)
        margin = ctypes.c_float()
        steps = ctypes.c_int64()
        with torch.cuda.device(self.device):
            check(_lib.load().ckd_mlp_get(self.handle, _fptr(params), _fptr(norm),
                                          ctypes.byref(margin), ctypes.byref(steps)))
        return {"params": params, "norm": norm, "margin": float(margin.value),
                "steps": int(steps.value)}

    def load_state_dict(self, sd: dict) -> None:
        params = None if sd.get("params") is None else \
            np.ascontiguousarray(sd["params"], dtype=np.float32)
        norm = None if sd.get("norm") is None else np.ascontiguousarray(sd["norm"], dtype=np.float32)
        if params is not None and params.shape != (MLP_PARAMS,):
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, f"params must have {MLP_PARAMS} entries")
        if norm is not None and norm.shape != (MLP_NORM,):
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, f"norm must have {MLP_NORM} entries")
        with torch.cuda.device(self.device):
            check(_lib.load().ckd_mlp_set(self.handle, None if params is None else _fptr(params),
                                          None if norm is None else _fptr(norm),
                                          float(sd.get("margin", self.margin))))

    def save(self, path: str) -> None:
        sd = self.state_dict()
        np.savez(path, params=sd["params"], norm=sd["norm"], margin=sd["margin"],
                 steps=sd["steps"])

    @classmethod
    def load(cls, path: str, device: int | None = None) -> "LearnedBound":
        z = np.load(path)
        lb = cls(device=device)
        lb.load_state_dict({"params": z["params"], "norm": z["norm"], "margin": float(z["margin"])})
        return lb

    @property
    def margin(self) -> float:
        m = ctypes.c_float()
        check(_lib.load().ckd_mlp_get(self.handle, None, None, ctypes.byref(m), None))
        return float(m.value)

    def set_margin(self, margin: float) -> None:
        with torch.cuda.device(self.device):
            check(_lib.load().ckd_mlp_set(self.handle, None, None, float(margin)))

    # ------------------------------------------------------------ pieces
    def features(self, tree: KDTree, target, k) -> torch.Tensor:
        """(nq, 12) float32 CUDA tensor of the network's inputs."""
        k = _check_k(k)
        with torch.cuda.device(tree.device):
            q, _ = _queries(tree, target)
            f = torch.empty((q.shape[0], MLP_FEATURES), dtype=torch.float32, device=q.device)
            check(_lib.load().ckd_mlp_features(tree.handle, _ptr(q), q.shape[0], k, _ptr(f),
                                               _stream()))
        return f

    @staticmethod
    def targets(tree: KDTree, target, k) -> torch.Tensor:
        """log2 of the exact k-th-neighbour distance of every query (plain search)."""
        dist, _ = knn_search_batch(tree, target, k, sorted=True)
        dk = dist[:, -1].to(torch.float64)
        return torch.log2(dk.clamp_min(2.0 ** _MIN_LOG2)).to(torch.float32)

    def grad(self, feat: torch.Tensor, target: torch.Tensor) -> tuple[np.ndarray, float]:
        """Gradient of the mean squared error over all samples (FP32, host)."""
        feat, target = self._samples(feat, target)
        g = np.empty(MLP_PARAMS, np.float32)
        loss = ctypes.c_float()
        with torch.cuda.device(self.device):
            check(_lib.load().ckd_mlp_grad(self.handle, _ptr(feat), _ptr(target), feat.shape[0],
                                           _fptr(g), ctypes.byref(loss), _stream()))
        return g, float(loss.value)

    def train(self, feat: torch.Tensor, target: torch.Tensor, epochs: int = 1, batch: int = 4096,
              lr: float = 2e-3, seed: int = 0, lr_final: float | None = None) -> list[float]:
        """Adam over shuffled mini-batches; per-epoch cosine step size from ``lr`` to
        ``lr_final`` (default lr / 20).  Returns the mean loss of every epoch."""
        feat, target = self._samples(feat, target)
        n = feat.shape[0]
        lr_final = lr / 20.0 if lr_final is None else lr_final
        gen = torch.Generator(device=feat.device)
        gen.manual_seed(seed)
        out = []
        L = _lib.load()
        with torch.cuda.device(self.device):
            for e in range(epochs):
                perm = torch.randperm(n, device=feat.device, generator=gen)
                f, t = feat[perm].contiguous(), target[perm].contiguous()
                c = 0.5 * (1.0 + math.cos(math.pi * e / max(1, epochs - 1))) if epochs > 1 else 1.0
                lr_e = lr_final + (lr - lr_final) * c
                loss = (ctypes.c_float * 1)()
                check(L.ckd_mlp_train(self.handle, _ptr(f), _ptr(t), n, int(batch), 1,
                                      float(lr_e), ctypes.cast(loss, ctypes.c_void_p), _stream()))
                out.append(float(loss[0]))
        self.history.extend(out)
        return out

    def predict(self, feat: torch.Tensor) -> torch.Tensor:
        """Predicted log2 k-th distance (without the margin), float32 CUDA tensor."""
        feat = feat.to(device=f"cuda:{self.device}", dtype=torch.float32).contiguous()
        y = torch.empty(feat.shape[0], dtype=torch.float32, device=feat.device)
        with torch.cuda.device(self.device):
            check(_lib.load().ckd_mlp_predict(self.handle, _ptr(feat), feat.shape[0], _ptr(y),
                                              _stream()))
        return y

    def _samples(self, feat, target):
        dev = f"cuda:{self.device}"
        feat = feat.to(device=dev, dtype=torch.float32).contiguous()
        target = target.to(device=dev, dtype=torch.float32).contiguous().reshape(-1)
        if feat.dim() != 2 or feat.shape[1] != MLP_FEATURES or feat.shape[0] != target.shape[0]:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG,
                                   "features must be (n, 12) with one target per row")
        return feat, target

    # ------------------------------------------------------------ workflow
    def fit(self, tree: KDTree, queries, k, epochs: int = 30, batch: int = 4096, lr: float = 3e-3,
            quantile: float = 0.97, holdout: float = 0.1, seed: int = 0) -> dict:
        """Train on exact k-th distances of ``queries`` (plain search) and calibrate
        the margin so that a fraction ``quantile`` of held-out queries needs no
        rerun.  ``k`` is an int or a sequence of ints (the queries are split evenly
        among them).  Returns the loss history, margin and held-out rerun rate."""
        ks = [_check_k(k)] if np.ndim(k) == 0 else [_check_k(int(x)) for x in k]
        with torch.cuda.device(tree.device):
            q, _ = _queries(tree, queries)
            parts = torch.tensor_split(q, len(ks))
            feats, targs = [], []
            for kk, qq in zip(ks, parts):
                if qq.shape[0] == 0:
                    continue
                feats.append(self.features(tree, qq, kk))
                targs.append(self.targets(tree, qq, kk))
            feat = torch.cat(feats)
            targ = torch.cat(targs)
            n = feat.shape[0]
            gen = torch.Generator(device=feat.device)
            gen.manual_seed(seed + 1)
            perm = torch.randperm(n, device=feat.device, generator=gen)
            n_hold = max(1, int(round(holdout * n))) if n > 10 else 0
            hold, tr = perm[:n_hold], perm[n_hold:]
            hist = self.train(feat[tr], targ[tr], epochs=epochs, batch=batch, lr=lr, seed=seed)
            cal = hold if n_hold > 0 else tr
            resid = (targ[cal] - self.predict(feat[cal])).double()
            margin = float(torch.quantile(resid, quantile).item()) if resid.numel() > 1 else 1.0
            self.set_margin(margin)
            miss = float((resid > margin).double().mean().item())
            rms = float(resid.pow(2).mean().sqrt().item())
        return {"loss": hist, "margin": margin, "holdout_rerun_rate": miss,
                "holdout_rms_log2": rms, "n_train": int(tr.numel()), "n_holdout": int(n_hold)}

    def knn(self, tree: KDTree, target, k, sorted=True):
        """Exact kNN with the learned bound: (dist, idx) like ``knn_search``
        (numpy for host input, CUDA tensors for CUDA input).  The number of
        queries that needed the unbounded rerun is left in ``last_fallback``."""
        if not (isinstance(target, torch.Tensor) and target.is_cuda):
            k = _check_k(k)
            nq = np.shape(target)[0] if np.ndim(target) == 2 else 1
            if nq >= _PIPE_MIN_ROWS:
                if tree.device != self.device:
                    raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG,
                                           "tree and network are on different devices")
                L = _lib.load()
                nfb_total = [0]

                def search(qc, n, db, ib, st):  # one chunk of the pipeline
                    nfb = ctypes.c_int64()
                    check(L.ckd_knn_learned(tree.handle, self.handle, _ptr(qc), n, k,
                                            int(bool(sorted)), _ptr(db), _ptr(ib),
                                            ctypes.byref(nfb), st))
                    nfb_total[0] += int(nfb.value)

                # 4 chunks: each learned call pays an ordering pass, a radius pass
                # and a readback of its rerun count
                with torch.cuda.device(tree.device):
                    out = _knn_host_pipelined(tree, target, k, sorted, search=search, chunks=4)
                self.last_fallback = nfb_total[0]
                return out
        dist, idx = self.knn_batch(tree, target, k, sorted)
        if isinstance(target, torch.Tensor) and target.is_cuda:
            return dist, idx
        with torch.cuda.device(tree.device):
            return _to_host(dist), _to_host(idx)

    def knn_multi_k(self, tree: KDTree, target, ks, sorted=True):
        """Exact kNN with a k per target row and the learned bound, in one call:
        (dist, idx) of shape (ntar, max(ks)) like ``kdtree.knn_search_multi_k``
        (slots past a row's own k hold id -2); the reruns are counted in
        ``last_fallback``.  numpy for host input, CUDA tensors for CUDA input."""
        if tree.device != self.device:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "tree and network are on different devices")
        with torch.cuda.device(tree.device):
            q, _ = _queries(tree, target)
            nq = q.shape[0]
            kt = torch.as_tensor(np.asarray(ks) if not isinstance(ks, torch.Tensor) else ks)
            if kt.dim() != 1 or kt.shape[0] != nq:
                raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "ks must hold one k per target row")
            if kt.dtype.is_floating_point or kt.dtype == torch.bool:
                raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "k must be an integer")
            kt = kt.to(device=q.device, dtype=torch.int32).contiguous()
            kmax = int(kt.max().item()) if nq > 0 else 1
            if nq > 0 and int(kt.min().item()) < 1:
                raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "k must be a positive integer")
            dist = torch.empty((nq, kmax), dtype=torch.float64, device=q.device)
            idx = torch.empty((nq, kmax), dtype=torch.int64, device=q.device)
            nfb = ctypes.c_int64()
            if nq > 0:
                check(_lib.load().ckd_knn_learned_multi_k(
                    tree.handle, self.handle, _ptr(q), nq, _ptr(kt), kmax, int(bool(sorted)),
                    _ptr(dist), _ptr(idx), ctypes.byref(nfb), _stream()))
            self.last_fallback = int(nfb.value)
            if isinstance(target, torch.Tensor) and target.is_cuda:
                return dist, idx
            return _to_host(dist), _to_host(idx)

    def knn_batch(self, tree: KDTree, target, k, sorted=True):
        """As ``knn`` with CUDA-tensor results."""
        k = _check_k(k)
        if tree.device != self.device:
            raise CKDArgumentError(_lib.CKD_ERR_BAD_ARG, "tree and network are on different devices")
        with torch.cuda.device(tree.device):
            q, _ = _queries(tree, target)
            nq = q.shape[0]
            dist = torch.empty((nq, k), dtype=torch.float64, device=q.device)
            idx = torch.empty((nq, k), dtype=torch.int64, device=q.device)
            nfb = ctypes.c_int64()
            check(_lib.load().ckd_knn_learned(tree.handle, self.handle, _ptr(q), nq, k,
                                              int(bool(sorted)), _ptr(dist), _ptr(idx),
                                              ctypes.byref(nfb), _stream()))
            self.last_fallback = int(nfb.value)
        return dist, idx
