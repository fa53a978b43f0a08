"""Learned sample-count predictor: geometry features of a block pair -> log2 of the sample
count the plain adaptive method needs, from an 8 -> 64 -> 64 -> 1 GELU MLP whose forward,
backward and Adam kernels are this library's own (csrc/mlp.cu, through the C ABI).

Features (fixed list; wavelengths lambda = 2 pi / k):
  0 log2 m                       (test group size)
  1 log2 n                       (source group size)
  2 test group diameter / lambda (bounding sphere of the basis centres)
  3 source group diameter / lambda
  4 centre distance / lambda
  5 angular extent (d_t + d_s) / (2 dist)
  6 -log10 tol
  7 k d_t d_s / (4 dist)         (electrical aperture product, a Fresnel-number-like term)

The label of a block (see train_predictor.py) is the smallest sample count of a fixed grid
at which the plain method's randomized estimate meets tol / safety.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "predictor_weights.npz")
FEATURES = ("log2_m", "log2_n", "diam_t_lambda", "diam_s_lambda", "dist_lambda",
            "angular_extent", "neg_log10_tol", "aperture_product")


def features(part, k: float, tol: float) -> np.ndarray:
    """(B, 8) float64 feature matrix of the far blocks of a partition."""
    lam = 2 * np.pi / k
    sz = part.sizes().astype(np.float64)
    m = sz[part.gt]
    n = sz[part.gs]
    dt = part.extents[part.gt]
    ds = part.extents[part.gs]
    dist = np.linalg.norm(part.centres[part.gt] - part.centres[part.gs], axis=1)
    f = np.stack([np.log2(m), np.log2(n), dt / lam, ds / lam, dist / lam,
                  (dt + ds) / (2 * dist), np.full_like(m, -np.log10(tol)),
                  k * dt * ds / (4 * dist)], axis=1)
    return f


class Predictor:
    def __init__(self, params=None, mean=None, std=None, margin: float = 1.0):
        L = _lib.lib()
        self.nparam = L.pskel_mlp_num_params()
        if params is None:
            params = init_params(0)
        self.params = np.asarray(params, dtype=np.float32)
        assert self.params.size == self.nparam
        self.mean = np.zeros(8) if mean is None else np.asarray(mean, dtype=np.float64)
        self.std = np.ones(8) if std is None else np.asarray(std, dtype=np.float64)
        self.margin = margin

    # --------------------------------------------------------------- persistence
    def save(self, path=WEIGHTS, **meta):
        np.savez(path, params=self.params, mean=self.mean, std=self.std, margin=self.margin,
                 features=np.array(FEATURES), **meta)

    @staticmethod
    def load(path=WEIGHTS) -> "Predictor":
        d = np.load(path)
        return Predictor(d["params"], d["mean"], d["std"], float(d["margin"]))

    # --------------------------------------------------------------- GPU inference
    def _std(self, f):
        return ((f - self.mean) / self.std).astype(np.float32)

    def predict_log2(self, f: np.ndarray) -> np.ndarray:
        """log2 sample count for each feature row, computed on the GPU."""
        import torch
        x = torch.from_numpy(np.ascontiguousarray(self._std(f))).cuda()
        p = torch.from_numpy(self.params).cuda()
        y = torch.empty(len(f), dtype=torch.float32, device="cuda")
        _lib.check(_lib.lib().pskel_mlp_forward(ctypes.c_void_p(p.data_ptr()),
                                                ctypes.c_void_p(x.data_ptr()), len(f),
                                                ctypes.c_void_p(y.data_ptr()), None))
        return y.cpu().numpy().astype(np.float64)

    def sample_counts(self, part, k: float, tol: float) -> np.ndarray:
        """First-round sample count of every block (before the engine's oversampling)."""
        y = self.predict_log2(features(part, k, tol))
        r = np.ceil(self.margin * np.exp2(y)).astype(np.int64)
        D = np.minimum(part.sizes()[part.gt], part.sizes()[part.gs])
        return np.clip(r, 1, D).astype(np.int32)

    # --------------------------------------------------------------- GPU training
    def fit(self, f: np.ndarray, y: np.ndarray, steps: int = 3000, batch: int = 4096,
            lr: float = 3e-3, seed: int = 0, log_every: int = 500):
        """Mean-squared-error fit of log2 sample counts with the library's Adam kernel."""
        import torch
        L = _lib.lib()
        self.mean = f.mean(axis=0)
        self.std = f.std(axis=0) + 1e-6
        X = torch.from_numpy(self._std(f)).cuda()
        Y = torch.from_numpy(np.asarray(y, dtype=np.float32)).cuda()
        p = torch.from_numpy(self.params.copy()).cuda()
        g = torch.zeros_like(p)
        m = torch.zeros_like(p)
        v = torch.zeros_like(p)
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        gen = torch.Generator(device="cuda").manual_seed(seed)
        vp = lambda t: ctypes.c_void_p(t.data_ptr())
        hist = []
        n = len(f)
        for t in range(1, steps + 1):
            idx = torch.randint(0, n, (min(batch, n),), device="cuda", generator=gen)
            xb = X[idx].contiguous()
            yb = Y[idx].contiguous()
            _lib.check(L.pskel_mlp_grad(vp(p), vp(xb), vp(yb), len(idx), vp(g), vp(loss), None))
            lr_t = lr * 0.5 * (1 + np.cos(np.pi * t / steps))
            _lib.check(L.pskel_mlp_adam(vp(p), vp(g), vp(m), vp(v), t, lr_t, 0.9, 0.999, 1e-8, None))
            if t % log_every == 0 or t == steps:
                hist.append((t, float(loss.item()) / len(idx)))
        self.params = p.cpu().numpy()
        return hist


def init_params(seed: int) -> np.ndarray:
    """He-style random init of the parameter vector (layout of csrc/mlp.cu)."""
    rng = np.random.default_rng(seed)
    parts = [rng.standard_normal((64, 8)) * np.sqrt(2 / 8), np.zeros(64),
             rng.standard_normal((64, 64)) * np.sqrt(2 / 64), np.zeros(64),
             rng.standard_normal((1, 64)) * np.sqrt(1 / 64), np.array([4.0])]
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)
