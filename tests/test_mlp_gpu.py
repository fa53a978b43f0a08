"""Hand-written MLP kernels (forward, MSE gradient, Adam) against the numpy oracle."""
import ctypes

import numpy as np
import pytest

from oracle import mlp_oracle as mo
from pskel import _lib
from pskel.predictor import Predictor, init_params

pytestmark = pytest.mark.gpu


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("n", [1, 37, 128, 1000])
def test_forward_and_gradient_match_oracle(n):
    import torch
    L = _lib.lib()
    rng = np.random.default_rng(n)
    p = init_params(n).astype(np.float64) + 0.05 * rng.standard_normal(mo.NPARAM)
    x = rng.standard_normal((n, 8))
    t = rng.standard_normal(n) + 3
    pd, xd, td = _t(p), _t(x), _t(t)
    y = torch.empty(n, dtype=torch.float32, device="cuda")
    _lib.check(L.pskel_mlp_forward(_vp(pd), _vp(xd), n, _vp(y), None))
    yo = mo.forward(p.astype(np.float32).astype(np.float64), x.astype(np.float32).astype(np.float64))
    np.testing.assert_allclose(y.cpu().numpy(), yo, rtol=2e-5, atol=2e-5)
    g = torch.empty(mo.NPARAM, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    _lib.check(L.pskel_mlp_grad(_vp(pd), _vp(xd), _vp(td), n, _vp(g), _vp(loss), None))
    go, lo = mo.grad(p.astype(np.float32).astype(np.float64), x.astype(np.float32).astype(np.float64),
                     t.astype(np.float32).astype(np.float64))
    gg = g.cpu().numpy()
    assert np.linalg.norm(gg - go) / np.linalg.norm(go) < 1e-4
    assert abs(loss.item() - lo) / lo < 1e-4


def test_adam_matches_oracle():
    import torch
    L = _lib.lib()
    rng = np.random.default_rng(1)
    p = rng.standard_normal(mo.NPARAM)
    g = rng.standard_normal(mo.NPARAM)
    m = rng.standard_normal(mo.NPARAM) * 0.1
    v = np.abs(rng.standard_normal(mo.NPARAM)) * 0.1
    pd, gd, md, vd = _t(p), _t(g), _t(m), _t(v)
    _lib.check(L.pskel_mlp_adam(_vp(pd), _vp(gd), _vp(md), _vp(vd), 3, 1e-2, 0.9, 0.999, 1e-8, None))
    po, mo_, vo = mo.adam(p.astype(np.float32), g.astype(np.float32), m.astype(np.float32),
                          v.astype(np.float32), 3, 1e-2)
    np.testing.assert_allclose(pd.cpu().numpy(), po, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(md.cpu().numpy(), mo_, rtol=1e-5, atol=1e-7)


def test_training_fits_a_smooth_target():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((20000, 8))
    y = 3 + np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] + 0.2 * x[:, 3]
    pr = Predictor(init_params(3))
    hist = pr.fit(x, y, steps=1500, batch=2048, lr=3e-3, log_every=500)
    assert hist[-1][1] < 0.05 * np.var(y) + 0.01
    yp = pr.predict_log2(x[:2000])
    assert np.sqrt(np.mean((yp - y[:2000]) ** 2)) < 0.3
