"""The numpy MLP oracle's gradient against central finite differences (CPU)."""
import numpy as np

from oracle import mlp_oracle as mo


def test_oracle_gradient_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(mo.NPARAM) * 0.3
    x = rng.standard_normal((12, 8))
    t = rng.standard_normal(12)
    g, _ = mo.grad(p, x, t)
    f = lambda q: np.mean((mo.forward(q, x) - t) ** 2)
    idx = rng.choice(mo.NPARAM, 40, replace=False)
    h = 1e-6
    fd = np.array([(f(p + h * np.eye(1, mo.NPARAM, i)[0]) - f(p - h * np.eye(1, mo.NPARAM, i)[0])) / (2 * h)
                   for i in idx])
    np.testing.assert_allclose(g[idx], fd, rtol=1e-5, atol=1e-8)


def test_predictor_features_shape():
    from pskel import mesh as pmesh
    from pskel import octree
    from pskel.predictor import FEATURES, features
    m = pmesh.icosphere(2.0, 3)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20)
    f = features(part, 2 * np.pi, 1e-4)
    assert f.shape == (part.n_blocks, len(FEATURES)) == (part.n_blocks, 8)
    assert np.all(np.isfinite(f)) and np.allclose(f[:, 6], 4.0)
    assert np.all(f[:, 4] >= 2 * np.sqrt(3) * 0.5 - 1e-9)
