"""Validation of the 7-point rule of the oracle (no reference counterpart): self-convergence
against a refined composite centroid rule, Galerkin symmetry, and agreement with the
reference's centroid rule far away."""
import numpy as np

from oracle import element as el
from pskel import mesh as pmesh


def test_q7_matches_refined_composite_rule():
    m = pmesh.two_plates(1.0, 4, 1.0)
    k, eta = 2 * np.pi, 376.73
    h = m.N // 2
    pairs = [(1, h + 1), (3, h + 7), (h // 2, h + h // 2)]
    for a, b in pairs:
        z7 = el.fill(m, [a], [b], k, eta, 7, 7)[0, 0]
        zc = el.element_composite(m, a, b, k, eta, 4)
        assert abs(z7 - zc) / abs(zc) < 2e-3  # composite midpoint error O(h^2 / 4^4)
        z1 = el.fill(m, [a], [b], k, eta, 1, 1)[0, 0]
        assert abs(z7 - zc) < abs(z1 - zc)  # Q=7 beats the centroid rule


def test_q7_galerkin_symmetry():
    m = pmesh.two_plates(1.0, 6, 2.0)
    k, eta = 2 * np.pi, 376.73
    ids = np.arange(1, m.N + 1, 9)
    Z = el.fill(m, ids, ids[::-1][:len(ids)], k, eta, 7, 7)
    Zt = el.fill(m, ids[::-1][:len(ids)], ids, k, eta, 7, 7)
    off = ~np.eye(len(ids), dtype=bool)[:, ::-1]  # skip coincident pairs
    np.testing.assert_allclose(Z[off], Zt.T[off], rtol=1e-12, atol=0)


def test_q7_approaches_centroid_rule_far_away():
    diffs = []
    for gap in (3.0, 12.0, 48.0):
        m = pmesh.two_plates(1.0, 4, gap)
        h = m.N // 2
        r1 = np.arange(1, h + 1, 5)
        r2 = np.arange(h + 1, m.N + 1, 5)
        z7 = el.fill(m, r1, r2, 2 * np.pi, 376.73, 7, 7)
        z1 = el.fill(m, r1, r2, 2 * np.pi, 376.73, 1, 1)
        diffs.append(np.abs(z7 - z1).max() / np.abs(z7).max())
    assert diffs[0] < 0.05
    assert diffs[2] < diffs[0]
