"""CPU checks of two restatements used as checkers: the ACA of ACA_julia.jl (exact recovery of a
low-rank matrix, the rank cap, agreement of its running norm estimate with ||U V||_F) and
test_fields (against a per-RWG loop written from the formula)."""
import numpy as np

from oracle import aca_oracle as ao
from oracle import fields_oracle as fo
from pskel import mesh as pmesh


def test_aca_recovers_low_rank():
    rng = np.random.default_rng(0)
    m, n, k = 60, 45, 7
    Z = (rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))) @ \
        (rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n)))
    r = ao.aca(lambda i: Z[i], lambda j: Z[:, j], m, n, 1e-12)
    assert r["k"] in (k, k + 1)  # the last cross can be a rounding-level one
    assert np.linalg.norm(Z - r["U"] @ r["V"]) < 1e-10 * np.linalg.norm(Z)
    assert len(set(r["I"].tolist())) == r["k"] and len(set(r["J"].tolist())) == r["k"]
    assert r["I"][0] == 0  # the first row pivot is the first row
    capped = ao.aca(lambda i: Z[i], lambda j: Z[:, j], m, n, 1e-12, kmax=3)
    assert capped["k"] == 3 and capped["status"] == 1


def test_aca_pivots_follow_the_largest_residual():
    rng = np.random.default_rng(1)
    Z = rng.standard_normal((30, 20)) + 1j * rng.standard_normal((30, 20))
    r = ao.aca(lambda i: Z[i], lambda j: Z[:, j], 30, 20, 1e-3)
    # the first column pivot is the largest entry of row 0
    assert r["J"][0] == int(np.argmax(np.abs(Z[0])))
    # the second row pivot is the largest entry of the first column residual outside row 0
    col = Z[:, r["J"][0]]
    cand = np.abs(col).copy()
    cand[0] = -1
    assert r["I"][1] == int(np.argmax(cand))


def test_plane_wave_against_loop():
    m = pmesh.icosphere(1.0, 2)
    k, eta = 2 * np.pi, 376.73
    th, ph, rot = 30.0, 40.0, 15.0
    E, H = fo.test_fields(m, th, ph, rot, k, eta)
    t, p, a = np.radians(th), ph / 180.0, np.radians(rot)
    ki = -np.array([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)])
    ei = np.cos(a) * np.array([-np.sin(p), np.cos(p), 0]) + \
        np.sin(a) * np.array([np.cos(t) * np.cos(p), np.cos(t) * np.sin(p), -np.sin(t)])
    for e in (0, 17, m.N - 1):
        tp, tm, vp, vm = (int(x) - 1 for x in m.edges[:4, e])
        cp, cm = m.cent[:, tp], m.cent[:, tm]
        val = m.ln[e] / 2 * (ei @ (cp - m.vertex[:, vp]) * np.exp(-1j * k * ki @ cp) +
                             ei @ (m.vertex[:, vm] - cm) * np.exp(-1j * k * ki @ cm))
        assert abs(E[e] - val) < 1e-14 * max(1.0, abs(val))
    assert np.all(np.isfinite(H))
