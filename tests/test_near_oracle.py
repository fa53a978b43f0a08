"""The near-field oracle (oracle/near_oracle.c) against golden blocks from the reference's own
shipped element routine run with its integration radii switched on (tests/golden/make_golden.py
near): every entry without a same-triangle pair to 1e-12 of the block's largest entry. The
same-triangle term is the project's own converged double integral (the library's is an
approximation a few per cent off): it is checked against the closed-form static integral and
by refinement."""
import glob
import os

import numpy as np
import pytest

from oracle import element as el
from pskel import mesh as pmesh

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
NEAR = sorted(glob.glob(os.path.join(GOLDEN, "near_*.npz")))


def _mesh_from(d):
    return pmesh.RWGMesh(vertex=d["vertex"], topol=d["topol"], trian=d["trian"], edges=d["edges"],
                         un=d["un"], ds=d["ds"], ln=d["ln"], cent=d["cent"])


def shared_triangle(m, rows, cols):
    """(len(rows), len(cols)) mask: the two RWGs (1-based) share a triangle."""
    tri = m.edges[:2].T  # (N, 2) 1-based triangles
    a = tri[np.asarray(rows) - 1]
    b = tri[np.asarray(cols) - 1]
    return ((a[:, None, :, None] == b[None, :, None, :]).any(axis=(2, 3)))


def test_near_fixtures_present():
    assert len(NEAR) == 4


@pytest.mark.parametrize("path", NEAR, ids=os.path.basename)
def test_near_oracle_matches_shipped_routine(path):
    d = np.load(path)
    m = _mesh_from(d)
    rs, ra, rf = (float(x) for x in d["radii"])
    Z = el.fill_near(m, d["rows"], d["cols"], float(d["k"]), float(d["eta"]), rs, ra, rf)
    ref = d["Z"]
    share = shared_triangle(m, d["rows"], d["cols"])
    assert share.any() and (~share).any()
    scale = np.abs(ref).max()
    assert np.abs(Z - ref)[~share].max() < 1e-12 * scale
    # same-triangle pairs: the library's term is an approximation (unpinned); it stays within
    # 10 % of the converged integral on these meshes
    rel = np.abs(Z - ref)[share] / np.abs(ref)[share]
    assert rel.max() < 0.1


def test_same_triangle_static_closed_form():
    """<1/R> over a triangle times itself has the closed form
    (4/3) sum_i (1/a_i) log(((a_i + b_i)^2 - c_i^2) / (b_i^2 - (a_i - c_i)^2)) (sides a, b, c
    cyclically); the oracle's same-triangle moment <G> tends to it / (4 pi) as k -> 0."""
    m = pmesh.icosphere(1.0, 2)
    for t in (0, 17, 101):
        V = m.vertex[:, m.topol[:, t] - 1].T
        a, b, c = (np.linalg.norm(V[i] - V[(i + 1) % 3]) for i in range(3))

        def term(a, b, c):
            return (1 / a) * np.log(((a + b) ** 2 - c ** 2) / (b ** 2 - (a - c) ** 2))
        exact = (4 / 3) * (term(a, b, c) + term(b, c, a) + term(c, a, b)) / (4 * np.pi)
        mom = el.self_moments(m, t, 1e-9)
        assert abs(mom[0].real - exact) < 1e-9 * exact
        assert abs(mom[0].imag + 1e-9 / (4 * np.pi)) < 1e-15


def test_same_triangle_term_converged():
    m = pmesh.icosphere(1.0, 2)
    k = 2 * np.pi
    for t in (3, 250):
        a = el.self_moments(m, t, k, 16)
        b = el.self_moments(m, t, k, 40)
        assert np.abs(a - b).max() < 3e-9 * np.abs(b).max()


def test_near_rule_reduces_to_far_rule_outside_radii():
    m = pmesh.two_plates(1.0, 8, 3.0)
    half = m.N // 2
    rows, cols = np.arange(1, 21), np.arange(half + 1, half + 31)  # plate 1 vs plate 2
    k, eta = 2 * np.pi, 376.73
    for q in (1, 7):
        Zn = el.fill_near(m, rows, cols, k, eta, 0.0, 0.0, 0.0, q_far=q)
        Zf = el.fill(m, rows, cols, k, eta, q, q)
        assert np.abs(Zn - Zf).max() < 1e-13 * np.abs(Zf).max()
