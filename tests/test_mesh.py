"""Mesh generators and RWG topology invariants (get_edge.m conventions)."""
import numpy as np
import pytest

from pskel import mesh as pmesh


def _check_rwg(m):
    ne = m.N
    tp, tm, vp, vm = (m.edges[i] - 1 for i in range(4))
    assert np.all(tp != tm)
    # the opposite vertex belongs to its triangle and is not on the shared edge
    for t, v in ((tp, vp), (tm, vm)):
        tri = m.topol[:, t] - 1
        assert np.all(np.any(tri == v, axis=0))
    # trian holds +e at (slot of v+, T+) and -e at (slot of v-, T-)
    for e in range(0, ne, max(1, ne // 97)):
        slot_p = int(np.where(m.topol[:, tp[e]] - 1 == vp[e])[0][0])
        slot_m = int(np.where(m.topol[:, tm[e]] - 1 == vm[e])[0][0])
        assert m.trian[slot_p, tp[e]] == e + 1
        assert m.trian[slot_m, tm[e]] == -(e + 1)
    assert np.all(m.ln > 0) and np.all(m.ds > 0)
    np.testing.assert_allclose(np.linalg.norm(m.un, axis=0), 1.0, atol=1e-13)


def test_two_plates_counts():
    m = pmesh.two_plates(1.0, 20, 3.0)
    assert m.Nt == 1600 and m.N == 2320
    c = m.basis_centres()
    assert np.all(c[2, :1160] == 0.0) and np.all(c[2, 1160:] == 3.0)
    _check_rwg(m)


@pytest.mark.parametrize("sub,nt,ne", [(2, 320, 480), (5, 20480, 30720)])
def test_icosphere_counts(sub, nt, ne):
    m = pmesh.icosphere(2.0, sub)
    assert m.Nt == nt and m.N == ne
    np.testing.assert_allclose(np.linalg.norm(m.vertex, axis=0), 2.0, rtol=1e-13)
    _check_rwg(m)


@pytest.mark.parametrize("ne", [12, 48, 192, 768])
def test_octa_sphere_counts(ne):
    m = pmesh.octa_sphere(1.0, ne)
    assert m.N == ne and m.Nt == 2 * ne // 3
    _check_rwg(m)


def test_two_spheres_split():
    m = pmesh.two_spheres(1.0, 12.0, 192)
    c = m.basis_centres()
    assert np.all(c[0, :192] < 2) and np.all(c[0, 192:] > 10)


def test_training_geometries():
    e = pmesh.ellipsoid(1.5, 1.0, 2.0, 0.25)
    _check_rwg(e)
    c = pmesh.cube(1.0, 0.25)
    assert c.Nt == 6 * 2 * 16 and c.N == 3 * c.Nt // 2
    _check_rwg(c)
