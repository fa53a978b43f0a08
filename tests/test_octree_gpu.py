"""Device octree partition (pskel_octree_build) against the host restatement
(pskel/octree.py, partition): groups, group ids, centres and the far list bit for bit, extents to
rounding, on the sphere and plate workloads, with and without merging, a given or derived
origin, both far-list forms and other admissibility factors."""
import ctypes

import numpy as np
import pytest

from pskel import _lib
from pskel import mesh as pmesh
from pskel import octree
from pskel.engine import Engine

pytestmark = pytest.mark.gpu

K, ETA = 2 * np.pi, 376.73


def _same(a, b):
    assert a.n_groups == b.n_groups and a.n_blocks == b.n_blocks
    assert np.array_equal(a.group_ptr, b.group_ptr)
    assert np.array_equal(a.group_ids, b.group_ids)
    assert np.array_equal(a.centres, b.centres)  # exact: every step IEEE-rounded in one order
    assert np.array_equal(a.gt, b.gt) and np.array_equal(a.gs, b.gs)
    assert np.allclose(a.extents, b.extents, rtol=1e-12, atol=1e-14)


CASES = [
    # (radius, subdivisions, leaf, origin, min_group, admissibility)
    (2.0, 3, 0.5, (0, 0, 0), 20, 2.0),
    (2.0, 4, 0.5, (0, 0, 0), 30, 2.0),
    (2.0, 4, 0.5, None, 1, 2.0),
    (2.0, 5, 0.5, (0, 0, 0), 40, 2.0),
    (2.0, 5, 0.5, None, 40, 1.5),
    (2.0, 5, 0.37, (0.1, -0.2, 0.05), 25, 3.0),
    (4.0, 6, 0.5, (0, 0, 0), 40, 2.0),
]


@pytest.mark.parametrize("R,sub,leaf,origin,min_group,adm", CASES)
def test_octree_matches_host(R, sub, leaf, origin, min_group, adm):
    m = pmesh.icosphere(R, sub)
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        for sym in (False, True):
            d = eng.octree(leaf, origin=origin, admissibility=adm, min_group=min_group, symmetric=sym)
            h = octree.partition(m, leaf, origin=origin, admissibility=adm, min_group=min_group,
                                 symmetric=sym)
            _same(d, h)


def test_octree_plates_and_edge_cases():
    m = pmesh.two_plates(1.0, 20, 3.0)
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        for leaf, mg in [(0.25, 1), (0.25, 20), (0.5, 60), (10.0, 1)]:
            _same(eng.octree(leaf, min_group=mg), octree.partition(m, leaf, min_group=mg))
        # everything folds into one group: no far pairs
        one = eng.octree(0.25, min_group=m.N + 1)
        _same(one, octree.partition(m, 0.25, min_group=m.N + 1))
        assert one.n_groups == 1 and one.n_blocks == 0
        # the device partition drives a compression like the host one
        part = eng.octree(0.25, min_group=20)
        eng.set_blocks(part)
        assert eng.n_blocks == part.n_blocks
        lib = _lib.lib()
        ng, nb = ctypes.c_int(), ctypes.c_longlong()
        for leaf, adm in [(0.0, 2.0), (-1.0, 2.0), (float("nan"), 2.0), (0.5, -1.0)]:
            rc = lib.pskel_octree_build(eng._h, leaf, None, adm, 1, 0, ctypes.byref(ng), ctypes.byref(nb))
            assert rc == -1
    with Engine() as eng:
        with pytest.raises(RuntimeError):
            eng.octree(0.5)  # no mesh uploaded
