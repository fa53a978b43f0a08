"""Octree grouping and far-pair list invariants."""
import numpy as np

from pskel import mesh as pmesh
from pskel import octree


def test_partition_invariants():
    m = pmesh.icosphere(2.0, 4)
    p = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=30)
    ids = np.sort(p.group_ids)
    assert np.array_equal(ids, np.arange(m.N))
    assert p.sizes().min() >= 30
    d = np.linalg.norm(p.centres[p.gt] - p.centres[p.gs], axis=1)
    assert np.all(d >= 2 * np.sqrt(3) * 0.5 - 1e-12)
    assert np.all(p.gt != p.gs)
    # ordered pairs: (i, j) far <=> (j, i) far
    pairs = set(zip(p.gt.tolist(), p.gs.tolist()))
    assert all((j, i) in pairs for i, j in pairs)
    q = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=30, symmetric=True)
    assert 2 * q.n_blocks == p.n_blocks and np.all(q.gt < q.gs)


def test_sphere_workload_shape():
    """The 30,720-RWG sphere: groups of 40-600 unknowns after merging boxes below 40."""
    m = pmesh.icosphere(2.0, 5)
    p = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=40)
    s = p.sizes()
    assert m.N == 30720 and s.min() >= 40 and s.max() <= 600
    assert p.n_blocks > 20000
