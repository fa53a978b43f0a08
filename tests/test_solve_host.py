"""Host parts of the H-matrix solve: the near-pair list of a partition and the restarted GMRES
(run here on CPU tensors against a direct solve)."""
import numpy as np
import torch

from pskel import mesh as pmesh
from pskel import octree
from pskel.solve import gmres, near_pairs


def test_near_pairs_complement_far_list():
    m = pmesh.icosphere(2.0, 3)
    p = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20)
    t, s = near_pairs(p)
    G = p.n_groups
    pairs = set(zip(t.tolist(), s.tolist()))
    far = set(zip(p.gt.tolist(), p.gs.tolist()))
    assert len(pairs) + len(far) == G * G and not (pairs & far)
    assert all((g, g) in pairs for g in range(G))
    # the symmetric far list gives the same near list
    q = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20, symmetric=True)
    t2, s2 = near_pairs(q)
    assert np.array_equal(t, t2) and np.array_equal(s, s2)


def test_gmres_matches_direct_solve():
    rng = np.random.default_rng(0)
    n = 300
    A = np.eye(n) * 4 + (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    At = torch.as_tensor(A)
    x, hist, nmv = gmres(lambda v: At @ v, torch.as_tensor(b), tol=1e-10, restart=20, maxiter=500)
    xd = np.linalg.solve(A, b)
    assert np.linalg.norm(x.numpy() - xd) < 1e-8 * np.linalg.norm(xd)
    assert hist[-1] <= 1e-10 and nmv < 500
    assert np.linalg.norm(A @ x.numpy() - b) <= 1.01e-10 * np.linalg.norm(b)


def test_gmres_single_cycle_reaches_tolerance():
    """Without restarts GMRES minimises the residual over the Krylov space: one cycle of
    dimension n solves an n x n complex system to rounding, and the true residual after the
    cycle matches the rotated right-hand side."""
    rng = np.random.default_rng(1)
    n = 60
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) + 2j * np.eye(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    At = torch.as_tensor(A)
    x, hist, nmv = gmres(lambda v: At @ v, torch.as_tensor(b), tol=1e-11, restart=n, maxiter=n + 1)
    assert len(hist) == 2 and hist[-1] < 1e-9
    assert nmv <= n + 1
