"""H-matrix product and iterative solve on the device (near blocks dense with the near-field
rule, far blocks compressed):
- the plane-wave excitation against the restatement of the reference's test_fields;
- the H-matrix product against the dense product of the same rule (every pair filled with the
  near-field kernel) within the compression tolerance;
- GMRES on (-Z) x = E (the reference's solve_by_CBF(-Ze, Ei) system) against a dense direct
  solve of the same matrix."""
import numpy as np
import pytest
import torch

from oracle import fields_oracle as fo
from pskel import mesh as pmesh
from pskel import octree
from pskel.engine import Engine
from pskel.solve import HMatrix, gmres, plane_wave

pytestmark = pytest.mark.gpu

K, ETA = 2 * np.pi, 376.73
RADII = (0.15, 0.15, 0.15)


@pytest.fixture(scope="module")
def setup():
    m = pmesh.icosphere(2.0, 3)  # 1,920 RWG
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20)
    eng = Engine()
    eng.upload_mesh(m, K, ETA, q=7)
    eng.set_blocks(part)
    # the dense matrix of the same rule: every pair by the near-field kernel (7-point outside
    # the radii, like the far blocks' fill)
    dev = torch.device("cuda:0")
    ids = torch.arange(m.N, dtype=torch.int32, device=dev)
    Zt = torch.empty((m.N, m.N), dtype=torch.complex128, device=dev)
    torch.cuda.synchronize()
    eng.fill_near_device(ids.data_ptr(), m.N, ids.data_ptr(), m.N, Zt.data_ptr(), m.N, *RADII, q_far=7)
    torch.cuda.synchronize()
    Z = Zt.t().contiguous()  # row-major view of the column-major fill: Z[i, j]
    yield m, part, eng, Z
    eng.close()


def test_plane_wave_matches_test_fields(setup):
    m, part, eng, Z = setup
    for th, ph, rot in ((0.0, 0.0, 0.0), (37.0, 110.0, 25.0)):
        E = plane_wave(eng, th, ph, rot).cpu().numpy()
        Eo, _ = fo.test_fields(m, th, ph, rot, K, ETA)
        assert np.abs(E - Eo).max() < 1e-13 * np.abs(Eo).max()


@pytest.mark.parametrize("tol", [1e-4, 1e-6])
def test_hmatrix_product_matches_dense(setup, tol):
    m, part, eng, Z = setup
    eng.set_symmetric(True)
    eng.compress(tol, precision="c128", tau=1e-10, seed=1)
    err = eng.true_errors()
    H = HMatrix(eng, part, RADII, q_far=7)
    assert H.near_bytes > 0 and H.n_near + part.n_blocks == part.n_groups ** 2
    rng = np.random.default_rng(2)
    X = torch.as_tensor(rng.standard_normal((m.N, 4)) + 1j * rng.standard_normal((m.N, 4)), device="cuda")
    Y = H.matvec(X)
    Yd = Z @ X
    # near part exact (same entries), far part within the blocks' compression errors
    Yn = H.matvec(X, far=False)
    far_mask = torch.zeros((m.N, m.N), dtype=torch.bool, device="cuda")
    gp, gi = part.group_ptr, part.group_ids
    for t, s in zip(part.gt, part.gs):
        r = torch.as_tensor(gi[gp[t]:gp[t + 1]], device="cuda").long()
        c = torch.as_tensor(gi[gp[s]:gp[s + 1]], device="cuda").long()
        far_mask[r[:, None], c[None, :]] = True
    Zn = torch.where(far_mask, torch.zeros_like(Z), Z)
    assert float(torch.linalg.norm(Yn - Zn @ X) / torch.linalg.norm(Zn @ X)) < 1e-13
    rel = float(torch.linalg.norm(Y - Yd) / torch.linalg.norm(Yd))
    assert rel < 3 * err.max(), (rel, err.max())


def test_gmres_solution_matches_dense_solve(setup):
    m, part, eng, Z = setup
    eng.set_symmetric(True)
    eng.compress(1e-6, precision="c128", tau=1e-10, seed=1)
    H = HMatrix(eng, part, RADII, q_far=7)
    E = plane_wave(eng, 0.0, 0.0, 0.0)
    x, hist, nmv = gmres(lambda v: -H.matvec(v), E, tol=1e-8, restart=80, maxiter=1500)
    assert hist[-1] <= 1e-8
    xd = torch.linalg.solve(-Z, E)
    rel = float(torch.linalg.norm(x - xd) / torch.linalg.norm(xd))
    assert rel < 1e-4, (rel, nmv)

