"""The reference's error-versus-sample-count curves (its CPU CUR at fixed sample counts, the
lambda sweep of codes/ACA_vs_CUR/seed/compres_single_block_spheres_for_lambda_sweep.jl:683-751,
results in codes/ACA_vs_CUR/global_results.jld): two R = 1 m octahedral spheres of 12,288 RWG
each, 12 m apart, eta = 120 pi, lambda = 5 or 10 x 0.06048 m (the mesh's mean edge), every pair
on the centroid rule; CUR with r = ceil(12288 x {0.1, 0.5, 1, 5} %) = 13, 62, 123, 615 uniform
samples and the reference's absolute pinv threshold 1e-10 (cur_pinv3 / my_pinv).

The library's reference-named round (cuda_complete_compression through pskel.api) forms C, U, R
on the device; the error against the dense block (filled on the device) must land on the
reference's logged value within the spread of the random draw (a factor 3, 5 for r = 13 where
a single draw varies most). The logged values are single unseeded draws."""
import numpy as np
import pytest

from pskel import api
from pskel import mesh as pmesh
from pskel.engine import Engine

pytestmark = pytest.mark.gpu

# global_results.jld, CUR relative error at r = 13 / 62 / 123 / 615 (lambda cases 1 and 2)
LOGGED = {1: (0.846, 2.82e-2, 8.92e-5, 1.49e-8), 2: (7.99e-2, 3.24e-4, 2.56e-6, 8.47e-9)}
SAMPLES = (13, 62, 123, 615)


@pytest.fixture(scope="module")
def spheres():
    return pmesh.two_spheres(1.0, 12.0, 12288)


@pytest.mark.parametrize("case", [1, 2])
def test_error_versus_samples_matches_the_reference_sweep(spheres, case):
    import torch
    m = spheres
    ne = m.N // 2
    assert ne == 12288
    lam = 5 * case * 0.06048
    em = api.EMData.for_wavelength(lam)  # eta = 120 pi, radii 1 m: all pairs on the centroid rule
    r1, r2 = np.arange(1, ne + 1), np.arange(ne + 1, 2 * ne + 1)
    dev = torch.device("cuda:0")
    with Engine() as eng:
        eng.upload_mesh(m, em.k, em.eta, q=1)
        rows = torch.arange(0, ne, dtype=torch.int32, device=dev)
        cols = torch.arange(ne, 2 * ne, dtype=torch.int32, device=dev)
        Zt = torch.empty((ne, ne), dtype=torch.complex128, device=dev)  # Z^T row-major = Z col-major
        torch.cuda.synchronize()
        eng.fill_device(rows.data_ptr(), ne, cols.data_ptr(), ne, Zt.data_ptr(), ne)
        torch.cuda.synchronize()
    Z = Zt.t()
    nz = torch.linalg.norm(Z)
    rng = np.random.default_rng(100 + case)
    v = np.ones(ne, dtype=np.complex128)
    y0 = np.zeros(ne, dtype=np.complex128)
    errs = []
    for r, logged in zip(SAMPLES, LOGGED[case]):
        rl = np.sort(rng.choice(ne, r, replace=False)) + 1
        cl = np.sort(rng.choice(ne, r, replace=False)) + 1
        C, U, R = api.pure_cuda_compression2(v, y0, r, 1e-10, r1, r2, 1.0, m, em,
                                             samples=(rl, cl))[:3]
        Cd, Ud, Rd = (torch.as_tensor(np.ascontiguousarray(x), device=dev) for x in (C, U, R))
        e = float(torch.linalg.norm(Z - Cd @ (Ud @ Rd)) / nz)
        errs.append(e)
        f = 5.0 if r == 13 else 3.0
        assert logged / f <= e <= logged * f, (case, r, e, logged)
    assert all(a > b for a, b in zip(errs, errs[1:]))
