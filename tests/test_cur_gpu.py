"""The reference-named CUR round (cuda_complete_compression), the compressed-matvec error
(compute_error_compression) and the adaptive driver, against the numpy/LAPACK oracle and the
reference's own logged result on its two-sphere benchmark."""
import numpy as np
import pytest

from oracle import cur_oracle as co
from oracle import element as el
from pskel import api
from pskel import mesh as pmesh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def spheres768():
    m = pmesh.two_spheres(1.0, 12.0, 768)
    em = api.EMData.for_wavelength(4.0)
    return m, em, np.arange(1, 769), np.arange(769, 1537)


def test_round_with_given_samples(spheres768):
    m, em, r1, r2 = spheres768
    rng = np.random.default_rng(1)
    r = 40
    rows = np.sort(rng.choice(768, r, replace=False)) + 1
    cols = np.sort(rng.choice(768, r, replace=False)) + 1
    v = rng.random(768) + 1j * rng.random(768)
    yo = np.ones(768, complex)
    C, U, R, rs, cs, yn, err, ms = api.pure_cuda_compression2(
        v, yo, r, 1e-10, r1, r2, 1e-1, m, em, samples=(rows, cols))
    fill = lambda a, b: el.fill(m, a, b, em.k, em.eta, 1, 1)
    Co, Uo, Ro = co.cur_from_indices(fill, r1, r2, rows - 1, cols - 1, 1e-10)
    assert np.abs(C - Co).max() / np.abs(Co).max() < 1e-12
    assert np.abs(R - Ro).max() / np.abs(Ro).max() < 1e-12
    A, Ao = C @ U @ R, Co @ Uo @ Ro
    assert np.linalg.norm(A - Ao) / np.linalg.norm(Ao) < 1e-7
    y = co.compressed_matvec(Co, Uo, Ro, v)
    assert np.linalg.norm(yn - y) / np.linalg.norm(y) < 1e-7
    err_o = np.linalg.norm(yo - y) / np.linalg.norm(y)
    assert abs(err - err_o) / err_o < 1e-7
    assert ms > 0
    assert np.array_equal(rs, r1[rows - 1]) and np.array_equal(cs, r2[cols - 1])


def test_compute_error_matches_numpy():
    rng = np.random.default_rng(2)
    C = rng.standard_normal((50, 8)) + 1j * rng.standard_normal((50, 8))
    U = rng.standard_normal((8, 8)) + 1j * rng.standard_normal((8, 8))
    R = rng.standard_normal((8, 30)) + 1j * rng.standard_normal((8, 30))
    v = rng.random(30) + 1j * rng.random(30)
    yo = rng.random(50) + 0j
    err, yn = api.compute_error_cuda(C, U, R, yo, v)
    err_o, y = co.estimate_error(C, U, R, yo, v)
    assert np.linalg.norm(yn - y) / np.linalg.norm(y) < 1e-13
    assert abs(err - err_o) < 1e-12


def test_adaptive_driver_meets_tolerance(spheres768):
    m, em, r1, r2 = spheres768
    C, U, R, rs, cs, err, t = api.cuda_cur_compress3(r1, r2, 1e-3, m, em, rng=np.random.default_rng(3))
    Z = el.fill(m, r1, r2, em.k, em.eta, 1, 1)
    assert err <= 1e-3
    assert co.rel_fro_error(Z, C, U, R) < 1e-3
    assert t > 0


def test_reference_two_sphere_benchmark():
    """The reference's logged run (codes/GPU_implementation/seed/compres_single_block_spheres.txt:
    19-50): two R = 1 m octahedral spheres with Ne = 3072 each, 12 m apart, tol 1e-1; sizes
    307 -> 614 and a final relative Frobenius error of 3.6e-8..3.8e-8 against the dense block.
    The sizes are reproduced exactly; the error lands below the logged one (about 3e-9 here,
    for every wavelength tried from 0.5 to 4 m, with the numpy restatement on the same mesh),
    so the bar is the logged error's order of magnitude. The log's wavelength is not printed;
    the fixed-sample-count curves of the lambda sweep pin the error level instead
    (test_lambda_sweep_gpu.py)."""
    m = pmesh.two_spheres(1.0, 12.0, 3072)
    em = api.EMData.for_wavelength(2.0)
    r1, r2 = np.arange(1, 3073), np.arange(3073, 6145)
    Z, _ = api.user_impedance_cuda5(r1, r2, m, em)
    C, U, R, rs, cs, err, t = api.cuda_cur_compress3(r1, r2, 1e-1, m, em, rng=np.random.default_rng(0))
    assert C.shape == (3072, 614)
    e = co.rel_fro_error(Z, C, U, R)
    assert e < 1e-7, e
