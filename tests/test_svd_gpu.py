"""Batched one-sided Jacobi SVD / truncated pinv against LAPACK (numpy), through the
reference-named entry points cuda_svd, cuda_pinv, cuda_filter and aux_pinv_compression."""
import numpy as np
import pytest

from oracle import cur_oracle as co
from pskel import api

pytestmark = pytest.mark.gpu


def _rand(m, n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))


@pytest.mark.parametrize("m,n", [(1, 1), (5, 3), (3, 5), (40, 40), (64, 40), (100, 100),
                                 (200, 150), (90, 260)])
def test_svd_matches_lapack(m, n):
    A = _rand(m, n, m * 1000 + n)
    U, S, Vt = api.cuda_svd(A)
    s_ref = np.linalg.svd(A, compute_uv=False)
    np.testing.assert_allclose(S, s_ref, rtol=1e-12, atol=1e-12 * s_ref[0])
    k = min(m, n)
    rec = (U * S) @ Vt[:k, :]
    assert np.linalg.norm(rec - A) / np.linalg.norm(A) < 1e-12
    assert np.linalg.norm(U.conj().T @ U - np.eye(k)) < 1e-12 * k
    assert np.linalg.norm(Vt[:k] @ Vt[:k].conj().T - np.eye(k)) < 1e-12 * k
    assert np.all(Vt[k:] == 0)


def test_pinv_rank_deficient_absolute_threshold():
    rng = np.random.default_rng(3)
    A = (rng.standard_normal((60, 12)) + 1j * rng.standard_normal((60, 12))) @ \
        (rng.standard_normal((12, 50)) + 1j * rng.standard_normal((12, 50)))
    P, U, S, Vt = api.cuda_pinv(A, 1e-10)
    ref = co.my_pinv(A, 1e-10)
    assert np.linalg.norm(P - ref) / np.linalg.norm(ref) < 1e-9
    assert np.sum(S >= 1e-10) == 12
    # the reference returns diag(1/s) V^H (zero rows below the threshold) in Vt
    assert np.all(Vt[12:] == 0)


def test_pinv_graded_spectrum():
    rng = np.random.default_rng(4)
    q1, _ = np.linalg.qr(_rand(80, 80, 1))
    q2, _ = np.linalg.qr(_rand(80, 80, 2))
    s = np.logspace(0, -14, 80)
    A = (q1 * s) @ q2.conj().T
    P, _, S, _ = api.cuda_pinv(A, 1e-8)
    np.testing.assert_allclose(S[:40], s[:40], rtol=1e-6)
    ref = co.my_pinv(A, 1e-8)
    assert np.linalg.norm(P - ref) / np.linalg.norm(ref) < 1e-6


def test_cuda_filter():
    v = np.array([1e-12, 0.5, 2.0, 1e-10, 3e-11])
    out = api.cuda_filter(v, 1e-10)
    np.testing.assert_allclose(out, [0, 2.0, 0.5, 1e10, 0])


def test_aux_pinv_compression():
    rng = np.random.default_rng(9)
    A = _rand(70, 20, 7) @ _rand(20, 90, 8)
    rows = np.sort(rng.choice(70, 25, replace=False)) + 1
    cols = np.sort(rng.choice(90, 25, replace=False)) + 1
    C, U, R, _, _ = api.cuda_cur_pinv2(A, 25, 1e-10, samples=(rows, cols))
    assert np.array_equal(C, A[:, cols - 1]) and np.array_equal(R, A[rows - 1, :])
    ref = co.my_pinv(A[np.ix_(rows - 1, cols - 1)], 1e-10)
    assert np.linalg.norm(C @ U @ R - C @ ref @ R) / np.linalg.norm(A) < 1e-8
    assert np.linalg.norm(C @ U @ R - A) / np.linalg.norm(A) < 1e-8
