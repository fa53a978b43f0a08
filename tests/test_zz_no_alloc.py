"""The allocation-free pseudo-inverse entry point (pskel_pinv_noalloc), checked against the
allocating one (cuda_pinv) through the C ABI.

It serves callers that cannot call cudaMalloc - code running inside a framework that owns
device memory through its own pool, or a latency-critical loop where an allocation could block
or synchronise the device - so it works in a fixed 256 KiB device array (matrices up to
64 x 64). This file is named to be collected last: if it fails, a run that stops at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from pskel import _lib, api

pytestmark = pytest.mark.gpu


def _noalloc(A, tau, relative=0):
    import torch
    M, N = A.shape
    a = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()  # column-major storage
    p = torch.zeros((M, N), dtype=torch.complex128, device="cuda")  # N x M column-major
    s = torch.zeros(min(M, N), dtype=torch.float64, device="cuda")
    r = torch.zeros(1, dtype=torch.int32, device="cuda")
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    _lib.check(_lib.lib().pskel_pinv_noalloc(vp(a), M, N, float(tau), int(relative), vp(p),
                                            vp(s), vp(r), None))
    return p.cpu().numpy().T, s.cpu().numpy(), int(r.item())


def _case(M, N, rank, seed):
    rng = np.random.default_rng(seed)
    A = (rng.standard_normal((M, rank)) + 1j * rng.standard_normal((M, rank))) @ \
        (rng.standard_normal((rank, N)) + 1j * rng.standard_normal((rank, N)))
    return A


@pytest.mark.parametrize("shapes", [((40, 40, 40), (64, 48, 20)), ((30, 60, 25), (64, 64, 64))])
def test_noalloc_matches_allocating_pinv_on_two_calls(shapes):
    for i, (M, N, k) in enumerate(shapes):  # two calls in a row, different sizes and data
        A = _case(M, N, k, 100 * i + M)
        P, S, rank = _noalloc(A, 1e-10)
        P_ref, _, S_ref, _ = api.cuda_pinv(A, 1e-10)
        assert P.shape == (N, M)
        assert np.linalg.norm(P - P_ref) <= 1e-10 * np.linalg.norm(P_ref)
        np.testing.assert_allclose(S, S_ref, rtol=1e-12, atol=1e-12 * S_ref[0])
        assert rank == int(np.sum(S_ref >= 1e-10)) == min(k, M, N)


def test_noalloc_relative_threshold_and_limit():
    A = _case(50, 50, 50, 7)
    P, S, rank = _noalloc(A, 1e-3, relative=1)
    assert rank == int(np.sum(S >= 1e-3 * S[0]))
    with pytest.raises(_lib.PskelError) as e:
        _noalloc(_case(65, 10, 5, 1), 1e-10)
    assert e.value.code == -1
