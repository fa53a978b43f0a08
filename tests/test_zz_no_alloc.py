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


def _buffers(A):
    import torch
    M, N = A.shape
    a = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()  # column-major storage
    p = torch.zeros((M, N), dtype=torch.complex128, device="cuda")  # N x M column-major
    s = torch.zeros(min(M, N), dtype=torch.float64, device="cuda")
    r = torch.zeros(1, dtype=torch.int32, device="cuda")
    return a, p, s, r


def _call(bufs, M, N, tau, relative=0, stream=None):
    a, p, s, r = bufs
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    return _lib.lib().pskel_pinv_noalloc(vp(a), M, N, float(tau), int(relative), vp(p), vp(s),
                                         vp(r), stream)


def _noalloc(A, tau, relative=0):
    M, N = A.shape
    bufs = _buffers(A)
    _lib.check(_call(bufs, M, N, tau, relative))
    _, p, s, r = bufs
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


def test_noalloc_leaves_free_device_memory_unchanged():
    """The property the entry point exists for: once the device is set up (first call), calls
    take no device memory - the free memory the driver reports is the same before and after."""
    import torch
    A = _case(48, 40, 30, 3)
    bufs = _buffers(A)
    _lib.check(_call(bufs, 48, 40, 1e-10))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        _lib.check(_call(bufs, 48, 40, 1e-10))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_refuses_a_capturing_stream():
    """The call waits for its stream, which a stream capture forbids: on a capturing stream it
    returns PSKEL_ERR_STATE before touching the stream, and the caller's capture still ends
    cleanly."""
    import torch
    A = _case(20, 20, 20, 4)
    bufs = _buffers(A)
    _lib.check(_call(bufs, 20, 20, 1e-10))  # device set up before any capture
    x = torch.zeros(4, device="cuda")
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            x.add_(1.0)
            code = _call(bufs, 20, 20, 1e-10, stream=ctypes.c_void_p(s.cuda_stream))
        finally:
            g.capture_end()
    assert code == -8  # PSKEL_ERR_STATE
    g.replay()
    torch.cuda.synchronize()
    assert float(x.sum()) == 4.0
