"""Library state on a second device: kernel shared-memory limits, the reference entry points'
context and the allocation-free scratch are all kept per device ordinal, so work on device 1
after device 0 in one process must run. Skipped where fewer than two GPUs are visible (the
per-device keying itself is checked on the CPU in test_device_state_host.py)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _need_two():
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")


def test_second_device_after_first():
    _need_two()
    import torch

    from pskel import _lib, api
    from pskel import mesh as pmesh
    from pskel import octree
    from pskel.engine import Engine

    rng = np.random.default_rng(0)
    A = rng.standard_normal((64, 64)) + 1j * rng.standard_normal((64, 64))
    s = pmesh.icosphere(2.0, 2)
    part = octree.partition(s, 0.6, origin=(0, 0, 0), min_group=10)
    results = []
    for dev in (0, 1):
        torch.cuda.set_device(dev)
        # reference-named pinv (per-device legacy context; 64 x 64 resident SVD needs the
        # > 48 KiB shared-memory limit on this device)
        P, _, S, _ = api.cuda_pinv(A, 1e-10)
        # allocation-free pinv on the same device
        a = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda(dev)
        p = torch.zeros((64, 64), dtype=torch.complex128, device=f"cuda:{dev}")
        vp = lambda t: ctypes.c_void_p(t.data_ptr())
        _lib.check(_lib.lib().pskel_pinv_noalloc(vp(a), 64, 64, 1e-10, 0, vp(p), None, None, None))
        assert np.linalg.norm(p.cpu().numpy().T - P) <= 1e-10 * np.linalg.norm(P)
        # a batched compression on a context bound to this device
        with Engine(dev) as eng:
            eng.upload_mesh(s, 2 * np.pi, 376.73, q=7)
            eng.set_blocks(part)
            st = eng.compress(1e-3, precision="c128", seed=0)
            results.append((S, st["r"].copy()))
    np.testing.assert_allclose(results[0][0], results[1][0], rtol=1e-12)
    assert np.array_equal(results[0][1], results[1][1])
