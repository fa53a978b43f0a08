"""Element fill on the GPU against the golden vectors of the reference's shipped element
routine and against the CPU oracle (FP64 1e-6 / complex FP32 1e-4 bars; FP64 lands near
1e-13)."""
import glob
import os

import numpy as np
import pytest

from oracle import element as el
from pskel import _lib, api
from pskel import mesh as pmesh

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "so_*.npz")))


def _mesh(d):
    return pmesh.RWGMesh(vertex=d["vertex"], topol=d["topol"], trian=d["trian"], edges=d["edges"],
                         un=d["un"], ds=d["ds"], ln=d["ln"], cent=d["cent"])


def _em(d):
    r = float(d["rint"])
    return api.EMData(2 * np.pi / float(d["k"]), float(d["k"]), float(d["eta"]), 1, r, r, r, 0, 0)


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_elbyel4_matches_shipped_routine(path):
    d = np.load(path)
    m = _mesh(d)
    Z, ms = api.user_impedance_cuda5(d["rows"], d["cols"], m, _em(d))
    assert ms >= 0
    ref = d["Z"]
    rows = list(d["rows"])
    last = np.array([i == len(rows) - 1 - rows[::-1].index(r) for i, r in enumerate(rows)])
    rel = np.abs(Z[last] - ref[last]).max() / np.abs(ref).max()
    assert rel < 1e-12, rel
    # every requested entry is filled (repeated ids included), as the oracle does
    Zo = el.fill(m, d["rows"], d["cols"], float(d["k"]), float(d["eta"]), 1, 1)
    assert np.abs(Z - Zo).max() / np.abs(Zo).max() < 1e-12


def test_fill_variants_agree():
    d = np.load(FIXTURES[0])
    m, em = _mesh(d), _em(d)
    Z4, _ = api.user_impedance_cuda5(d["rows"], d["cols"], m, em)
    Z3 = api.user_impedance_cuda4(d["rows"], d["cols"], m, em)
    Z2 = api.user_impedance_cuda3(d["rows"], d["cols"], m, em)
    assert np.array_equal(Z4, Z3) and np.array_equal(Z4, Z2)


def test_bad_ids_are_reported():
    m = pmesh.two_spheres(1.0, 12.0, 48)
    em = api.EMData.for_wavelength(2.0)
    with pytest.raises(_lib.PskelError) as e:
        api.user_impedance_cuda5(np.array([1, 2, 97]), np.arange(49, 52), m, em)
    assert e.value.code == -6
    with pytest.raises(_lib.PskelError):
        api.user_impedance_cuda5(np.array([1]), np.array([2]), m, api.EMData(2.0, np.pi, 377.0, field=2))


def test_empty_fill():
    m = pmesh.two_spheres(1.0, 12.0, 48)
    Z, _ = api.user_impedance_cuda5(np.zeros(0, int), np.arange(49, 52), m, api.EMData.for_wavelength(2.0))
    assert Z.shape == (0, 3)


@pytest.mark.parametrize("prec,bar", [("c128", 1e-6), ("c64", 1e-4)])
def test_q7_device_fill_matches_oracle(prec, bar):
    import torch
    from pskel.engine import Engine
    m = pmesh.two_plates(1.0, 20, 3.0)
    k, eta = 2 * np.pi, 376.73
    rng = np.random.default_rng(5)
    rows = np.sort(rng.choice(1160, 70, replace=False))
    cols = np.sort(rng.choice(np.arange(1160, 2320), 90, replace=False))
    ref = el.fill(m, rows + 1, cols + 1, k, eta, 7, 7)
    with Engine() as eng:
        eng.upload_mesh(m, k, eta, q=7)
        r_d = torch.tensor(rows, dtype=torch.int32, device="cuda")
        c_d = torch.tensor(cols, dtype=torch.int32, device="cuda")
        dt = torch.complex128 if prec == "c128" else torch.complex64
        out = torch.zeros((len(cols), len(rows)), dtype=dt, device="cuda")  # column-major view
        eng.fill_device(r_d.data_ptr(), len(rows), c_d.data_ptr(), len(cols), out.data_ptr(),
                        len(rows), prec)
        torch.cuda.synchronize()
        Z = out.cpu().numpy().T.astype(np.complex128)
    rel_max = np.abs(Z - ref).max() / np.abs(ref).max()
    rel_fro = np.linalg.norm(Z - ref) / np.linalg.norm(ref)
    assert rel_max < bar and rel_fro < bar, (rel_max, rel_fro)
    if prec == "c128":
        assert rel_max < 1e-12


def test_fill_sincos_against_cuda_sincospi():
    """The fill kernels' own sin/cos against CUDA's sincospi: the quarter-turn Taylor forms in
    FP64 within a few ulp and in FP32 within a few FP32 ulp, the half-turn near-minimax FP32 form
    within a few FP32 ulp, over phases of 0 to 40 wavelengths."""
    import ctypes
    import torch
    rng = np.random.default_rng(0)
    t = np.concatenate([rng.uniform(0, 40, 200000), np.arange(0, 40, 0.125),
                        np.arange(0, 40, 0.125) + 1e-9, [1e-12, 0.0625, 0.1875]])
    td = torch.from_numpy(t).cuda()
    out = torch.empty(8 * len(t), dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().pskel_diag_sincos(ctypes.c_void_p(td.data_ptr()), len(t),
                                           ctypes.c_void_p(out.data_ptr())))
    o = out.cpu().numpy().reshape(-1, 8)
    assert np.abs(o[:, 0] - o[:, 4]).max() < 4e-16 and np.abs(o[:, 1] - o[:, 5]).max() < 4e-16
    assert np.abs(o[:, 2] - o[:, 4]).max() < 3e-7 and np.abs(o[:, 3] - o[:, 5]).max() < 3e-7
    assert np.abs(o[:, 6] - o[:, 4]).max() < 3e-7 and np.abs(o[:, 7] - o[:, 5]).max() < 3e-7
