"""Near-field element rule on the device against the near-field oracle and the reference's
shipped routine (golden blocks, tests/golden/make_golden.py near):
- the reference-named fill (impedance_matrix_cuda_elbyel4 via api.user_impedance_cuda5) with
  the integration radii switched on: every entry without a same-triangle pair equals the
  shipped routine's to 1e-12 of the block's largest entry, every entry the oracle's to 1e-11;
- the handle API's near fill (pskel_fill_near_device) against the oracle for several radii and
  both outside-radius rules (centroid, 7-point);
- requests with no near pair keep the centroid-rule path (bit-identical to radii 0)."""
import glob
import os

import numpy as np
import pytest
import torch

from oracle import element as el
from pskel import api
from pskel import mesh as pmesh
from pskel.engine import Engine
from test_near_oracle import _mesh_from, shared_triangle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
NEAR = sorted(glob.glob(os.path.join(GOLDEN, "near_*.npz")))


@pytest.mark.parametrize("path", NEAR, ids=os.path.basename)
def test_reference_named_fill_near(path):
    d = np.load(path)
    m = _mesh_from(d)
    rs, ra, rf = (float(x) for x in d["radii"])
    k, eta = float(d["k"]), float(d["eta"])
    em = api.EMData(2 * np.pi / k, k, eta, 1, rs, rf, ra, 0, 0)
    Z, _ = api.user_impedance_cuda5(d["rows"], d["cols"], m, em)
    ref = d["Z"]
    share = shared_triangle(m, d["rows"], d["cols"])
    scale = np.abs(ref).max()
    assert np.abs(Z - ref)[~share].max() < 1e-12 * scale
    Zo = el.fill_near(m, d["rows"], d["cols"], k, eta, rs, ra, rf)
    assert np.abs(Z - Zo).max() < 1e-11 * scale


def _device_near(eng, rows0, cols0, radii, q_far):
    dev = torch.device("cuda:0")
    r = torch.as_tensor(np.asarray(rows0, dtype=np.int32), device=dev)
    c = torch.as_tensor(np.asarray(cols0, dtype=np.int32), device=dev)
    Z = torch.empty((len(cols0), len(rows0)), dtype=torch.complex128, device=dev)
    torch.cuda.synchronize()
    eng.fill_near_device(r.data_ptr(), len(rows0), c.data_ptr(), len(cols0), Z.data_ptr(),
                         len(rows0), *radii, q_far=q_far)
    torch.cuda.synchronize()
    return Z.cpu().numpy().T


@pytest.mark.parametrize("q_far", [1, 7])
def test_handle_near_fill_matches_oracle(q_far):
    k, eta = 2 * np.pi, 376.73
    for m in (pmesh.icosphere(1.0, 3), pmesh.two_plates(1.0, 12, 3.0)):
        c = m.basis_centres().T
        rng = np.random.default_rng(3)
        rows0 = np.sort(rng.choice(m.N, 64, replace=False))
        d = np.linalg.norm(c[:, None, :] - c[None, rows0, :], axis=2).min(axis=1)
        cols0 = np.sort(np.argsort(d, kind="stable")[:96])
        with Engine() as eng:
            eng.upload_mesh(m, k, eta, q=7)
            for radii in ((0.3, 0.3, 0.3), (0.2, 0.0, 0.25), (0.0, 0.4, 0.0), (0.0, 0.0, 0.0)):
                Z = _device_near(eng, rows0, cols0, radii, q_far)
                Zo = el.fill_near(m, rows0 + 1, cols0 + 1, k, eta, *radii, q_far=q_far)
                assert np.abs(Z - Zo).max() < 1e-11 * np.abs(Zo).max(), (radii, q_far)


def test_far_request_keeps_centroid_path():
    """Radii that no triangle pair falls inside: the result is the centroid rule's, bit for bit
    (the near kernel is not launched)."""
    m = pmesh.two_spheres(1.0, 12.0, 48)
    em0 = api.EMData.for_wavelength(2.0, rint=0.0)
    em1 = api.EMData.for_wavelength(2.0, rint=1.0)
    Z0, _ = api.user_impedance_cuda5(np.arange(1, 49), np.arange(49, 97), m, em0)
    Z1, _ = api.user_impedance_cuda5(np.arange(1, 49), np.arange(49, 97), m, em1)
    assert np.array_equal(Z0, Z1)
