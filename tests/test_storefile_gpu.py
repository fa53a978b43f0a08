"""Store file written and read by the library (pskel_store_save / pskel_store_load) against the
format's numpy reader/writer (pskel/storefile.py): the saved factors are the recompressed ones
bit for bit, a reloaded context reproduces the tensor-core store matvec (to the order of its
FP32 atomic adds), a file
written by the numpy writer is byte-identical, and corrupt or mismatched files are refused."""
import numpy as np
import pytest
import torch

from pskel import _lib
from pskel import mesh as pmesh
from pskel import octree, storefile
from pskel.engine import Engine

pytestmark = pytest.mark.gpu

K, ETA = 2 * np.pi, 376.73


@pytest.fixture(scope="module")
def saved(tmp_path_factory):
    m = pmesh.icosphere(2.0, 3)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20)
    path = tmp_path_factory.mktemp("store") / "sphere.pst"
    rng = np.random.default_rng(4)
    X = torch.as_tensor((rng.standard_normal((m.N, 16)) + 1j * rng.standard_normal((m.N, 16))).astype(np.complex64),
                        device="cuda")
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        eng.compress(1e-5, precision="c128", tau=1e-10, seed=3)
        ks = eng.recompress(1e-6)
        eng.save_store(path, 1e-6)
        facs = [eng.get_recompressed(b) for b in range(eng.n_blocks)]
        eng.build_store()
        Y = eng.store_matvec(X).cpu().numpy()
        assert eng.store_status() == 0
    return m, part, path, ks, facs, X, Y


def test_saved_factors_are_the_recompressed_ones(saved):
    m, part, path, ks, facs, X, Y = saved
    d = storefile.read(path)
    assert d["N"] == m.N and np.array_equal(d["gt"], part.gt) and np.array_equal(d["gs"], part.gs)
    assert np.array_equal(d["k"], ks) and (d["mirror"] >= 0).sum() == part.n_blocks // 2
    for b, (Cp, S, Rp) in enumerate(facs):
        C2, S2, R2 = d["blocks"][b]
        assert np.array_equal(C2, Cp) and np.array_equal(S2, S) and np.array_equal(R2, Rp)


def test_reload_reproduces_store_matvec(saved, tmp_path):
    m, part, path, ks, facs, X, Y = saved
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        assert eng.load_store(path) == part.n_blocks
        for b in (0, 1, part.n_blocks // 2, part.n_blocks - 1):
            Cp, S, Rp = eng.get_recompressed(b)
            assert np.array_equal(Cp, facs[b][0]) and np.array_equal(S, facs[b][1])
            assert np.array_equal(Rp, facs[b][2])
        eng.build_store()
        Y2 = eng.store_matvec(X).cpu().numpy()
        assert eng.store_status() == 0
        # same factors, same store: equal up to the order of the FP32 atomic adds of the
        # split-K phase (not deterministic run to run)
        assert np.linalg.norm(Y2 - Y) <= 1e-6 * np.linalg.norm(Y)
        # the CUR-form matvec needs the CUR factors, which a store does not hold
        with pytest.raises(RuntimeError):
            eng.matvec(torch.zeros((m.N, 1), dtype=torch.complex128, device="cuda"))
    # the numpy writer produces the same bytes
    d = storefile.read(path)
    blocks = [(int(d["m"][b]), int(d["n"][b]), int(d["k"][b]), int(d["mirror"][b]),
               *(d["blocks"][b] if d["mirror"][b] < 0 else (None, None, None)))
              for b in range(len(d["m"]))]
    p2 = tmp_path / "numpy_written.pst"
    storefile.write(p2, d["N"], d["group_ptr"], d["group_ids"], d["gt"], d["gs"], blocks, d["thresh"])
    assert p2.read_bytes() == path.read_bytes()


def test_bad_files_refused(saved, tmp_path):
    m, part, path, *_ = saved
    raw = bytes(path.read_bytes())
    bad = tmp_path / "bad.pst"
    flipped = bytearray(raw)
    flipped[len(raw) // 2] ^= 0x10
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        for data in (bytes(flipped), raw[:-100], raw + b"\0"):
            bad.write_bytes(data)
            with pytest.raises(_lib.PskelError):
                eng.load_store(bad)
        with pytest.raises(_lib.PskelError):
            eng.load_store(tmp_path / "missing.pst")
    with Engine() as eng:
        eng.upload_mesh(pmesh.icosphere(2.0, 2), K, ETA, q=7)  # a different RWG count
        with pytest.raises(_lib.PskelError):
            eng.load_store(path)
