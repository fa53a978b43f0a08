"""Symmetric mode: only one block of each (t, s) / (s, t) pair is compressed and the other is its
transpose. Every block, mirrors included, is checked against its own dense FP64 fill, and the
matvec, recompression and store paths treat mirrors as transposes."""
import numpy as np
import pytest
import torch

from oracle import cur_oracle as co
from pskel import mesh as pmesh
from pskel import octree
from pskel.engine import Engine

pytestmark = pytest.mark.gpu

K, ETA = 2 * np.pi, 376.73


@pytest.fixture(scope="module")
def sphere():
    m = pmesh.icosphere(2.0, 3)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20)
    return m, part


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_mirror_blocks(sphere, prec):
    m, part = sphere
    tol = 1e-4
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        st = eng.compress(tol, precision=prec, tau=1e-7, seed=1)
        timing = eng.timing()
        err = eng.true_errors()  # each block against its own dense fill
        mir = eng.mirror_of()
        assert np.all(mir >= 0)  # every far pair comes with its transpose
        for b in range(eng.n_blocks):
            p = mir[b]
            assert st["m"][b] == st["n"][p] and st["n"][b] == st["m"][p]
            assert st["r"][b] == st["r"][p] and st["est"][b] == st["est"][p]
        # mirror error equals the primary's (Z symmetric to rounding); blocks sampled on their
        # whole smaller side reproduce Z to ~1e-9, where the two dense fills' roundings, through
        # the core's inverse, set the difference
        np.testing.assert_allclose(err, err[mir], rtol=1e-6, atol=1e-7)
        assert np.median(err) < tol and err.max() <= tol
        # factors of a mirror are the transposes, with swapped samples
        b = int(np.argmax(mir < np.arange(eng.n_blocks)))  # a block whose partner is primary
        p = mir[b]
        C, U, R, I, J = eng.get_block(b, st)
        Cp, Up, Rp, Ip, Jp = eng.get_block(p, st)
        assert np.array_equal(I, Jp) and np.array_equal(J, Ip)
        np.testing.assert_array_equal(C, Rp.T)
        np.testing.assert_array_equal(U, Up.T)
        np.testing.assert_array_equal(R, Cp.T)
        # half of the fill work
        with Engine() as e2:
            e2.upload_mesh(m, K, ETA, q=7)
            e2.set_blocks(part)
            e2.compress(tol, precision=prec, tau=1e-7, seed=1)
            full = e2.timing()
        assert timing["fill_entries"] < 0.6 * full["fill_entries"]


def test_mirror_matvec_recompress_store(sphere):
    m, part = sphere
    rng = np.random.default_rng(3)
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        st = eng.compress(1e-4, precision="c64", tau=1e-7, seed=2)
        X = rng.standard_normal((m.N, 4)) + 1j * rng.standard_normal((m.N, 4))
        Y = eng.matvec(torch.as_tensor(X.astype(np.complex64), device="cuda:0")).cpu().numpy()
        Yo = np.zeros_like(X)
        scale = 0.0
        for b in range(eng.n_blocks):
            rows, cols = eng.block_ids(b)
            C, U, R, _, _ = eng.get_block(b, st)
            Yo[rows] += co.compressed_matvec(C, U, R, X[cols])
            scale += np.linalg.norm(C, 2) * np.linalg.norm(U, 2) * np.linalg.norm(R, 2) * np.linalg.norm(X[cols])
        assert np.linalg.norm(Y - Yo) < 6e-6 * scale
        ks = eng.recompress(1e-5)
        mir = eng.mirror_of()
        assert np.array_equal(ks, ks[mir])
        for b in (0, eng.n_blocks // 2, eng.n_blocks - 1):
            C, U, R, _, _ = eng.get_block(b, st)
            Cp, S, Rp = eng.get_recompressed(b)
            A = C @ U @ R
            scale = np.linalg.norm(C, 2) * np.linalg.norm(U, 2) * np.linalg.norm(R, 2)
            assert np.linalg.norm((Cp * S) @ Rp - A) < 2e-5 * np.linalg.norm(A) + 1e-10 * scale
        eng.build_store()
        X16 = (rng.standard_normal((m.N, 16)) + 1j * rng.standard_normal((m.N, 16))).astype(np.complex64)
        Ys = eng.store_matvec(torch.as_tensor(X16, device="cuda:0")).cpu().numpy()
        assert eng.store_status() == 0
        Yr = np.zeros((m.N, 16), dtype=np.complex128)
        for b in range(eng.n_blocks):
            rows, cols = eng.block_ids(b)
            Cp, S, Rp = eng.get_recompressed(b)
            Yr[rows] += Cp @ (S[:, None] * (Rp @ X16[cols].astype(np.complex128)))
        assert np.linalg.norm(Ys - Yr) / np.linalg.norm(Yr) < 5e-5
