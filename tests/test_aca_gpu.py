"""Batched device ACA (pskel_aca_compress) against the restatement of the reference's
ACA_julia (oracle/aca_oracle.py) driven by the oracle's element fill on the same blocks: the
same pivot rows and columns, ranks and stop reasons, factors to 1e-9 of the block; every block's
error against its dense FP64 fill; the symmetric mode's transposed blocks; argument checks."""
import numpy as np
import pytest

from oracle import aca_oracle as ao
from oracle import element as el
from pskel import _lib
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


@pytest.mark.parametrize("tol", [1e-3, 1e-5])
def test_aca_matches_oracle(sphere, tol):
    m, part = sphere
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        out = eng.aca_compress(tol)
        err = eng.aca_true_errors()
        nb = eng.n_blocks
        picks = sorted(set([0, 1, 7, nb // 3, nb // 2, nb - 1]))
        for b in picks:
            rows, cols = eng.block_ids(b)
            Z = el.fill(m, rows + 1, cols + 1, K, ETA, 7, 7)
            ref = ao.aca(lambda i: Z[i], lambda j: Z[:, j], len(rows), len(cols), tol, kmax=128)
            U, V, I, J = eng.aca_get_block(b)
            assert out["k"][b] == ref["k"] and out["status"][b] == ref["status"], b
            assert np.array_equal(I, ref["I"]) and np.array_equal(J, ref["J"]), b
            nz = np.linalg.norm(Z)
            assert np.linalg.norm(U @ V - ref["U"] @ ref["V"]) < 1e-9 * nz
            e = np.linalg.norm(Z - U @ V) / nz
            assert abs(e - err[b]) <= 1e-6 * e + 1e-13
    # the stopping rule is an estimate: the errors sit near tol
    assert np.median(err) < tol and err.max() < 30 * tol


def test_aca_symmetric_mirrors(sphere):
    m, part = sphere
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        out = eng.aca_compress(1e-4)
        err = eng.aca_true_errors()
        pos = {(t, s): b for b, (t, s) in enumerate(zip(part.gt, part.gs))}
        checked = 0
        for b, (t, s) in enumerate(zip(part.gt, part.gs)):
            p = pos[(s, t)]
            if p < b:
                Ub, Vb, Ib, Jb = eng.aca_get_block(b)
                Up, Vp, Ip, Jp = eng.aca_get_block(p)
                assert np.array_equal(Ub, Vp.T) and np.array_equal(Vb, Up.T)
                assert np.array_equal(Ib, Jp) and np.array_equal(Jb, Ip)
                assert out["k"][b] == out["k"][p]
                assert abs(err[b] - err[p]) <= 1e-6 * err[p] + 1e-14  # Z = Z^T
                checked += 1
                if checked > 20:
                    break
        assert checked > 0


def test_aca_arguments(sphere):
    m, part = sphere
    lib = _lib.lib()
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        assert lib.pskel_aca_compress(eng._h, 0.0, 64, None, None) == -1
        assert lib.pskel_aca_compress(eng._h, 1e-3, 0, None, None) == -1
        out = eng.aca_compress(1e-6, kmax=4)  # rank cap
        assert out["k"].max() <= 4 and (out["status"] == 1).all()
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=1)
        eng.set_blocks(part)
        assert lib.pskel_aca_compress(eng._h, 1e-3, 64, None, None) == -1  # 7-point rule only
