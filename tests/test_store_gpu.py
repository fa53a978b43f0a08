"""Tensor-core matvec over the compressed store (tcgen05, bf16 hi/lo split, FP32 accumulation)
against the FP64 product of the recompressed factors and against the dense far-field product."""
import numpy as np
import pytest
import torch

from pskel import mesh as pmesh
from pskel import octree
from pskel.engine import Engine

pytestmark = pytest.mark.gpu

K, ETA = 2 * np.pi, 376.73


@pytest.fixture(scope="module")
def compressed():
    m = pmesh.icosphere(2.0, 3)  # 1920 RWG
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20)
    eng = Engine()
    eng.upload_mesh(m, K, ETA, q=7)
    eng.set_blocks(part)
    st = eng.compress(1e-4, precision="c64", tau=1e-7, seed=3)
    ks = eng.recompress(1e-5)
    nbytes = eng.build_store()
    yield m, eng, st, ks, nbytes
    eng.close()


def _recompressed_product(eng, X):
    Y = np.zeros((eng.mesh.N, X.shape[1]), dtype=np.complex128)
    for b in range(eng.n_blocks):
        rows, cols = eng.block_ids(b)
        Cp, S, Rp = eng.get_recompressed(b)
        Y[rows] += Cp @ (S[:, None] * (Rp @ X[cols]))
    return Y


@pytest.mark.parametrize("nrhs", [16, 5, 1])
def test_store_matvec_matches_fp64_product(compressed, nrhs):
    m, eng, st, ks, nbytes = compressed
    assert nbytes > 0
    rng = np.random.default_rng(nrhs)
    X = (rng.standard_normal((m.N, nrhs)) + 1j * rng.standard_normal((m.N, nrhs))).astype(np.complex64)
    Y = eng.store_matvec(torch.as_tensor(X, device="cuda:0")).cpu().numpy()
    assert eng.store_status() == 0
    Yo = _recompressed_product(eng, X.astype(np.complex128))
    # bf16 hi + lo carries 16 mantissa bits: about 1e-5 relative
    err = np.linalg.norm(Y - Yo) / np.linalg.norm(Yo)
    assert err < 5e-5, err
    for j in range(nrhs):
        ej = np.linalg.norm(Y[:, j] - Yo[:, j]) / np.linalg.norm(Yo[:, j])
        assert ej < 1e-4, (j, ej)


def test_store_matvec_against_dense_far_field(compressed):
    m, eng, st, ks, nbytes = compressed
    rng = np.random.default_rng(11)
    X = (rng.standard_normal((m.N, 16)) + 1j * rng.standard_normal((m.N, 16))).astype(np.complex64)
    Y = eng.store_matvec(torch.as_tensor(X, device="cuda:0")).cpu().numpy()
    err_blocks = eng.true_errors()
    dev = torch.device("cuda:0")
    Yd = np.zeros((m.N, 16), dtype=np.complex128)
    for b in range(eng.n_blocks):
        rows, cols = eng.block_ids(b)
        r = torch.as_tensor(rows.astype(np.int32), device=dev)
        c = torch.as_tensor(cols.astype(np.int32), device=dev)
        Z = torch.empty((len(cols), len(rows)), dtype=torch.complex128, device=dev)
        torch.cuda.synchronize()
        eng.fill_device(r.data_ptr(), len(rows), c.data_ptr(), len(cols), Z.data_ptr(), len(rows))
        torch.cuda.synchronize()
        Yd[rows] += Z.cpu().numpy().T @ X[cols].astype(np.complex128)
    err = np.linalg.norm(Y - Yd) / np.linalg.norm(Yd)
    # compression at tol 1e-4 (every block within it), recompression at 1e-5 and the bf16
    # split: the product stays at the compression tolerance
    assert np.median(err_blocks) < 1e-5 and err_blocks.max() <= 1e-4
    assert err < 1e-4, err


def test_store_rejects_bad_calls(compressed):
    m, eng, st, ks, nbytes = compressed
    with pytest.raises(RuntimeError):
        eng.store_matvec(torch.zeros((m.N, 17), dtype=torch.complex64, device="cuda:0"))
    with Engine() as e2:
        e2.upload_mesh(m, K, ETA, q=7)
        e2.set_blocks(octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20))
        e2.compress(1e-3, precision="c64", seed=0)
        with pytest.raises(RuntimeError):
            e2.build_store()  # no recompression yet
        e2.recompress(1e-4)
        e2.build_store()
        e2.compress(1e-3, precision="c64", seed=1)
        with pytest.raises(RuntimeError):  # the store belongs to the previous compression
            e2.store_matvec(torch.zeros((m.N, 1), dtype=torch.complex64, device="cuda:0"))


@pytest.mark.parametrize("mode,bar", [("tf32", 3e-3), ("tf32x3", 1e-5), ("bf16x3", 5e-5)])
def test_store_formats_match_fp64_product(compressed, mode, bar):
    """The three operand formats of the store against the FP64 product of the recompressed
    factors: one TF32 plane (10 mantissa bits: about 5e-4), TF32 hi + lo with three products
    (about 1e-6) and bf16 hi + lo (about 1e-5). The bf16 store is built last, as the fixture
    left it."""
    m, eng, st, ks, nbytes = compressed
    nb = eng.build_store(mode)
    assert nb > 0
    if mode == "tf32x3":
        assert nb > nbytes  # two 4-byte planes against two 2-byte planes
    rng = np.random.default_rng(21)
    X = (rng.standard_normal((m.N, 16)) + 1j * rng.standard_normal((m.N, 16))).astype(np.complex64)
    Y = eng.store_matvec(torch.as_tensor(X, device="cuda:0")).cpu().numpy()
    assert eng.store_status() == 0
    Yo = _recompressed_product(eng, X.astype(np.complex128))
    err = np.linalg.norm(Y - Yo) / np.linalg.norm(Yo)
    assert err < bar, (mode, err)


def test_store_matvec_layouts_agree(compressed):
    """The strided entry point: X row-major (the tensor as it is) and column-major (through
    pskel_store_matvec with ldx), Y column-major and row-major, give the same products; Y strides
    that overlap are refused."""
    import ctypes

    from pskel import _lib
    m, eng, st, ks, nbytes = compressed
    rng = np.random.default_rng(21)
    X = (rng.standard_normal((m.N, 7)) + 1j * rng.standard_normal((m.N, 7))).astype(np.complex64)
    Xd = torch.as_tensor(X, device="cuda:0")  # row-major
    Y1 = eng.store_matvec(Xd).cpu().numpy()
    L = _lib.lib()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    ldx = m.N + 3
    Xc = torch.zeros((7, ldx), dtype=torch.complex64, device="cuda:0")
    Xc[:, :m.N] = Xd.t()
    Yc = torch.zeros((7, ldx), dtype=torch.complex64, device="cuda:0")
    _lib.check(L.pskel_store_matvec(eng._h, vp(Xc), ldx, vp(Yc), ldx, 7, None))
    Yr = torch.zeros((m.N, 7), dtype=torch.complex64, device="cuda:0")
    _lib.check(L.pskel_store_matvec_strided(eng._h, vp(Xd), 7, 1, vp(Yr), 7, 1, 7, None))
    torch.cuda.synchronize()
    # the same products; the phase-2 FP32 atomics add K slices in run-dependent order
    for Y2 in (Yc[:, :m.N].t().cpu().numpy(), Yr.cpu().numpy()):
        assert np.linalg.norm(Y2 - Y1) <= 1e-6 * np.linalg.norm(Y1)
    with pytest.raises(_lib.PskelError):  # Y rows overlapping
        _lib.check(L.pskel_store_matvec_strided(eng._h, vp(Xd), 7, 1, vp(Yr), 3, 1, 7, None))
