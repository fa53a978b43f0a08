"""Operations on the compressed blocks: the far-field matvec Y = sum_b C_b U_b R_b X(cols_b)
(the reference's C(U(Rv)), cu1:1929-1960, over all blocks and many right-hand sides) and the
recompression of every C U R into an SVD-truncated C' S R' (svd_compress.m:19-33), both checked
against the oracle on the factors the engine kept."""
import numpy as np
import pytest
import torch

from oracle import cur_oracle as co
from pskel import _lib
from pskel import mesh as pmesh
from pskel import octree
from pskel.engine import Engine

pytestmark = pytest.mark.gpu

K, ETA = 2 * np.pi, 376.73


@pytest.fixture(scope="module")
def sphere():
    m = pmesh.icosphere(2.0, 3)  # 1280 triangles, 1920 RWG
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20)
    return m, part


def _factor_product(eng, st, X):
    """sum_b C_b (U_b (R_b X(cols_b))) scattered into rows_b, in FP64 on the host, and the
    rounding-error scale sum_b ||C_b|| ||U_b|| ||R_b|| ||X(cols_b)|| (the product runs through
    the inverse of an ill-conditioned core, so its rounding error is relative to this scale,
    not to ||Y||)."""
    Y = np.zeros((eng.mesh.N, X.shape[1]), dtype=np.complex128)
    scale = 0.0
    for b in range(eng.n_blocks):
        rows, cols = eng.block_ids(b)
        C, U, R, _, _ = eng.get_block(b, st)
        Y[rows] += co.compressed_matvec(C, U, R, X[cols])
        scale += (np.linalg.norm(C, 2) * np.linalg.norm(U, 2) * np.linalg.norm(R, 2)
                  * np.linalg.norm(X[cols]))
    return Y, scale


def _dense_far_product(eng, X):
    """sum_b Z_b X(cols_b) with Z_b filled densely in FP64 on the device."""
    dev = torch.device("cuda:0")
    Y = np.zeros((eng.mesh.N, X.shape[1]), dtype=np.complex128)
    for b in range(eng.n_blocks):
        rows, cols = eng.block_ids(b)
        r = torch.as_tensor(rows.astype(np.int32), device=dev)
        c = torch.as_tensor(cols.astype(np.int32), device=dev)
        Z = torch.empty((len(cols), len(rows)), dtype=torch.complex128, device=dev)
        torch.cuda.synchronize()
        eng.fill_device(r.data_ptr(), len(rows), c.data_ptr(), len(cols), Z.data_ptr(), len(rows))
        torch.cuda.synchronize()
        Zh = Z.cpu().numpy().T  # column-major m x n
        Y[rows] += Zh @ X[cols]
    return Y


@pytest.mark.parametrize("nrhs", [1, 16])
def test_matvec_matches_factors_c128(sphere, nrhs):
    m, part = sphere
    rng = np.random.default_rng(7)
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        st = eng.compress(1e-6, precision="c128", tau=1e-10, seed=2)
        X = rng.standard_normal((m.N, nrhs)) + 1j * rng.standard_normal((m.N, nrhs))
        Xd = torch.as_tensor(X, device="cuda:0")
        Y = eng.matvec(Xd).cpu().numpy()
        Yo, scale = _factor_product(eng, st, X)
    # FP64: a few hundred accumulated roundings of size eps relative to the scale
    assert np.linalg.norm(Y - Yo) < 1e-13 * scale, (np.linalg.norm(Y - Yo), scale)
    assert np.linalg.norm(Y - Yo) / np.linalg.norm(Yo) < 1e-6


def test_matvec_matches_factors_c64(sphere):
    m, part = sphere
    rng = np.random.default_rng(8)
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        st = eng.compress(1e-4, precision="c64", tau=1e-7, seed=2)
        X = rng.standard_normal((m.N, 16)) + 1j * rng.standard_normal((m.N, 16))
        Xd = torch.as_tensor(X.astype(np.complex64), device="cuda:0")
        Y = eng.matvec(Xd).cpu().numpy()
        Yo, scale = _factor_product(eng, st, X.astype(np.complex64).astype(np.complex128))
    # FP32 arithmetic: rounding of size eps32 = 6e-8 relative to the scale
    assert np.linalg.norm(Y - Yo) < 6e-6 * scale, (np.linalg.norm(Y - Yo), scale)


def test_matvec_against_dense_far_field(sphere):
    """The compressed product against the dense far-field product: within the compression
    tolerance (each block's relative error is below it)."""
    m, part = sphere
    tol = 1e-5
    rng = np.random.default_rng(9)
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        eng.compress(tol, precision="c128", tau=1e-10, seed=4)
        err = eng.true_errors()
        X = rng.standard_normal((m.N, 4)) + 1j * rng.standard_normal((m.N, 4))
        Y = eng.matvec(torch.as_tensor(X, device="cuda:0")).cpu().numpy()
        Yd = _dense_far_product(eng, X)
    assert err.max() <= tol
    assert np.linalg.norm(Y - Yd) / np.linalg.norm(Yd) < 2 * err.max()


def test_dense_far_matvec_matches_blockwise_product(sphere):
    """The library's dense reference product (every far block filled in FP64 and applied on the
    device) against the block-by-block product of dense fills on the host."""
    m, part = sphere
    rng = np.random.default_rng(13)
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        X = rng.standard_normal((m.N, 3)) + 1j * rng.standard_normal((m.N, 3))
        Y = eng.dense_far_matvec(torch.as_tensor(X, device="cuda:0")).cpu().numpy()
        Yd = _dense_far_product(eng, X)
    assert np.linalg.norm(Y - Yd) / np.linalg.norm(Yd) < 1e-12


def test_matvec_rejects_bad_calls(sphere):
    m, part = sphere
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        X = torch.zeros((m.N, 1), dtype=torch.complex128, device="cuda:0")
        with pytest.raises(RuntimeError):
            eng.matvec(X)  # nothing compressed yet
        eng.compress(1e-3, precision="c128", seed=0)
        with pytest.raises(RuntimeError):
            eng.matvec(torch.zeros((m.N, 65), dtype=torch.complex128, device="cuda:0"))
        lib = _lib.lib()
        assert lib.pskel_matvec(eng._h, None, m.N, None, m.N, 1, 0, None) == -1


# split path (tensor-core products of TF32 hi + lo operands, FP32 accumulation): its singular
# values and factors carry errors of ~1e-6 of the largest singular value, its trailing-term cut
# moves a singular value by at most 1e-2 thresh s_0 and its truncated core SVD by at most
# 0.25 thresh s_0; the bars allow 2e-5 s_0 + 0.3 thresh s_0 and an orthonormality defect of 1e-5
SPLIT_S_BAR = 2e-5
SPLIT_S_THRESH = 0.3
SPLIT_ORTH_BAR = 1e-5


@pytest.mark.parametrize("prec,tol,path", [("c128", 1e-7, "auto"), ("c64", 1e-4, "fp64"),
                                           ("c64", 1e-4, "split"), ("c64", 1e-3, "split")])
def test_recompress_matches_oracle(sphere, prec, tol, path):
    """Device recompression against the oracle's QR-based one on the same factors. C U R is
    formed from an ill-conditioned core inverse, so both results carry rounding errors of
    order eps ||C|| ||U|| ||R||: the comparisons are scaled by that product. The split path
    adds its FP32-level product errors (relative to the largest singular value)."""
    m, part = sphere
    thresh = tol / 10
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        st = eng.compress(tol, precision=prec, tau=1e-8 if prec == "c128" else 1e-7, seed=5)
        ks = eng.recompress(thresh, path=path)
        split = eng.recompress_split_blocks()
        if path == "split":
            # every core has rank <= 64 here; the blocks whose pinv kept values far below tau
            # (full sample count, common on this small sphere) go to the FP64 path
            assert 0 < split < eng.n_blocks
        else:
            assert split == 0
        assert np.all(ks >= 1) and np.all(ks <= st["r"])
        nb = eng.n_blocks
        for b in sorted(set([0, 1, nb // 3, nb // 2, nb - 1])):
            C, U, R, _, _ = eng.get_block(b, st)
            Cp, S, Rp = eng.get_recompressed(b)
            Co, So, Ro = co.svd_compress(C, U, R, thresh)
            so = np.diag(So)
            A = C @ U @ R
            scale = np.linalg.norm(C, 2) * np.linalg.norm(U, 2) * np.linalg.norm(R, 2)
            bar = 1e-12 * scale
            s_all = np.linalg.svd(A, compute_uv=False)
            if path == "split":
                bar += (SPLIT_S_BAR + SPLIT_S_THRESH * thresh) * s_all[0]
            # the kept count agrees with the oracle unless a value lies within rounding of the
            # threshold
            if len(so) != len(S):
                edge = s_all[min(len(so), len(S))]
                assert abs(edge - thresh * s_all[0]) < 10 * bar, (b, len(so), len(S))
            kk = min(len(so), len(S))
            assert np.abs(S[:kk] - so[:kk]).max() < bar, (b, np.abs(S[:kk] - so[:kk]).max(), scale)
            B = (Cp * S) @ Rp
            Bo = Co @ So @ Ro
            nA = np.linalg.norm(A)
            assert np.linalg.norm(B - Bo) < 2 * thresh * nA + 10 * bar * np.sqrt(kk)
            assert np.linalg.norm(B - A) < 2 * thresh * nA + 10 * bar * np.sqrt(kk)
            # orthonormal factors
            orth = SPLIT_ORTH_BAR if path == "split" else 1e-9
            assert np.abs(Cp.conj().T @ Cp - np.eye(len(S))).max() < orth
            assert np.abs(Rp @ Rp.conj().T - np.eye(len(S))).max() < orth


def test_recompress_split_matches_fp64(sphere):
    """The split tensor-core path and the FP64 path on the same complex-FP32 compression:
    equal ranks (up to values within the split path's error of the threshold) and products
    C' S R' that agree to the split path's error, block by block; the default path at
    thresh 1e-5 is the split one (but for blocks kept to core values below 1e-7 of the
    largest), at 1e-6 the FP64 one."""
    m, part = sphere
    thresh = 1e-5
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        st = eng.compress(1e-4, precision="c64", tau=1e-7, seed=3)
        k64 = eng.recompress(thresh, path="fp64")
        f64 = [eng.get_recompressed(b) for b in range(eng.n_blocks)]
        ks = eng.recompress(thresh, path="auto")
        assert eng.recompress_split_blocks() > 0
        assert np.abs(ks - k64).max() <= 1 and np.mean(ks == k64) > 0.95
        worst = 0.0
        for b in range(eng.n_blocks):
            Cp, S, Rp = eng.get_recompressed(b)
            Cq, Sq, Rq = f64[b]
            P, Q = (Cp * S) @ Rp, (Cq * Sq) @ Rq
            worst = max(worst, np.linalg.norm(P - Q, 2) / Sq[0])
        assert worst < 5 * thresh, worst
        eng.recompress(1e-6, path="auto")
        assert eng.recompress_split_blocks() == 0
        eng.recompress(1e-4, path="fp64")
        assert eng.recompress_split_blocks() == 0
        eng.recompress(1e-4, path="split")
        assert eng.recompress_split_blocks() > 0
