"""Handle API: device sampler bit-parity with the oracle, batched fills against the oracle,
and per-block errors of the batched compression against dense FP64 fills."""
import numpy as np
import pytest

from oracle import cur_oracle as co
from oracle import element as el
from pskel import mesh as pmesh
from pskel import octree
from pskel.engine import Engine

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_sphere():
    m = pmesh.icosphere(2.0, 3)  # 1280 triangles, 1920 RWG
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20)
    return m, part


def test_sampler_and_fill_parity(small_sphere):
    m, part = small_sphere
    k, eta = 2 * np.pi, 376.73
    with Engine() as eng:
        eng.upload_mesh(m, k, eta, q=7)
        eng.set_blocks(part)
        nb = eng.n_blocks
        r0 = np.full(nb, 6, dtype=np.int32)
        st = eng.compress(1.0, precision="c128", r0=r0, oversample=4, seed=1234, max_rounds=1)
        assert np.all(st["r"] == np.minimum(10, np.minimum(st["m"], st["n"])))
        for b in list(range(0, nb, max(1, nb // 7)))[:7]:
            rows, cols = eng.block_ids(b)
            C, U, R, I, J = eng.get_block(b, st)
            r = st["r"][b]
            assert np.array_equal(I, el.sample(r, len(rows), b, 0, 0, 1234))
            assert np.array_equal(J, el.sample(r, len(cols), b, 0, 1, 1234))
            Co = el.fill(m, rows + 1, cols[J] + 1, k, eta, 7, 7)
            Ro = el.fill(m, rows[I] + 1, cols + 1, k, eta, 7, 7)
            assert np.abs(C - Co).max() / np.abs(Co).max() < 1e-12
            assert np.abs(R - Ro).max() / np.abs(Ro).max() < 1e-12
            Uo = co.my_pinv(Co[I, :], 1e-8, relative=True)
            assert np.linalg.norm(C @ U @ R - Co @ Uo @ Ro) / np.linalg.norm(Co @ Uo @ Ro) < 1e-6


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_batched_compression_errors(small_sphere, prec):
    m, part = small_sphere
    tol = 1e-4
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        st = eng.compress(tol, precision=prec, tau=1e-7, seed=0, est_safety=2.0)
        assert np.all(st["status"] == 0)
        err = eng.true_errors()
    assert np.all(np.isfinite(err))
    assert np.median(err) < tol
    assert np.max(err) <= tol, np.max(err)
    # every block met the estimate's threshold or was sampled on its whole smaller side
    ok = (st["est"] <= tol / 2) | (st["r"] == np.minimum(st["m"], st["n"]))
    assert np.all(ok)


def test_true_error_matches_oracle(small_sphere):
    m, part = small_sphere
    k, eta = 2 * np.pi, 376.73
    with Engine() as eng:
        eng.upload_mesh(m, k, eta, q=7)
        eng.set_blocks(part)
        st = eng.compress(1e-3, precision="c128", tau=1e-6, seed=3)
        err = eng.true_errors()
        for b in (0, eng.n_blocks // 2, eng.n_blocks - 1):
            rows, cols = eng.block_ids(b)
            C, U, R, I, J = eng.get_block(b, st)
            Z = el.fill(m, rows + 1, cols + 1, k, eta, 7, 7)
            e = co.rel_fro_error(Z, C, U, R)
            # forming C U R rounds at eps |C| |U| |R| (U inverts an ill-conditioned core); the
            # two errors agree to that scale (relative to |Z|) or to 1e-6 of themselves
            scale = (np.linalg.norm(C, 2) * np.linalg.norm(U, 2) * np.linalg.norm(R, 2)
                     / np.linalg.norm(Z))
            assert abs(e - err[b]) <= 1e-6 * e + 1e-13 * scale + 1e-15, (b, e, err[b], scale)


def test_adaptive_rounds_match_oracle(small_sphere):
    """The device adaptive loop takes the same sample counts and rounds as the oracle's
    restatement (same Philox index sets, same randomized estimate and acceptance rule)."""
    m, part = small_sphere
    k, eta = 2 * np.pi, 376.73
    tol, tau, seed = 1e-4, 1e-7, 11
    with Engine() as eng:
        eng.upload_mesh(m, k, eta, q=7)
        eng.set_blocks(part)
        st = eng.compress(tol, precision="c128", tau=tau, seed=seed, extra_rows=16,
                          extra_cols=16, est_safety=2.0)
        for b in (1, eng.n_blocks // 3, eng.n_blocks - 2):
            rows, cols = eng.block_ids(b)
            fill = lambda a, c: el.fill(m, a, c, k, eta, 7, 7)
            o = co.plain_adaptive(fill, rows + 1, cols + 1, tol, b, seed, extra_rows=16,
                                  extra_cols=16, safety=2.0, tau=tau)
            assert st["r"][b] == o["r"] and st["rounds"][b] == o["rounds"], (b, st[b], o["r"], o["rounds"])
            # estimates agree to rounding (those near 1e-11 are FP64 noise of a converged CUR)
            assert abs(st["est"][b] - o["est"]) <= 1e-6 * o["est"] + 1e-9
            C, U, R, I, J = eng.get_block(b, st)
            assert np.array_equal(I, o["I"]) and np.array_equal(J, o["J"])


@pytest.mark.parametrize("prec,bar", [("c128", 1e-12), ("c64", 2e-6)])
def test_fill_variants_agree(small_sphere, prec, bar):
    """The triangle-moment fill, the two-rows-per-thread fill and the shuffle-split fill give
    the same C and R for the same samples."""
    m, part = small_sphere
    out = {}
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        for v in (8, 0, 2):
            eng.set_fill_split(split_c128=v, split_c64=v)
            st = eng.compress(1.0, precision=prec, r0=np.full(eng.n_blocks, 12), oversample=0,
                              max_rounds=1, seed=5)
            out[v] = [eng.get_block(b, st)[:3] for b in (0, eng.n_blocks // 2)]
    for v in (0, 2):
        for (C, U, R), (C8, U8, R8) in zip(out[v], out[8]):
            assert np.abs(C - C8).max() <= bar * np.abs(C8).max()
            assert np.abs(R - R8).max() <= bar * np.abs(R8).max()


def test_pipelined_round_gives_the_same_result():
    """A pipelined round (fill of chunk k + 1 beside the SVD, pinv and estimate of chunk k) runs
    the same kernels on the same data as the unpipelined one: identical sample counts, rounds,
    estimates and factors, with and without the graph replay of the first round."""
    m = pmesh.icosphere(2.0, 4)  # 7,680 RWG, 22,312 blocks: above the pipelining threshold
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=30)
    out = {}
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        for chunks in (1, 4, 3):
            eng.set_pipeline(chunks)
            for graph in (False, True, True):  # eager, capture, replay
                st = eng.compress(1e-4, precision="c64", tau=1e-7, seed=6, use_graph=graph)
            picks = (0, 7777, eng.n_blocks - 1)
            out[chunks] = (st, [eng.get_block(b, st) for b in picks])
    for chunks in (4, 3):
        st, blocks = out[chunks]
        st1, blocks1 = out[1]
        for k in ("r", "rounds", "rank", "est"):
            np.testing.assert_array_equal(st[k], st1[k])
        for f, f1 in zip(blocks, blocks1):
            for a, b in zip(f, f1):
                np.testing.assert_array_equal(a, b)
