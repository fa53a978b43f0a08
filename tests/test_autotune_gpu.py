"""Fill-variant autotuner: the triangle-moment fill gives the same entries for every tile width,
and the autotuner picks one of the timed variants and leaves the engine compressing correctly."""
import json

import numpy as np
import pytest

from pskel import autotune
from pskel import mesh as pmesh
from pskel import octree
from pskel.engine import Engine

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sphere():
    m = pmesh.icosphere(2.0, 3)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=20)
    return m, part


@pytest.mark.parametrize("prec", ["c64", "c128"])
def test_tile_widths_agree(sphere, prec):
    m, part = sphere
    out = {}
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        r0 = np.full(eng.n_blocks, 12, dtype=np.int32)
        for cols in (0, 4, 8, 16):
            eng.set_tri_cols(cols)
            st = eng.compress(1.0, precision=prec, r0=r0, oversample=0, max_rounds=1, seed=9)
            out[cols] = [eng.get_block(b, st)[0] for b in (0, eng.n_blocks // 2, eng.n_blocks - 1)]
        with pytest.raises(RuntimeError):
            eng.set_tri_cols(5)
    bar = 1e-6 if prec == "c64" else 1e-13
    for cols in (0, 4, 16):
        for a, b in zip(out[cols], out[8]):
            assert np.abs(a - b).max() <= bar * np.abs(b).max()


def test_autotune_picks_a_variant(sphere, tmp_path):
    m, part = sphere
    cache = str(tmp_path / "tune.json")
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        rep = autotune.autotune_fill(eng, "c64", samples=16, repeats=1, include_entry=True,
                                     cache=cache, gpu_name="test")
        assert not rep["cached"]
        assert set(rep["ms"]) == {"tri0", "tri4", "tri8", "tri16", "tri32_0", "tri32_4", "tri32_8",
                                  "tri32_16", "entry0", "entry1", "entry2", "entry4"}
        best = min(rep["ms"], key=rep["ms"].get)
        assert f"{rep['choice'][0]}{rep['choice'][1]}" == best
        st = eng.compress(1e-4, precision="c64", tau=1e-7, seed=0)
        err = eng.true_errors()
        assert np.median(err) < 1e-4 and np.all(st["status"] == 0)
        rep2 = autotune.autotune_fill(eng, "c64", cache=cache, gpu_name="test")
        assert rep2["cached"] and tuple(rep2["choice"]) == tuple(rep["choice"])
    assert "test|" in next(iter(json.load(open(cache))))


def test_fp32_geometry_matches_fp64_geometry(sphere):
    """The complex-FP32 fill with FP32 pair geometry against the FP64-geometry fill and the
    errors of a compression that uses it."""
    m, part = sphere
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        r0 = np.full(eng.n_blocks, 12, dtype=np.int32)
        picks = (0, eng.n_blocks // 3, eng.n_blocks // 2, eng.n_blocks - 1)
        out = {}
        for g in (False, True):
            eng.set_fill_geometry(g)
            st = eng.compress(1.0, precision="c64", r0=r0, oversample=0, max_rounds=1, seed=4)
            out[g] = [eng.get_block(b, st)[0] for b in picks]
        ref = {}
        st = eng.compress(1.0, precision="c128", r0=r0, oversample=0, max_rounds=1, seed=4)
        ref = [eng.get_block(b, st)[0] for b in picks]
        for a, b, c in zip(out[True], out[False], ref):
            ea = np.linalg.norm(a - c) / np.linalg.norm(c)
            eb = np.linalg.norm(b - c) / np.linalg.norm(c)
            assert ea < 3e-6 and eb < 3e-6, (ea, eb)
        eng.set_fill_geometry(True)
        st = eng.compress(1e-4, precision="c64", tau=1e-7, seed=0)
        err = eng.true_errors()
        assert np.median(err) < 2e-5 and err.max() <= 1e-4


def test_pipeline_autotuner_applies_a_timed_setting():
    """The pipelined-round autotuner times the product step per chunk count and applies the
    fastest; the compression it leaves behind is unchanged (pipelining does not change results).
    The 7,680-RWG sphere has more than 2,048 blocks, so its first round is pipelined."""
    m = pmesh.icosphere(2.0, 4)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=30)
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        r0 = np.full(eng.n_blocks, 20, dtype=np.int32)
        step = lambda: eng.compress(1e-4, precision="c64", tau=1e-7, r0=r0, oversample=0,
                                    use_graph=True, seed=4)
        eng.set_pipeline(1)
        ref = step()
        out = autotune.autotune_pipeline(eng, step, chunks=(1, 2, 3), repeats=1)
        assert out["choice"] in (1, 2, 3) and set(out["ms"]) == {1, 2, 3}
        assert out["ms"][out["choice"]] == min(out["ms"].values())
        st = step()
        for f in ("r", "rank", "rounds", "est"):
            assert np.array_equal(st[f], ref[f]), f
