"""Store-file format (pskel/storefile.py, the layout pskel_store_save writes): write / read round
trip with mirrored blocks, and rejection of corrupt files."""
import numpy as np
import pytest

from pskel import storefile


def _random_store(rng):
    gp = np.array([0, 3, 7, 12], dtype=np.int32)
    gi = rng.permutation(12).astype(np.int32)
    gt = np.array([0, 2, 1, 2], dtype=np.int32)
    gs = np.array([2, 0, 2, 1], dtype=np.int32)
    sz = np.diff(gp)
    blocks = []
    for b in range(4):
        m, n = int(sz[gt[b]]), int(sz[gs[b]])
        if b == 1:  # transpose of block 0
            blocks.append((m, n, blocks[0][2], 0, None, None, None))
            continue
        k = int(rng.integers(1, min(m, n) + 1))
        Cp = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
        Rp = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
        blocks.append((m, n, k, -1, Cp, np.sort(rng.random(k))[::-1], Rp))
    return gp, gi, gt, gs, blocks


def test_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    gp, gi, gt, gs, blocks = _random_store(rng)
    p = tmp_path / "s.pst"
    storefile.write(p, 12, gp, gi, gt, gs, blocks, thresh=1e-5)
    d = storefile.read(p)
    assert d["N"] == 12 and d["thresh"] == 1e-5 and d["flags"] == 1
    for key, ref in (("group_ptr", gp), ("group_ids", gi), ("gt", gt), ("gs", gs)):
        assert np.array_equal(d[key], ref)
    for b, (m, n, k, mir, Cp, S, Rp) in enumerate(blocks):
        assert (d["m"][b], d["n"][b], d["k"][b], d["mirror"][b]) == (m, n, k, mir)
        C2, S2, R2 = d["blocks"][b]
        if mir < 0:
            assert np.array_equal(C2, Cp) and np.array_equal(S2, S) and np.array_equal(R2, Rp)
        else:  # the transpose of its primary
            _, _, _, _, Cq, Sq, Rq = blocks[mir]
            assert np.array_equal(C2, Rq.T) and np.array_equal(R2, Cq.T) and np.array_equal(S2, Sq)


def test_corrupt_files_rejected(tmp_path):
    rng = np.random.default_rng(1)
    gp, gi, gt, gs, blocks = _random_store(rng)
    p = tmp_path / "s.pst"
    storefile.write(p, 12, gp, gi, gt, gs, blocks)
    raw = bytearray(p.read_bytes())
    bad = tmp_path / "bad.pst"
    flipped = bytearray(raw)
    flipped[200] ^= 1
    for data in (bytes(flipped), bytes(raw[:-9]), b"NOTASTORE" + bytes(raw[9:])):
        bad.write_bytes(data)
        with pytest.raises(ValueError):
            storefile.read(bad)
