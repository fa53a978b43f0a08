"""Seeded index sampler: Philox4x32-10 known-answer vectors (Random123 kat_vectors) and the
properties of the Floyd draw."""
import numpy as np
import pytest

from oracle import element as el

KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,out", KAT)
def test_philox_kat(ctr, key, out):
    assert el.philox4(ctr, key) == out


@pytest.mark.parametrize("r,D", [(0, 5), (1, 1), (3, 3), (7, 100), (64, 600), (600, 600)])
def test_sample_sorted_distinct(r, D):
    s = el.sample(r, D, 17, 2, 0, 12345)
    assert len(s) == r
    assert np.all(np.diff(s) > 0)
    assert (r == 0) or (s[0] >= 0 and s[-1] < D)


def test_sample_reproducible_and_stream_dependent():
    a = el.sample(20, 200, 3, 0, 0, 0)
    assert np.array_equal(a, el.sample(20, 200, 3, 0, 0, 0))
    assert not np.array_equal(a, el.sample(20, 200, 3, 0, 1, 0))
    assert not np.array_equal(a, el.sample(20, 200, 4, 0, 0, 0))
    assert not np.array_equal(a, el.sample(20, 200, 3, 1, 0, 0))


def test_sample_uniform_marginals():
    counts = np.zeros(50)
    for b in range(2000):
        counts[el.sample(10, 50, b, 0, 0, 7)] += 1
    expected = 2000 * 10 / 50
    assert np.abs(counts - expected).max() < 5 * np.sqrt(expected)


def test_sample_extra_avoids_I():
    I = el.sample(30, 100, 1, 0, 0, 9)
    x = el.sample_extra(10, I, 100, 1, 0, 9)
    assert len(x) == 10 and not set(x) & set(I)
    assert np.all(np.diff(x) > 0)
    # fewer free rows than requested
    I2 = np.arange(95, dtype=np.int32)
    x2 = el.sample_extra(10, I2, 100, 1, 0, 9)
    assert sorted(x2) == [95, 96, 97, 98, 99]
    assert len(el.sample_extra(10, np.arange(100, dtype=np.int32), 100, 1, 0, 9)) == 0


def test_sample_rejects_r_above_D():
    with pytest.raises(ValueError):
        el.sample(6, 5, 0, 0, 0, 0)


def test_recheck_samples_avoid_every_earlier_sample():
    """The re-check of a block draws its new extra rows outside I and the first extra rows
    (stream 4), so the pooled estimate never counts a row twice."""
    I = el.sample(30, 120, 7, 1, 0, 3)
    Ix = el.sample_extra(16, I, 120, 7, 1, 3, stream=2)
    Ix2 = el.sample_extra(16, np.union1d(I, Ix), 120, 7, 1, 3, stream=4)
    assert len(Ix2) == 16 and np.all(np.diff(Ix2) > 0)
    assert not set(Ix2) & (set(I) | set(Ix))
    # the free rows run out: only what is left
    J = np.arange(100, dtype=np.int32)
    Jx = np.arange(100, 110, dtype=np.int32)
    assert list(el.sample_extra(16, np.union1d(J, Jx), 120, 7, 1, 3, stream=5)) == list(range(110, 120))
