"""Host-side logic of the engine wrapper (no device calls)."""
import ctypes

import numpy as np

from pskel import _lib
from pskel.engine import STAT_DTYPE, stats_array


def test_stat_layout_matches_c():
    assert ctypes.sizeof(_lib.BlockStat) == STAT_DTYPE.itemsize == 40
    st = (_lib.BlockStat * 3)()
    for i in range(3):
        st[i].m, st[i].n, st[i].r, st[i].rank, st[i].rounds, st[i].status, st[i].est = \
            10 + i, 20 + i, 5, 4, 2, -3 * i, 1.5e-4 * i
    a = stats_array(st)
    assert list(a["m"]) == [10, 11, 12] and list(a["status"]) == [0, -3, -6]
    np.testing.assert_allclose(a["est"], [0, 1.5e-4, 3e-4])


def test_opts_layout():
    # pskel_opts_t: 2 doubles, 8 ints, uint64, 2 doubles, 2 ints, 2 doubles
    assert ctypes.sizeof(_lib.Opts) == 96
    assert _lib.Opts.est_verify.offset == 80 and _lib.Opts.full_tau.offset == 88
    assert ctypes.sizeof(_lib.EM) == 24


def test_roofline_work_counts():
    """The fixed work conventions of the roofline numerators."""
    from pskel import roofline
    assert roofline.FLOPS_PER_PAIR == 32
    assert roofline.fill_flops(10) == 320
    assert roofline.pinv_flops([2]) == 92 * 8
    assert roofline.matvec_flops([4], [5], [3], 2) == 8 * 2 * (12 + 9 + 15)
    # 30 factor entries of 8 bytes, 9 core entries of 16 bytes, 2 x 9 vector entries of 8 bytes
    assert roofline.matvec_bytes([4], [6], [3], 2, 8.0, 16.0) == 30 * 8 + 9 * 16 + 2 * 10 * 8
    assert roofline.recompress_flops([4], [6], [2], [1]) == 8 * (2 * 4 * 4 + 2 * 6 * 4) + 84 * 8 + 8 * 10 * 2
    # store: (4 + 6) x 3 factor entries of 8 bytes; X and Y (N = 20) and T (2 x 3) for 2 sides
    assert roofline.store_matvec_bytes([4], [6], [3], 20, 2) == 30 * 8 + 2 * 8 * (40 + 6)


def test_balanced_tile_width_rule():
    """The per-job tile width of the triangle-moment fill: items = triangles x width fill the
    256 threads of a CTA best (restated here in Python against the rule's examples)."""
    def width(nt, most=16):
        best, best_eff = most, -1.0
        for c in range(most, 3, -1):
            items = nt * c
            eff = items / (-(-items // 256) * 256)
            if eff > best_eff + 1e-9:
                best, best_eff = c, eff
        return best
    assert width(100) == 15      # 1500 of 1536 slots (as good as 10, and wider)
    assert width(128) == 16      # 2048 = 8 x 256 exactly
    assert width(64) == 16       # 1024
    assert 4 <= width(37) <= 16
