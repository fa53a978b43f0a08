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
    # pskel_opts_t: 2 doubles, 8 ints, uint64, 2 doubles, 2 ints
    assert ctypes.sizeof(_lib.Opts) == 80
    assert ctypes.sizeof(_lib.EM) == 24
