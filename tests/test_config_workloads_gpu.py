"""The two-plate workload (two parallel 1 m plates, 3 m apart, lambda = 1 m, 1160 RWG each, the
7-point rule, p = 10 oversampling, pinv threshold 1e-3 relative): one 1160 x 1160 block compressed
by the engine against the oracle's restatement of the same adaptive method on the same seeded
samples, and against a dense FP64 fill."""
import numpy as np
import pytest

from oracle import cur_oracle as co
from oracle import element as el
from pskel import mesh as pmesh
from pskel.engine import Engine

pytestmark = pytest.mark.gpu

K, ETA = 2 * np.pi, 376.73


def test_two_plate_block_matches_oracle():
    m = pmesh.two_plates(1.0, 20, 3.0)
    half = m.N // 2
    assert half == 1160
    gp = np.array([0, half, m.N], dtype=np.int32)
    gi = np.arange(m.N, dtype=np.int32)  # RWG 0..1159 on the first plate
    tol, seed, r0, p = 1e-3, 5, 20, 10
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(group_ptr=gp, group_ids=gi, gt=np.array([0], np.int32), gs=np.array([1], np.int32))
        # the workload's pinv threshold (1e-3 relative) also at full sample count
        st = eng.compress(tol, precision="c128", tau=1e-3, tau_relative=True, r0=[r0],
                          oversample=p, seed=seed, full_tau=0.0)
        C, U, R, I, J = eng.get_block(0, st)
        err = eng.true_errors()[0]
    rows, cols = gi[:half], gi[half:]
    fill = lambda rr, cc: el.fill(m, rr + 1, cc + 1, K, ETA, 7, 7)
    ref = co.plain_adaptive(fill, rows, cols, tol, block_id=0, seed=seed, tau=1e-3,
                            relative=True, r0=r0 + p, full_tau=0.0)
    assert st["r"][0] == ref["r"] and st["rounds"][0] == ref["rounds"]
    assert np.array_equal(I, ref["I"]) and np.array_equal(J, ref["J"])
    assert abs(st["est"][0] - ref["est"]) <= 1e-6 * ref["est"] + 1e-12
    A, Ao = C @ U @ R, ref["C"] @ ref["U"] @ ref["R"]
    assert np.linalg.norm(A - Ao) / np.linalg.norm(Ao) < 1e-8
    Z = fill(rows, cols)
    e_ref = co.rel_fro_error(Z, ref["C"], ref["U"], ref["R"])
    assert abs(err - e_ref) <= 1e-6 * e_ref + 1e-12
    assert err <= tol
