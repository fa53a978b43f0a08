"""What the trained predictor gains: on a held-out geometry the learned first sample count
cuts the sampled fill work and the rounds of the plain adaptive method, with every block still
within tolerance against dense FP64 fills."""
import os

import numpy as np
import pytest

from pskel import octree
from pskel.engine import Engine
from pskel.predictor import WEIGHTS, Predictor
from pskel.train_predictor import geometry

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="predictor weights not trained yet")
def test_learned_sampling_gain_on_heldout_geometry():
    m, _ = geometry(103)  # held-out seed (training uses seeds < 100)
    part = octree.partition(m, 0.5, min_group=40)
    k, eta, tol = 2 * np.pi, 376.73, 1e-4
    pred = Predictor.load()
    r0 = pred.sample_counts(part, k, tol)
    opts = dict(precision="c128", tau=1e-7, extra_rows=16, extra_cols=16, est_safety=2.0, seed=0)
    with Engine() as eng:
        eng.upload_mesh(m, k, eta, q=7)
        eng.set_blocks(part)
        st_plain = eng.compress(tol, **opts)
        t_plain = eng.timing()
        err_plain = eng.true_errors()
        st = eng.compress(tol, r0=r0, oversample=0, **opts)
        t_l = eng.timing()
        err = eng.true_errors()
    assert np.all(err <= tol), err.max()
    assert np.all(err_plain <= tol), err_plain.max()
    assert t_l["point_pairs"] < 0.8 * t_plain["point_pairs"], (t_l, t_plain)
    assert st["rounds"].mean() < st_plain["rounds"].mean()
    assert np.mean(st["rounds"] == 1) > 0.7
