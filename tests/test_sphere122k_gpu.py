"""The full combined form at scale: the 122,880-RWG sphere (icosphere R = 4 lambda, 6
subdivisions, 81,920 triangles; octree leaf 0.5 lambda, groups merged to >= 40 RWG), every far
block compressed in one call with the learned first sample count, the complex-FP32 fill, the
batched rounds and the symmetric mode at tol 1e-4. A seeded sample of blocks (mirrored ones
included) is checked against dense FP64 fills: every sampled block is within tolerance, and the
compressed far field is a small fraction of the dense far-field blocks."""
import numpy as np
import pytest

from pskel import mesh as pmesh
from pskel import octree
from pskel.engine import Engine
from pskel.predictor import Predictor

pytestmark = pytest.mark.gpu

K, ETA, TOL = 2 * np.pi, 376.73, 1e-4


def test_sphere122k_sampled_blocks_within_tolerance():
    m = pmesh.icosphere(4.0, 6)
    assert m.N == 122880
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=40)
    r0 = Predictor.load().sample_counts(part, K, TOL)
    with Engine() as eng:
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        st = eng.compress(TOL, precision="c64", tau=1e-7, r0=r0, oversample=0, seed=0)
        assert np.all(st["status"] == 0)
        rng = np.random.default_rng(122880)
        sample = np.sort(rng.choice(eng.n_blocks, 256, replace=False))
        err = eng.true_errors(sample)
        mirror = eng.mirror_of()
    assert err.max() <= TOL, (err.max(), sample[int(np.argmax(err))])
    sz = part.sizes().astype(np.float64)
    dense = float((sz[part.gt] * sz[part.gs]).sum()) * 16
    # the blocks that keep factors (a mirrored block is its partner's transpose): C and R in
    # complex64, U in complex128
    own = np.array([p < 0 or b < p for b, p in enumerate(mirror)])
    mm, nn, rr = (st[k][own].astype(np.float64) for k in ("m", "n", "r"))
    stored = float(((mm + nn) * rr * 8 + rr * rr * 16).sum())
    assert stored < 0.25 * dense, (stored, dense)
