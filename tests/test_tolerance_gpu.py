"""The per-block tolerance contract: every compressed far block's relative Frobenius error
against its dense FP64 fill, ||Z - C U R||_F / ||Z||_F, is at most the requested tolerance -
for the product configuration (learned first sample count, symmetric mode) and for the plain
method (start at min(m, n) / 10, doubling), in complex FP64 and complex FP32, at tolerances
1e-3, 1e-4 and 1e-5, on the 1,920- and 7,680-RWG spheres (groups of 20-50 and 34-76 RWG, where
tight tolerances drive many blocks to full sample count)."""
import numpy as np
import pytest

from pskel import mesh as pmesh
from pskel import octree
from pskel.engine import Engine
from pskel.predictor import Predictor

pytestmark = pytest.mark.gpu

K, ETA = 2 * np.pi, 376.73
SPHERES = {3: 20, 4: 30}  # subdivisions -> smallest group after merging


@pytest.fixture(scope="module", params=sorted(SPHERES))
def sphere(request):
    sub = request.param
    m = pmesh.icosphere(2.0, sub)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=SPHERES[sub])
    eng = Engine()
    eng.upload_mesh(m, K, ETA, q=7)
    eng.set_blocks(part)
    yield sub, part, eng
    eng.close()


@pytest.mark.parametrize("tol", [1e-3, 1e-4, 1e-5])
@pytest.mark.parametrize("prec", ["c128", "c64"])
@pytest.mark.parametrize("mode", ["product", "plain"])
def test_every_block_within_tolerance(sphere, tol, prec, mode):
    sub, part, eng = sphere
    opts = dict(precision=prec, tau=1e-7, extra_rows=16, extra_cols=16, est_safety=2.0, seed=0)
    if mode == "product":
        eng.set_symmetric(True)
        r0 = Predictor.load().sample_counts(part, K, tol)
        st = eng.compress(tol, r0=r0, oversample=0, **opts)
    else:
        eng.set_symmetric(False)
        st = eng.compress(tol, **opts)
    err = eng.true_errors()
    assert np.all(st["status"] == 0)
    assert np.all(np.isfinite(err))
    worst = int(np.argmax(err))
    assert err.max() <= tol, (sub, mode, prec, tol, err.max(), int((err > tol).sum()),
                              st[worst])
