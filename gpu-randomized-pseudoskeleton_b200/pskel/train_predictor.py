"""Train the sample-count predictor on the GPU (run on a machine with a CUDA device).

Data: seeded random geometries, lambda = 1 - ellipsoids with semi-axes uniform in [1, 3] and
cubes with side uniform in [1, 4], meshed at about lambda/12 (5,000-40,000 RWG) - partitioned
with 0.5-lambda leaf boxes. For every far block the plain method is run with max_rounds = 1 at
each sample count of GRID; the label at tolerance tol is the smallest grid count whose
randomized estimate meets tol / safety (or min(m, n) if none does). Geometry seeds below 100
train the network, seeds from 100 up are held out for evaluation.

    python gpu-randomized-pseudoskeleton_b200/pskel/train_predictor.py [out_dir]

writes predictor_weights.npz and train_report.json to out_dir (default: next to this file).
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    __package__ = "pskel"

from pskel import mesh as pmesh  # noqa: E402
from pskel import octree  # noqa: E402
from pskel.engine import Engine  # noqa: E402
from pskel.predictor import Predictor, features, init_params  # noqa: E402

GRID = (6, 8, 11, 16, 22, 32, 45, 64, 90, 128)
TOLS = (1e-3, 1e-4, 1e-5)
SAFETY = 2.0
EXTRA = 16
K, ETA = 2 * np.pi, 376.73
TAU = {1e-3: 1e-5, 1e-4: 1e-7, 1e-5: 1e-8}


def geometry(seed: int):
    rng = np.random.default_rng(seed)
    if seed % 2 == 0:
        a, b, c = rng.uniform(1, 3, 3)
        return pmesh.ellipsoid(a, b, c, 1 / 12, max_rwg=40000), f"ellipsoid({a:.2f},{b:.2f},{c:.2f})"
    s = rng.uniform(1, 4)
    return pmesh.cube(s, 1 / 12, max_rwg=40000), f"cube({s:.2f})"


def label_blocks(eng: Engine, part, tols=TOLS):
    """Smallest grid sample count passing each tolerance (rows: blocks, cols: tols)."""
    D = np.minimum(part.sizes()[part.gt], part.sizes()[part.gs])
    lab = np.tile(D[:, None], (1, len(tols))).astype(np.float64)
    done = np.zeros((part.n_blocks, len(tols)), dtype=bool)
    for r in GRID:
        st = eng.compress(1.0, precision="c128", tau=1e-8, r0=np.full(part.n_blocks, r),
                          oversample=0, max_rounds=1, extra_rows=EXTRA, extra_cols=EXTRA, seed=r)
        for j, tol in enumerate(tols):
            ok = (st["est"] <= tol / SAFETY) & ~done[:, j]
            lab[ok, j] = np.minimum(r, D[ok])
            done[:, j] |= ok
        if done.all():
            break
    return lab


def dataset(seeds, eng=None):
    X, Y, info = [], [], []
    own = eng is None
    eng = eng or Engine()
    for sd in seeds:
        t0 = time.time()
        m, name = geometry(sd)
        part = octree.partition(m, 0.5, min_group=40)
        eng.upload_mesh(m, K, ETA, q=7)
        eng.set_blocks(part)
        lab = label_blocks(eng, part)
        for j, tol in enumerate(TOLS):
            X.append(features(part, K, tol))
            Y.append(np.log2(lab[:, j]))
        info.append(dict(seed=sd, geometry=name, rwg=m.N, blocks=part.n_blocks,
                         seconds=round(time.time() - t0, 2)))
        print(info[-1], flush=True)
    if own:
        eng.close()
    return np.concatenate(X), np.concatenate(Y), info


def main(out_dir=None):
    out_dir = out_dir or os.path.dirname(os.path.abspath(__file__))
    os.makedirs(out_dir, exist_ok=True)
    eng = Engine()
    Xtr, Ytr, info_tr = dataset(range(0, 12), eng)
    Xte, Yte, info_te = dataset(range(100, 104), eng)
    eng.close()
    pred = Predictor(init_params(0))
    hist = pred.fit(Xtr, Ytr, steps=4000, batch=4096, lr=3e-3)
    yp = pred.predict_log2(Xte)
    resid = yp - Yte
    # margin: the first-round sample count ceil(margin * 2^pred) covers 90% of held-out labels
    q = float(np.quantile(Yte - yp, 0.90))
    pred.margin = float(2 ** max(q, 0.0))
    covered = float(np.mean(np.ceil(pred.margin * np.exp2(yp)) >= np.exp2(Yte) - 1e-9))
    pred.save(os.path.join(out_dir, "predictor_weights.npz"))
    report = dict(train=info_tr, heldout=info_te, samples_train=int(len(Ytr)),
                  samples_heldout=int(len(Yte)), loss_history=hist,
                  heldout_rmse_log2=float(np.sqrt(np.mean(resid ** 2))),
                  margin=pred.margin, heldout_first_round_coverage=covered, grid=GRID,
                  tols=TOLS, safety=SAFETY, extra=EXTRA)
    with open(os.path.join(out_dir, "train_report.json"), "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps({k: v for k, v in report.items() if k not in ("train", "heldout", "loss_history")}))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
