"""One small, repeatable compression workload for kernel profiling and variant timing.

    python gpu-randomized-pseudoskeleton_b200/pskel/profile_case.py PRECISION [CALLS] [SPLIT] [GEOM32]
    python gpu-randomized-pseudoskeleton_b200/pskel/profile_case.py store [CALLS]
    python gpu-randomized-pseudoskeleton_b200/pskel/profile_case.py extras

builds the 7,680-RWG sphere (icosphere R = 2 lambda, 4 subdivisions, 0.5-lambda leaves), then
makes CALLS (default 3) single-round compressions of every far block at a fixed sample count of
24 with the given precision (c128 or c64) and fill variant (8: triangle moments, the default;
0: two rows per thread; 1, 2, 4: lanes per entry; GEOM32 = 1: complex-FP32 fill with FP32 pair
geometry), printing the fill time and point-pair
rate of each call. Under a profiler the fill launch of call i is the i-th launch of the chosen fill kernel.
The store form compresses the same sphere, recompresses it, builds the compressed store and runs
CALLS tensor-core matvecs of 16 right-hand sides.
The extras form runs, once each on the same sphere: the device octree partition, the batched ACA
of every far block (tol 1e-4, symmetric mode), a 2,048 x 2,048 near-field fill (radii 0.15
lambda) and one H-matrix product (CUR far blocks at tol 1e-4 + near blocks, one right-hand side).
"""
from __future__ import annotations

import os
import sys

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from pskel import mesh as pmesh  # noqa: E402
from pskel import octree  # noqa: E402
from pskel.engine import Engine  # noqa: E402


def store_case(calls):
    """Compress the same sphere at tol 1e-4 (c64), recompress to 1e-4, build the compressed
    store and run CALLS tensor-core matvecs with 16 right-hand sides."""
    import torch
    m = pmesh.icosphere(2.0, 4)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=30)
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        eng.compress(1e-4, precision="c64", tau=1e-7, seed=0)
        eng.recompress(1e-4)
        nbytes = eng.build_store()
        X = torch.randn((m.N, 16), dtype=torch.complex64, device="cuda")
        for i in range(calls):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            eng.store_matvec(X)
            e1.record()
            torch.cuda.synchronize()
            print(f"store matvec call {i}: {e0.elapsed_time(e1):.4f} ms, store {nbytes / 1e6:.1f} MB, "
                  f"status {eng.store_status()}", flush=True)


def extras_case():
    """Octree, ACA, near-field fill and one H-matrix product on the 7,680-RWG sphere."""
    import time

    import torch

    from pskel.solve import HMatrix
    m = pmesh.icosphere(2.0, 4)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=30)
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        t0 = time.perf_counter()
        p2 = eng.octree(0.5, origin=(0, 0, 0), min_group=30)
        print(f"octree: {1e3 * (time.perf_counter() - t0):.3f} ms, {p2.n_groups} groups, "
              f"{p2.n_blocks} far blocks", flush=True)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        t0 = time.perf_counter()
        out = eng.aca_compress(1e-4)
        print(f"aca: {1e3 * (time.perf_counter() - t0):.3f} ms, rank mean {out['k'].mean():.1f}",
              flush=True)
        c = m.basis_centres().T
        patch = np.argsort(np.linalg.norm(c - c[0], axis=1), kind="stable")[:2048].astype(np.int32)
        ids = torch.as_tensor(patch, device="cuda")
        Z = torch.empty((2048, 2048), dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.fill_near_device(ids.data_ptr(), 2048, ids.data_ptr(), 2048, Z.data_ptr(), 2048,
                             0.15, 0.15, 0.15, q_far=1)
        torch.cuda.synchronize()
        print(f"near fill 2048 x 2048: {1e3 * (time.perf_counter() - t0):.3f} ms", flush=True)
        eng.compress(1e-4, precision="c128", tau=1e-10, seed=0)
        H = HMatrix(eng, part, (0.15, 0.15, 0.15), q_far=7)
        X = torch.randn(m.N, dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        H.matvec(X)
        torch.cuda.synchronize()
        print(f"H-matrix product: {1e3 * (time.perf_counter() - t0):.3f} ms, near blocks "
              f"{H.near_bytes / 1e6:.0f} MB", flush=True)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "extras":
        extras_case()
        return
    if len(sys.argv) > 1 and sys.argv[1] == "store":
        store_case(int(sys.argv[2]) if len(sys.argv) > 2 else 3)
        return
    prec = sys.argv[1] if len(sys.argv) > 1 else "c64"
    calls = int(sys.argv[2]) if len(sys.argv) > 2 else 3
    split = int(sys.argv[3]) if len(sys.argv) > 3 else 8
    geom32 = int(sys.argv[4]) if len(sys.argv) > 4 else 0
    m = pmesh.icosphere(2.0, 4)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=30)
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        if prec == "c128":
            eng.set_fill_split(split_c128=split)
        else:
            eng.set_fill_split(split_c64=split)
            eng.set_fill_geometry(bool(geom32))
        for i in range(calls):
            eng.compress(1.0, precision=prec, r0=np.full(part.n_blocks, 24), oversample=0,
                         max_rounds=1, seed=i)
            t = eng.timing()
            print(f"{prec} split {split} call {i}: fill {t['fill']:.3f} ms, "
                  f"{t['point_pairs'] / t['fill'] / 1e6:.1f} G point pairs/s, pinv "
                  f"{t['pinv']:.3f} ms, Jacobi sweeps mean {t['sweeps_mean']:.2f} "
                  f"max {t['sweeps_max']:.0f}", flush=True)


if __name__ == "__main__":
    main()
