"""Autotuners: the fill launch (times the fill variants on the engine's own block list and
keeps the fastest) and the pipelined first round (times the product step per chunk count).

The variants are the triangle-moment kernel with 4, 8 or 16 columns per CTA tile (usable while
every group has at most 512 RWG; in complex FP32 also with the FP32 pair geometry) and the
per-entry kernels (two rows per thread; 1, 2 or 4 lanes
per entry with a shuffle reduction over the quadrature points). Each candidate runs one
single-round compression of every block at a fixed sample count (the first round's fill, the
launch that dominates a compression) and is timed by the engine's own device events
(`Engine.timing()['fill']`); the best of `repeats` runs counts. The choice is applied to the
engine and returned with the timings, and can be cached in a JSON file keyed by the GPU name and
a signature of the workload.
"""
from __future__ import annotations

import json
import os

import numpy as np

# tile width 0: per job, the width in [4, 16] whose (triangle, column) item count fills the
# CTA's 256 threads best
TRI_VARIANTS = [("tri", 0), ("tri", 4), ("tri", 8), ("tri", 16)]
# complex-FP32 only: the triangle-moment fill with FP32 pair geometry from per-item offsets
TRI32_VARIANTS = [("tri32_", 0), ("tri32_", 4), ("tri32_", 8), ("tri32_", 16)]
ENTRY_VARIANTS = [("entry", 0), ("entry", 1), ("entry", 2), ("entry", 4)]


def apply(eng, precision, variant):
    """Set a fill variant (as returned in an autotune report's 'choice') on an engine."""
    kind, v = variant
    if precision != "c128":
        eng.set_fill_geometry(kind == "tri32_")
    if kind in ("tri", "tri32_"):
        eng.set_tri_cols(v)
        split = 8
    else:
        split = v
    if precision == "c128":
        eng.set_fill_split(split_c128=split)
    else:
        eng.set_fill_split(split_c64=split)


def signature(eng, precision: str, q: int) -> str:
    sizes = np.diff(np.asarray(eng._gp))
    return f"{precision}-q{q}-rwg{eng.mesh.N}-blocks{eng.n_blocks}-gmax{int(sizes.max())}"


def autotune_fill(eng, precision: str = "c64", samples: int = 24, repeats: int = 2,
                  include_entry: bool = False, cache: str | None = None, gpu_name: str = "",
                  q: int = 7) -> dict:
    """Time the fill variants on eng's blocks and apply the fastest; returns
    {"choice": (kind, value), "ms": {variant: fill ms}, "cached": bool}."""
    key = f"{gpu_name}|{signature(eng, precision, q)}"
    if cache and os.path.exists(cache):
        with open(cache) as f:
            table = json.load(f)
        if key in table:
            choice = tuple(table[key]["choice"])
            apply(eng, precision, choice)
            return {"choice": choice, "ms": table[key]["ms"], "cached": True}
    sizes = np.diff(np.asarray(eng._gp))
    variants = list(TRI_VARIANTS) if sizes.max() <= 512 else []
    if variants and precision != "c128":
        variants += TRI32_VARIANTS
    if include_entry or not variants:
        variants += ENTRY_VARIANTS
    r0 = np.minimum(samples, np.minimum(sizes[eng._gt], sizes[eng._gs])).astype(np.int32)
    timings = {}
    for variant in variants:
        apply(eng, precision, variant)
        best = float("inf")
        for rep in range(repeats + 1):  # the first run sets kernel attributes and warms up
            eng.compress(1.0, precision=precision, r0=r0, oversample=0, max_rounds=1, seed=rep)
            if rep > 0:
                best = min(best, eng.timing()["fill"])
        timings[f"{variant[0]}{variant[1]}"] = round(best, 4)
    best_name = min(timings, key=timings.get)
    choice = next(v for v in variants if f"{v[0]}{v[1]}" == best_name)
    apply(eng, precision, choice)
    if cache:
        table = {}
        if os.path.exists(cache):
            with open(cache) as f:
                table = json.load(f)
        table[key] = {"choice": list(choice), "ms": timings}
        with open(cache, "w") as f:
            json.dump(table, f, indent=1)
    return {"choice": choice, "ms": timings, "cached": False}


PIPELINE_CHUNKS = (1, 2, 3, 4)


def autotune_pipeline(eng, step, chunks=PIPELINE_CHUNKS, repeats: int = 3, flush=None) -> dict:
    """Time the product step `step()` (a callable running one compression on eng) with the first
    round split into each chunk count of `chunks` (1: not pipelined; pskel_set_pipeline) and
    apply the fastest; returns {"choice": chunks, "ms": {chunks: best step ms}}. Device time of
    the whole call (CUDA events), after one untimed run per setting; flush, if given, is a
    tensor larger than L2 written before every timed run."""
    import torch
    timings = {}
    for k in chunks:
        eng.set_pipeline(k)
        step()  # warm: tables, graph capture for this setting
        step()
        best = float("inf")
        for _ in range(repeats):
            if flush is not None:
                flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            step()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        timings[k] = round(best, 3)
    choice = min(timings, key=timings.get)
    eng.set_pipeline(choice)
    return {"choice": choice, "ms": timings}
