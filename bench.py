"""Benchmark: far-block CUR compression time at relative error 1e-4, learned + mixed precision
+ batched (product) against the plain FP64 GPU pseudoskeleton, on the 30,720-RWG sphere.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sphere30k|sphere7k|sphere122k] [--save out.npz]

A step compresses every far-field block of the workload once: rank predictor inference on the
GPU (own MLP kernel), then one pskel_compress_blocks call (complex FP32 fill with FP64
geometry, FP64 Jacobi pinv, randomized extra-row/extra-column estimate, plain adaptive growth
as fallback; the first round replayed from a CUDA graph). ``value`` is ms per step (lower is
better). Under torchrun the block list is split across ranks (strong scaling, no collective on
the data path); the step time is the maximum over ranks.

``--impl reference`` times the CPU restatement of the reference's algorithm for this path
(oracle/: C element integral + numpy LAPACK pinv, plain adaptive growth) on a bounded sample of
blocks over all host cores and extrapolates to the whole workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gpu-randomized-pseudoskeleton_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from pskel import roofline  # noqa: E402

METRIC = "far-block CUR compress time @ rel err 1e-4: learned+mixed+batched vs plain GPU"
K_WAVE, ETA = 2 * np.pi, 376.73
TOL = 1e-4

WORKLOADS = {
    "sphere30k": dict(R=2.0, sub=5, leaf=0.5, min_group=40,
                      desc="PEC icosphere R=2 lambda, 5 subdivisions (20,480 triangles, 30,720 RWG), "
                           "octree leaf 0.5 lambda, far pairs at >= 2 box diameters"),
    "sphere7k": dict(R=2.0, sub=4, leaf=0.5, min_group=30,
                     desc="PEC icosphere R=2 lambda, 4 subdivisions (7,680 RWG), leaf 0.5 lambda"),
    "sphere122k": dict(R=4.0, sub=6, leaf=0.5, min_group=40,
                       desc="PEC icosphere R=4 lambda, 6 subdivisions (81,920 triangles, 122,880 RWG), "
                            "octree leaf 0.5 lambda"),
}

# DRAM bytes (read + write) of the round-1 fill launch of the product step on sphere30k, from
# one ncu capture (profiles/tri_fill_traffic_sphere30k.md)
FILL_TRAFFIC_BYTES = 2.186e9

# the product's later rounds grow the sample count by sqrt(2) (the grid the rank predictor is
# trained on) instead of doubling: the learned first count misses by little
PRODUCT = dict(precision="c64", tau=1e-7, extra_rows=16, extra_cols=16, est_safety=2.0,
               oversample=0, max_rounds=12, seed=0, round_growth=2 ** 0.5)
PLAIN = dict(precision="c128", tau=1e-7, extra_rows=16, extra_cols=16, est_safety=2.0,
             max_rounds=12, seed=0)


def build_workload(name):
    from pskel import mesh as pmesh
    from pskel import octree
    w = WORKLOADS[name]
    m = pmesh.icosphere(w["R"], w["sub"])
    part = octree.partition(m, w["leaf"], origin=(0, 0, 0), min_group=w["min_group"])
    return m, part


# ----------------------------------------------------------------------------- CPU baseline
def _cpu_worker(args):
    name, blocks = args
    from oracle import cur_oracle as co
    from oracle import element as el
    m, part = build_workload(name)
    fill = lambda a, c: el.fill(m, a, c, K_WAVE, ETA, 7, 7)
    out = []
    for b in blocks:
        rows = part.members(part.gt[b]) + 1
        cols = part.members(part.gs[b]) + 1
        t0 = time.perf_counter()
        r = co.plain_adaptive(fill, rows, cols, TOL, int(b), 0, extra_rows=16, extra_cols=16,
                              safety=2.0, tau=1e-7)
        out.append((int(b), time.perf_counter() - t0, int(r["r"])))
    return out


def cpu_baseline(name, n_sample=96, seed=0):
    """Oracle plain adaptive compression (C element integral, numpy/LAPACK pinv) of a random
    sample of blocks over all host cores; extrapolated to the whole block list."""
    _, part = build_workload(name)
    rng = np.random.default_rng(seed)
    sample = rng.choice(part.n_blocks, min(n_sample, part.n_blocks), replace=False)
    cores = os.cpu_count() or 1
    chunks = [(name, sample[i::cores].tolist()) for i in range(cores) if len(sample[i::cores])]
    ctx = mp.get_context("spawn")
    # one BLAS thread per worker: the spawned workers inherit this environment before they
    # import numpy, so each worker is one single-threaded reference process
    saved = {k: os.environ.get(k) for k in _BLAS_THREADS}
    os.environ.update({k: "1" for k in _BLAS_THREADS})
    try:
        t0 = time.perf_counter()
        with ctx.Pool(len(chunks)) as pool:
            res = [x for part_res in pool.map(_cpu_worker, chunks) for x in part_res]
        wall = time.perf_counter() - t0
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    per_block = np.array([t for _, t, _ in res])
    core_s = per_block.sum()
    est_ms = per_block.mean() * part.n_blocks / cores * 1e3
    return dict(value=float(est_ms), unit="ms", cores=cores, kind="port",
                single_core_ms=float(per_block.mean() * part.n_blocks * 1e3),
                sample=f"{len(sample)} random far blocks of {part.n_blocks} (seed {seed}), each "
                       f"compressed by a single-threaded worker (one BLAS thread); {core_s:.1f} "
                       f"core-s, {wall:.1f} s wall; whole-job time EXTRAPOLATED as mean block "
                       f"time x blocks / cores (single_core_ms: x blocks)",
                cpu=_cpu_model())


_BLAS_THREADS = ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS")


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="pskel_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}",
                                          f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return None
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return dict(sm_mhz=float(np.median(sm)) if sm else None,
                    sm_max_mhz=float(max(mx)) if mx else None, reasons=reasons,
                    samples=len(rows), power_w_max=max(float(r[3]) for r in rows
                                                        if r[3].replace(".", "").isdigit()))


# ----------------------------------------------------------------------------- GPU arm
def shard_blocks(gt, gs, rank: int, world: int) -> np.ndarray:
    """Block indices of one rank: the unordered group pairs {t, s} dealt round-robin, each rank
    taking both (t, s) and (s, t) of its pairs, so the symmetric mode still halves every rank's
    work. No data crosses ranks: every block is independent."""
    gt = np.asarray(gt)
    gs = np.asarray(gs)
    where = {(int(t), int(s)): b for b, (t, s) in enumerate(zip(gt, gs))}
    primaries = [b for b, (t, s) in enumerate(zip(gt, gs))
                 if where.get((int(s), int(t)), -1) < 0 or b < where[(int(s), int(t))]]
    mine = []
    for i, b in enumerate(primaries):
        if i % world != rank:
            continue
        mine.append(b)
        p = where.get((int(gs[b]), int(gt[b])), -1)
        if p >= 0 and p != b:
            mine.append(p)
    return np.array(sorted(mine), dtype=np.int64)


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The largest of the ranks' values (the job's time is its slowest rank's)."""
    if world <= 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, rank, world, dev):
    import torch

    from pskel import _lib
    from pskel.engine import Engine
    from pskel import autotune
    from pskel.predictor import Predictor, features

    torch.cuda.set_device(dev)
    L = _lib.lib()
    m, part = build_workload(args.workload)
    # shard blocks over ranks (interleaved: balanced sizes)
    mine = shard_blocks(part.gt, part.gs, rank, world)
    sub_gt, sub_gs = part.gt[mine], part.gs[mine]
    pred = Predictor.load()
    eng = Engine(dev)
    eng.upload_mesh(m, K_WAVE, ETA, q=7)
    eng.set_blocks(group_ptr=part.group_ptr, group_ids=part.group_ids, gt=sub_gt, gs=sub_gs)
    nb = len(mine)
    # fill variant picked by the autotuner on this GPU and block list (outside the timed region)
    if args.fill_variant:  # given (e.g. for a profile without the autotuner's launches)
        kind = args.fill_variant.rstrip("0123456789")
        tune = {"choice": (kind, int(args.fill_variant[len(kind):])), "ms": "given", "cached": False}
        autotune.apply(eng, PRODUCT["precision"], tune["choice"])
    else:
        tune = autotune.autotune_fill(eng, PRODUCT["precision"], samples=24, repeats=1,
                                      gpu_name=torch.cuda.get_device_name(dev))

    class Sub:  # the rank's block list, for the feature builder
        pass
    sp = Sub()
    sp.gt, sp.gs = sub_gt, sub_gs
    sp.sizes = part.sizes
    sp.extents, sp.centres = part.extents, part.centres
    feats = features(sp, K_WAVE, TOL)
    x_dev = torch.from_numpy(((feats - pred.mean) / pred.std).astype(np.float32)).cuda()
    p_dev = torch.from_numpy(pred.params).cuda()
    y_dev = torch.empty(nb, dtype=torch.float32, device="cuda")
    Dmin = np.minimum(part.sizes()[sub_gt], part.sizes()[sub_gs])
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    vp = lambda t: ctypes.c_void_p(t.data_ptr())

    def predict_r0():
        _lib.check(L.pskel_mlp_forward(vp(p_dev), vp(x_dev), nb, vp(y_dev), None))
        y = y_dev.cpu().numpy().astype(np.float64)
        return np.clip(np.ceil(pred.margin * np.exp2(y)), 1, Dmin).astype(np.int32)

    def step():
        eng.set_symmetric(True)
        r0 = predict_r0()
        return eng.compress(TOL, r0=r0, use_graph=True, **PRODUCT)

    # chunks of the pipelined first round, picked by timing the product step (outside the timed
    # region; 2 unless --pipeline is given)
    if args.pipeline:
        pipe = {"choice": args.pipeline, "ms": "given"}
        eng.set_pipeline(args.pipeline)
    else:
        pipe = autotune.autotune_pipeline(eng, step, repeats=2, flush=flush)

    def without_symmetry(fn):
        def run():
            eng.set_symmetric(False)
            return fn()
        return run

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        times = []
        launches0 = L.pskel_kernel_launches()
        for _ in range(steps):
            flush.zero_()
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            out = fn()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        launches = L.pskel_kernel_launches() - launches0
        return max_over_ranks(float(np.mean(times)), world, "cuda"), out, launches // max(steps, 1), times

    with ClockSampler(dev) as clk:
        ms, st, launches, times = timed(step, args.steps, args.warmup)
    clocks = clk.summary()
    tinfo = eng.timing()
    if args.product_only:
        eng.close()
        return dict(metric=METRIC, value=round(ms, 3), unit="ms", n_gpus=world, steps=args.steps,
                    warmup=args.warmup, ms_per_step=round(ms, 3), higher_is_better=False,
                    mode="product steps only", gpu_launches=int(launches), clocks=clocks,
                    sweeps=dict(mean=tinfo["sweeps_mean"], max=tinfo["sweeps_max"]),
                    config=dict(workload=args.workload, blocks=int(part.n_blocks)))
    # plain FP64 GPU pseudoskeleton (the drop-in baseline): start at min(m,n)/10 and double,
    # driven one block at a time as the reference's drivers call its GPU CUR; same kernels,
    # samples and estimator as the batched modes
    large = args.large or args.workload == "sphere122k"
    plain_pb = without_symmetry(lambda: eng.compress(TOL, per_block=True, **PLAIN))
    plain_ms = None if large else timed(plain_pb, 1, 1)[0]
    # ablations, all blocks batched per round, every block compressed (no symmetry): plain FP64,
    # mixed precision only, learned only, learned + mixed
    plain = without_symmetry(lambda: eng.compress(TOL, **PLAIN))
    if not large:
        plain_b_ms, st_plain, _, _ = timed(plain, max(1, min(2, args.steps)), 1)
        t_plain = eng.timing()
    else:
        plain_b_ms, st_plain, t_plain = None, None, None

    # the same plain method with the symmetric mode: the product against it isolates what the
    # three patterns (learned, mixed precision, batched + graph) gain on their own
    def plain_symmetric():
        eng.set_symmetric(True)
        return eng.compress(TOL, **PLAIN)
    if not large:
        plain_sym_ms, _, _, _ = timed(plain_symmetric, max(1, min(2, args.steps)), 1)
    else:
        # the complex-FP64 plain rounds of every block do not fit the device's memory at once:
        # the blocks (both directions of each pair together) in four batches, one batched call
        # each, the device times summed
        plain_sym_ms, pairs = 0.0, 0.0
        for q in range(4):
            sel = shard_blocks(sub_gt, sub_gs, q, 4)
            eng.set_blocks(group_ptr=part.group_ptr, group_ids=part.group_ids, gt=sub_gt[sel], gs=sub_gs[sel])
            eng.set_symmetric(True)
            eng.compress(TOL, **PLAIN)  # warm-up of this batch's tables
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            eng.compress(TOL, **PLAIN)
            e1.record()
            torch.cuda.synchronize()
            plain_sym_ms += e0.elapsed_time(e1)
            pairs += eng.timing()["point_pairs"]
        t_plain = dict(point_pairs=pairs)
        eng.set_blocks(group_ptr=part.group_ptr, group_ids=part.group_ids, gt=sub_gt, gs=sub_gs)
    mixed_ms = learned_ms = lm_nosym_ms = lsym128_ms = None
    if not large:
        mixed_only = without_symmetry(lambda: eng.compress(TOL, **dict(PLAIN, precision="c64")))
        mixed_ms, _, _, _ = timed(mixed_only, 1, 1)
        learned_only = without_symmetry(lambda: eng.compress(TOL, r0=predict_r0(), use_graph=True,
                                                             **dict(PRODUCT, precision="c128")))
        learned_ms, _, _, _ = timed(learned_only, 1, 2)
        lm_nosym = without_symmetry(lambda: eng.compress(TOL, r0=predict_r0(), use_graph=True, **PRODUCT))
        lm_nosym_ms, _, _, _ = timed(lm_nosym, 1, 2)

        # learned + batched + symmetric in complex FP64: the same-precision counterpart of the
        # ACA comparison (which computes in complex FP64)
        def learned_sym_c128():
            eng.set_symmetric(True)
            return eng.compress(TOL, r0=predict_r0(), use_graph=True, **dict(PRODUCT, precision="c128"))
        lsym128_ms, _, _, _ = timed(learned_sym_c128, 1, 2)
    # per-phase timing of the product without the graph and without the pipelined round (the
    # fill launches alone on the GPU: the roofline of the fill kernel)
    eng.set_symmetric(True)
    r0 = predict_r0()
    eng.set_pipeline(1)
    st_np = eng.compress(TOL, r0=r0, use_graph=False, **PRODUCT)
    tph = eng.timing()
    eng.set_pipeline(pipe["choice"])
    fp32_peak = ctypes.c_double()
    fp64_peak = ctypes.c_double()
    _lib.check(L.pskel_fma_peak(ctypes.byref(fp32_peak), ctypes.byref(fp64_peak)))
    achieved = roofline.fill_flops(tph["point_pairs"]) / (tph["fill"] * 1e-3) / 1e12
    # accuracy of the timed product and of the plain baseline against dense FP64 fills
    st = eng.compress(TOL, r0=r0, use_graph=True, **PRODUCT)
    err = eng.true_errors()
    err_plain = None
    if not (args.no_plain_errors or large):
        eng.set_symmetric(False)
        st_plain = eng.compress(TOL, **PLAIN)
        err_plain = eng.true_errors()
        eng.set_symmetric(True)
        st = eng.compress(TOL, r0=r0, use_graph=True, **PRODUCT)
    blockops = run_blockops(eng, st, m, flush, fp64_recompress=not large)
    footprint = run_footprint(eng, st, part, blockops)
    config3 = None
    if not (args.no_config3 or large):
        def r0_for(tol):
            fe = features(sp, K_WAVE, tol)
            y = pred.predict_log2(fe)
            return np.clip(np.ceil(pred.margin * np.exp2(y)), 1, Dmin).astype(np.int32)
        config3 = run_config3(eng, m, r0_for)
        eng.set_symmetric(True)
        st = eng.compress(TOL, r0=r0, use_graph=True, **PRODUCT)
    octree_t = run_octree(args, m, part, dev) if rank == 0 else None
    aca_t = run_aca(m, part, dev) if (rank == 0 and not args.product_only and not large) else None
    # e2e: the public call path from host buffers: mesh up, octree partition and far list built on
    # the device and copied out, features on the host, block lists + features up, stats down (its
    # own engine; this one's device memory is released first, which the 122,880-RWG workload
    # needs)
    mirror = eng.mirror_of()
    eng.close()
    e2e_ms, h2d, d2h = run_e2e(args, m, part, sub_gt, sub_gs, pred, dev, rank, world, flush,
                                   fill_choice=tune["choice"], pipeline=pipe["choice"])
    if args.save and rank == 0:
        np.savez(args.save, m=st["m"], n=st["n"], r=st["r"], rounds=st["rounds"], est=st["est"],
                 err=err, r_plain=st_plain["r"], rounds_plain=st_plain["rounds"],
                 err_plain=err_plain if err_plain is not None else np.zeros(0))
    out = dict(
        metric=METRIC, value=round(ms, 3), unit="ms", n_gpus=world, steps=args.steps,
        warmup=args.warmup, ms_per_step=round(ms, 3), higher_is_better=False,
        scaling="strong" if world > 1 else "weak", vs_baseline=None,
        dtype="c64 fill (" + ("FP32 pair geometry" if tune["choice"][0] == "tri32_" else "FP64 geometry")
              + ") + FP64 Jacobi pinv",
        data="synthetic: " + WORKLOADS[args.workload]["desc"] + "; no dataset",
        config=dict(workload=args.workload, rwg=m.N, groups=part.n_groups,
                    blocks=int(part.n_blocks), blocks_this_rank=int(nb), tol=TOL,
                    quadrature="7-point per triangle", precision=PRODUCT["precision"],
                    pinv_tau_relative=PRODUCT["tau"], estimator="16 extra rows + 16 extra columns, safety 2",
                    l2="512 MB write before every timed step (inputs also exceed L2)",
                    fill_variant=f"{tune['choice'][0]}{tune['choice'][1]} (autotuned: {tune['ms']} ms)",
                    pipeline_chunks=f"{pipe['choice']} (autotuned step ms: {pipe['ms']})",
                    symmetry="one block of each (t,s)/(s,t) pair compressed, the other taken as its "
                             "transpose (Galerkin Z = Z^T); every block's error measured against its "
                             "own dense FP64 fill"),
        plain_ms=None if plain_ms is None else round(plain_ms, 3),
        speedup_vs_plain=None if plain_ms is None else round(plain_ms / ms, 3),
        plain_desc="plain FP64 GPU pseudoskeleton: start min(m,n)/10, doubling, same estimator, "
                   "driven one block at a time (the reference's per-block driving)",
        ablation_ms={k: (None if v is None else round(v, 3)) for k, v in dict(
            plain_batched=plain_b_ms, plain_batched_symmetric=plain_sym_ms, mixed_batched=mixed_ms,
            learned_batched=learned_ms, learned_mixed_batched=lm_nosym_ms,
            learned_mixed_batched_symmetric=ms, learned_batched_symmetric_c128=lsym128_ms).items()},
        speedup_vs_plain_batched=None if plain_b_ms is None else round(plain_b_ms / ms, 3),
        speedup_three_patterns=round(plain_sym_ms / ms, 3),
        speedup_three_patterns_desc="plain FP64 batched with the symmetric mode / the product: the "
                                    "learned first sample count, complex-FP32 fill and graph "
                                    "replay alone (both arms use the symmetric mode)",
        step_times_ms=[round(t, 3) for t in times],
        phases_ms={k: round(v, 3) for k, v in tinfo.items() if k in ("fill", "total")},
        product=dict(r_mean=float(st["r"].mean()), rounds_mean=float(st["rounds"].mean()),
                     blocks_compressed=int(sum(1 for b, p in enumerate(mirror) if p < 0 or b < p)),
                     blocks_mirrored=int(sum(1 for b, p in enumerate(mirror) if 0 <= p < b)),
                     first_round_accepted=float(np.mean(st["rounds"] == 1)),
                     err_max=float(err.max()), err_median=float(np.median(err)),
                     blocks_over_tol=int((err > TOL).sum()),
                     fill_point_pairs=float(tph["point_pairs"])),
        plain=dict(r_mean=None if st_plain is None else float(st_plain["r"].mean()),
                   rounds_mean=None if st_plain is None else float(st_plain["rounds"].mean()),
                   fill_point_pairs=float(t_plain["point_pairs"]),
                   err_max=None if err_plain is None else float(err_plain.max()),
                   blocks_over_tol=None if err_plain is None else int((err_plain > TOL).sum())),
        roofline=dict(bound="alu",
                      kernel="tri_fill_kernel<float,7> (c64 triangle moments, "
                             + ("FP32 pair geometry" if tune["choice"][0] == "tri32_" else "FP64 geometry")
                             + f", tile width {tune['choice'][1] or 'balanced per job'})",
                      achieved=round(achieved, 3), peak=round(fp32_peak.value, 3), unit="TFLOP/s",
                      frac=round(achieved / fp32_peak.value, 4),
                      traffic=FILL_TRAFFIC_BYTES if args.workload == "sphere30k" else None,
                      traffic_source="dram__bytes_read.sum + dram__bytes_write.sum of the round-1 fill "
                                     "launch, one ncu capture of this workload "
                                     "(profiles/tri_fill_traffic_sphere30k.md)",
                      peak_source="measured FP32 FMA microbenchmark on this GPU (pskel_fma_peak); "
                                  f"FP64 FMA {fp64_peak.value:.2f} TFLOP/s",
                      flops="32 flops per point-pair evaluation x point pairs / fill device time",
                      fill_ms=round(tph["fill"], 3), fill_launches=int(tph["fill_launches"])),
        phases_nograph_ms={k: round(tph[k], 3) for k in ("sample", "fill", "pinv", "estimate", "total")},
        e2e=dict(value=round(e2e_ms, 3), unit="ms", h2d_bytes_per_step=int(h2d),
                 d2h_bytes_per_step=int(d2h),
                 scope="mesh upload, device octree partition and far list (copied out), host "
                       "features, block lists and features up, rank prediction, compression, "
                       "per-block stats down"),
        clocks=clocks, gpu_launches=int(launches),
        blockops=blockops,
        footprint=footprint,
        mixed_precision=config3,
        octree=octree_t,
        aca=aca_t,
    )
    eng.close()
    return out


def run_blockops(eng, st, m, flush, nrhs=16, reps=10, fp64_recompress=True):
    """Compressed far-field matvec (nrhs right-hand sides, complex64 like the stored factors),
    recompression of every block (default path; the FP64 path beside it when fp64_recompress)
    and the tensor-core store matvec, after the product compression."""
    import torch

    from pskel import _lib
    L = _lib.lib()
    g = torch.Generator(device="cuda").manual_seed(0)
    X = torch.randn((m.N, nrhs), dtype=torch.complex64, device="cuda", generator=g)
    for _ in range(3):
        eng.matvec(X)
    times = []
    l0 = L.pskel_kernel_launches()
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.matvec(X)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    mv_launches = (L.pskel_kernel_launches() - l0) // reps
    mv_ms = float(np.mean(times))
    mm, nn, rr = (st[k].astype(np.float64) for k in ("m", "n", "r"))
    mirror = eng.mirror_of()
    own = np.array([p < 0 or b < p for b, p in enumerate(mirror)]) if eng_symmetric(eng) else \
        np.ones(len(mirror), dtype=bool)
    factor_bytes = roofline.matvec_bytes(mm[own], nn[own], rr[own], 0, 8.0, 16.0)
    vec_bytes = 2.0 * nrhs * m.N * 8.0
    flops = roofline.matvec_flops(mm, nn, rr, nrhs)
    peak = _hbm_peak()
    gbs = (factor_bytes + vec_bytes) / (mv_ms * 1e-3) / 1e9
    matvec_out = dict(ms=round(mv_ms, 4), nrhs=nrhs, arithmetic="complex64", launches=int(mv_launches),
                      factor_bytes=factor_bytes, vector_bytes=vec_bytes,
                      achieved_gbs=round(gbs, 1), peak_gbs=peak, frac=round(gbs / peak, 4),
                      gflops=round(flops / (mv_ms * 1e-3) / 1e9, 1),
                      bytes="C and R in complex64 + U in complex128 of the blocks that keep factors "
                            "(a mirrored block reads its partner's), X read and Y written once "
                            "(algorithmic)")
    # recompression to the compression tolerance (device time of its launches, from the
    # library's own events on its stream): the default path (split tensor-core path for these
    # complex-FP32 factors) and, where its workspace fits, the FP64 path on the same blocks
    def time_recompress(path, calls):
        eng.recompress(TOL, path=path)
        ts = []
        for _ in range(calls):
            flush.zero_()
            torch.cuda.synchronize()
            k = eng.recompress(TOL, path=path)
            ts.append(eng.recompress_ms())
        return float(np.mean(ts)), k, eng.recompress_split_blocks()
    rc_fp64_ms = None
    if fp64_recompress:
        rc_fp64_ms, _, _ = time_recompress("fp64", 2)
    rc_ms, ks, split_blocks = time_recompress("auto", 3)
    # compressed store and the tensor-core matvec over it
    t0 = time.perf_counter()
    store_bytes = eng.build_store()
    build_ms = (time.perf_counter() - t0) * 1e3
    for _ in range(3):
        eng.store_matvec(X)
    st_times = []
    l0 = L.pskel_kernel_launches()
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.store_matvec(X)
        e1.record()
        torch.cuda.synchronize()
        st_times.append(e0.elapsed_time(e1))
    st_launches = (L.pskel_kernel_launches() - l0) // reps
    st_ms = float(np.mean(st_times))
    # the same calls back to back between two events (the store, 1.07 GB on the 30,720-RWG
    # sphere, is larger than L2, so no flush is needed between them): the device time per call
    # without the host's call latency in front of each
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        eng.store_matvec(X)
    e1.record()
    torch.cuda.synchronize()
    st_b2b_ms = e0.elapsed_time(e1) / reps
    st_status = eng.store_status()
    kk = ks.astype(np.float64)
    st_alg_bytes = roofline.store_matvec_bytes(mm, nn, kk, m.N, nrhs)
    st_gbs = st_alg_bytes / (st_ms * 1e-3) / 1e9
    st_b2b_gbs = st_alg_bytes / (st_b2b_ms * 1e-3) / 1e9
    return dict(
        matvec=matvec_out,
        store_matvec=dict(ms=round(st_ms, 4), nrhs=nrhs, launches=int(st_launches),
                          status=int(st_status), store_bytes=store_bytes,
                          build_ms=round(build_ms, 3), algorithmic_bytes=st_alg_bytes,
                          achieved_gbs=round(st_gbs, 1), peak_gbs=peak, frac=round(st_gbs / peak, 4),
                          ms_back_to_back=round(st_b2b_ms, 4), achieved_gbs_back_to_back=round(st_b2b_gbs, 1),
                          frac_back_to_back=round(st_b2b_gbs / peak, 4),
                          arithmetic="tcgen05 kind::f16, bf16 hi/lo split (3 products), FP32 accumulation",
                          bytes="C' and diag(S) R' as bf16 hi + lo (8 bytes per complex entry), X and Y "
                                "once each, T (the phase-2 operand) written and read once (algorithmic; "
                                "store_bytes is the tiled store including its padding); ms: one call "
                                "after an L2 flush, host call latency included; ms_back_to_back: "
                                f"{reps} calls between two events"),
        recompress=dict(ms=round(rc_ms, 3), thresh=TOL, r_mean=float(rr.mean()),
                        k_mean=float(ks.mean()), split_blocks=int(split_blocks),
                        primary_blocks=primary_blocks(eng),
                        ms_fp64_path=None if rc_fp64_ms is None else round(rc_fp64_ms, 3),
                        arithmetic="split path: X = C V S^-1, Yh = R^H W S^-1 and the rebuild "
                                   "C' = X Zx, R'^H = Yh Zy as tcgen05 kind::tf32 products of TF32 "
                                   "hi + lo operands (3 products, FP32 accumulation); FP64 Gram, "
                                   "Cholesky, core M = Lx^H S Ly and its Jacobi SVD. FP64 path: "
                                   "Householder QR of C and R^H, Jacobi SVD of the core",
                        timing="device time between the library's events around its launches "
                               "(mean of 3 calls; the FP64 path: mean of 2)"),
    )


STORE_ENTRY_BYTES = {"bf16x3": 8.0, "tf32": 8.0, "tf32x3": 16.0}  # per complex factor entry


def run_footprint(eng, st, part, blockops):
    """Memory of the compressed far field against the dense far-field blocks (complex FP64)."""
    mirror = eng.mirror_of()
    own = np.array([p < 0 or b < p for b, p in enumerate(mirror)]) if eng_symmetric(eng) else \
        np.ones(len(mirror), dtype=bool)
    sz = part.sizes().astype(np.float64)
    dense_far = float((sz[part.gt] * sz[part.gs]).sum()) * 16
    mm, nn, rr = (st[k][own].astype(np.float64) for k in ("m", "n", "r"))
    cur = float(((mm + nn) * rr * 8 + rr * rr * 16).sum())  # C, R complex64; U complex128
    recomp = store = None
    if blockops.get("store_matvec"):
        kk = np.asarray(eng._recomp_k, dtype=np.float64)[own]
        recomp = float(((mm + nn) * kk * 16 + kk * 8).sum())    # C', R' complex128; S
        store = float(blockops["store_matvec"]["store_bytes"])
    frac = lambda x: None if x is None else x / dense_far
    return dict(dense_far_bytes=dense_far, dense_all_bytes=float(eng.mesh.N) ** 2 * 16,
                cur_bytes=cur, cur_frac=cur / dense_far, recompressed_bytes=recomp,
                recompressed_frac=frac(recomp), store_bytes=store, store_frac=frac(store),
                desc="blocks that keep factors (a mirrored block is its partner's transpose): CUR "
                     "factors as compressed (C, R complex64, U complex128), recompressed C' S R' in "
                     "FP64, and the bf16 hi/lo tensor-core store; against the far blocks' dense "
                     "complex-FP64 entries")


def eng_symmetric(eng) -> bool:
    return bool(getattr(eng, "_symmetric", False))


def primary_blocks(eng) -> int:
    """Blocks that keep their own factors: all of them, or in the symmetric mode one block of
    each (t, s) / (s, t) pair (the one with the smaller index) and the blocks without a pair."""
    if not eng_symmetric(eng):
        return int(eng.n_blocks)
    mir = eng.mirror_of()
    return int(np.sum((mir < 0) | (np.arange(len(mir)) < mir)))


def run_config3(eng, m, r0_for, nrhs=16, reps=5):
    """Mixed precision at tolerances 1e-3 and 1e-4: the product compression (complex-FP32 fill,
    FP64 pinv) with every block's error against its dense FP64 fill, then the recompressed
    store in each operand format (one TF32 plane, TF32 hi + lo, bf16 hi + lo) and its 16-RHS
    matvec against the dense FP64 far-field product on complex Gaussian vectors (seed 0)."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(0)
    X = torch.randn((m.N, nrhs), dtype=torch.complex64, device="cuda", generator=g)
    Yd = eng.dense_far_matvec(X.to(torch.complex128))
    nd = float(torch.linalg.vector_norm(Yd))
    out = {}
    for tol in (1e-3, 1e-4):
        eng.set_symmetric(True)
        st = eng.compress(tol, r0=r0_for(tol), **PRODUCT)
        err = eng.true_errors()
        thresh = tol / 10
        ks = eng.recompress(thresh)
        mm, nn, kk = (x.astype(np.float64) for x in (st["m"], st["n"], ks))
        row = dict(blocks=int(len(err)), err_max=float(err.max()), err_median=float(np.median(err)),
                   blocks_over_tol=int((err > tol).sum()), recompress_thresh=thresh,
                   k_mean=float(kk.mean()), formats={})
        for mode in ("tf32", "tf32x3", "bf16x3"):
            nbytes = eng.build_store(mode)
            for _ in range(2):
                Y = eng.store_matvec(X)
            torch.cuda.synchronize()
            ts = []
            for _ in range(reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                Y = eng.store_matvec(X)
                e1.record()
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            ms = float(np.mean(ts))
            rel = float(torch.linalg.vector_norm(Y.to(torch.complex128) - Yd)) / nd
            alg = roofline.store_matvec_bytes(mm, nn, kk, m.N, nrhs, STORE_ENTRY_BYTES[mode])
            row["formats"][mode] = dict(matvec_ms=round(ms, 4), store_bytes=int(nbytes),
                                        status=int(eng.store_status()),
                                        rel_err_vs_dense=rel, achieved_gbs=round(alg / (ms * 1e-3) / 1e9, 1))
        out[f"tol_{tol:g}"] = row
    out["desc"] = ("complex-FP32 fill + FP64 pinv (product options), recompression at tol/10, "
                   "store matvec with 16 complex Gaussian right-hand sides against the dense FP64 "
                   "far-field product")
    return out


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def run_octree(args, m, part, dev, reps=5):
    """The workload's octree partition and far list built on the device (mesh resident) against
    the host restatement: wall times of the whole call (device build + copy-out to host arrays)
    and of the device build alone, and whether the two partitions are identical."""
    import time

    from pskel import octree
    from pskel.engine import Engine
    w = WORKLOADS[args.workload]
    kw = dict(origin=(0, 0, 0), min_group=w["min_group"])
    with Engine(dev) as eng:
        eng.upload_mesh(m, K_WAVE, ETA, q=7)
        d = eng.octree(w["leaf"], **kw)
        same = (np.array_equal(d.group_ptr, part.group_ptr) and np.array_equal(d.group_ids, part.group_ids)
                and np.array_equal(d.centres, part.centres) and np.array_equal(d.gt, part.gt)
                and np.array_equal(d.gs, part.gs))
        tg, tb = [], []
        o = np.zeros(3)
        ng, nbk = ctypes.c_int(), ctypes.c_longlong()
        for _ in range(reps):
            t0 = time.perf_counter()
            eng.octree(w["leaf"], **kw)
            tg.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            rc = eng._lib.pskel_octree_build(eng._h, w["leaf"], o.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                             2.0, w["min_group"], 0, ctypes.byref(ng), ctypes.byref(nbk))
            tb.append(time.perf_counter() - t0)
            assert rc == 0
    th = []
    for _ in range(3):
        t0 = time.perf_counter()
        octree.partition(m, w["leaf"], **kw)
        th.append(time.perf_counter() - t0)
    return dict(groups=int(d.n_groups), blocks=int(d.n_blocks), identical_to_host=bool(same),
                device_ms=round(1e3 * float(np.median(tg)), 3),
                device_build_only_ms=round(1e3 * float(np.median(tb)), 3),
                host_ms=round(1e3 * float(np.median(th)), 3),
                desc="Morton keys, CUB radix sort, key runs, far test on the device; small-group "
                     "merge on the host; host = numpy restatement (pskel/octree.py)")


def run_aca(m, part, dev, reps=3):
    """The comparison compressor: batched device ACA (the reference's ACA_julia steps and
    stopping rule, complex FP64, 7-point entries on demand) on the same blocks and tolerance,
    symmetric mode, with every block's error against its dense FP64 fill."""
    import torch

    from pskel.engine import Engine
    with Engine(dev) as eng:
        eng.upload_mesh(m, K_WAVE, ETA, q=7)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        eng.aca_compress(TOL)
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = eng.aca_compress(TOL)
            ts.append(time.perf_counter() - t0)
        err = eng.aca_true_errors()
    return dict(ms=round(1e3 * float(np.median(ts)), 3), rank_mean=float(out["k"].mean()),
                rank_max=int(out["k"].max()), err_max=float(err.max()),
                err_median=float(np.median(err)), blocks_over_tol=int((err > TOL).sum()),
                desc="partially pivoted ACA (ACA_julia.jl steps and stopping rule), complex FP64, "
                     "one CTA per block, symmetric mode; wall time of the call")


def run_e2e(args, m, part, sub_gt, sub_gs, pred, dev, rank, world, flush, fill_choice=None, pipeline=None):
    """Host data in, compressed blocks resident on the GPU, per-block stats out. Every step
    uploads the mesh, builds the octree partition and far list on the device (copied out to the
    host), takes this rank's blocks, computes the predictor features on the host, uploads the
    block lists and features, predicts the first sample counts and compresses."""
    import torch

    from pskel import _lib, autotune
    from pskel.engine import Engine
    from pskel.predictor import features

    class Sub:
        pass
    sp = Sub()
    a = m.as_f64()
    eng = Engine(dev)
    if fill_choice is not None:  # the fill variant the autotuner picked for this GPU and workload
        autotune.apply(eng, PRODUCT["precision"], fill_choice)
    if pipeline is not None:  # and the chunks of the pipelined round
        eng.set_pipeline(pipeline)
    eng.set_symmetric(True)
    L = _lib.lib()
    w = WORKLOADS[args.workload]
    x_pin = torch.empty((len(sub_gt), 8), dtype=torch.float32).pin_memory()
    p_dev = torch.from_numpy(pred.params).cuda()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    h2d = sum(a[k].nbytes for k in ("vertex", "topol", "edges", "ln", "cent"))
    h2d += part.group_ptr.nbytes + part.group_ids.nbytes + sub_gt.nbytes + sub_gs.nbytes
    h2d += x_pin.numel() * 4 + p_dev.numel() * 4
    d2h = len(sub_gt) * 40 + len(sub_gt) * 4
    d2h += sum(getattr(part, k).nbytes for k in ("group_ptr", "group_ids", "gt", "gs", "centres", "extents"))

    def one():
        eng.upload_mesh(m, K_WAVE, ETA, q=7)
        p = eng.octree(w["leaf"], origin=(0, 0, 0), min_group=w["min_group"])
        mine = shard_blocks(p.gt, p.gs, rank, world) if world > 1 else slice(None)
        sp.gt, sp.gs, sp.sizes, sp.extents, sp.centres = p.gt[mine], p.gs[mine], p.sizes, p.extents, p.centres
        x_pin.copy_(torch.from_numpy(((features(sp, K_WAVE, TOL) - pred.mean) / pred.std).astype(np.float32)))
        eng.set_blocks(group_ptr=p.group_ptr, group_ids=p.group_ids, gt=sp.gt, gs=sp.gs)
        Dmin = np.minimum(p.sizes()[sp.gt], p.sizes()[sp.gs])
        x = x_pin.cuda(non_blocking=True)
        y = torch.empty(len(sub_gt), dtype=torch.float32, device="cuda")
        _lib.check(L.pskel_mlp_forward(vp(p_dev), vp(x), len(sub_gt), vp(y), None))
        r0 = np.clip(np.ceil(pred.margin * np.exp2(y.cpu().numpy().astype(np.float64))), 1, Dmin)
        return eng.compress(TOL, r0=r0.astype(np.int32), use_graph=False, **PRODUCT)

    for _ in range(max(1, args.warmup)):
        one()
    torch.cuda.synchronize()
    ts = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        one()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    t = torch.tensor([float(np.mean(ts))], device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    eng.close()
    return float(t.item()), h2d, d2h


# ----------------------------------------------------------------------------- profiling cases
# Small, repeatable workloads on the 7,680-RWG sphere (icosphere R = 2 lambda, 4 subdivisions,
# 0.5-lambda leaves) that the kernel profiles in profiles/ are captured from:
#   python bench.py --profile-case fill --precision c64 --calls 2 --split 8 --geom32 1
#   python bench.py --profile-case store --calls 5
#   python bench.py --profile-case extras
#   python bench.py --profile-case recompress --calls 2 [--subdiv 5]
#   python bench.py --profile-case matvec --calls 5 [--subdiv 5]
def fill_case(prec, calls, split, geom32, tri_cols=8):
    """CALLS single-round compressions of every far block of the 7,680-RWG sphere at a fixed
    sample count of 24 with the given precision (c128 or c64) and fill variant (8: triangle
    moments, the default; 0: two rows per thread; 1, 2, 4: lanes per entry; geom32 = 1:
    complex-FP32 fill with FP32 pair geometry; tri_cols: columns per triangle-moment tile, 0 =
    balanced per job), printing the fill time and point-pair rate of each call. Under a profiler
    the fill launch of call i is the i-th launch of the fill kernel."""
    from pskel import mesh as pmesh
    from pskel import octree
    from pskel.engine import Engine
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
        eng.set_tri_cols(tri_cols)
        for i in range(calls):
            eng.compress(1.0, precision=prec, r0=np.full(part.n_blocks, 24), oversample=0,
                         max_rounds=1, seed=i)
            t = eng.timing()
            print(f"{prec} split {split} call {i}: fill {t['fill']:.3f} ms, "
                  f"{t['point_pairs'] / t['fill'] / 1e6:.1f} G point pairs/s, pinv "
                  f"{t['pinv']:.3f} ms, Jacobi sweeps mean {t['sweeps_mean']:.2f} "
                  f"max {t['sweeps_max']:.0f}", flush=True)


def store_case(calls, subdiv=4):
    """Compress the sphere (SUBDIV 4: 7,680 RWG, every block compressed; 5: the bench workload,
    30,720 RWG, symmetric mode with the learned first sample counts) at tol 1e-4 (c64),
    recompress to 1e-4, build the compressed store and run CALLS tensor-core matvecs with 16
    right-hand sides. Under a profiler each matvec is build_b1_kernel, store_gemm_kernel (phase
    1), build_b2_kernel, store_gemm_kernel (phase 2) after two memsets."""
    import torch
    from pskel import mesh as pmesh
    from pskel import octree
    from pskel.engine import Engine
    from pskel.predictor import Predictor
    m = pmesh.icosphere(2.0, subdiv)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=30 if subdiv <= 4 else 40)
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        if subdiv <= 4:
            eng.compress(1e-4, precision="c64", tau=1e-7, seed=0)
        else:
            eng.set_symmetric(True)
            r0 = Predictor.load().sample_counts(part, 2 * np.pi, 1e-4)
            eng.compress(1e-4, precision="c64", tau=1e-7, r0=r0, oversample=0, seed=0)
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


def matvec_case(calls, subdiv=4):
    """Compress the sphere (SUBDIV 4: 7,680 RWG, 5: 30,720 RWG, the bench workload) as the
    product does (learned first sample counts, complex64, symmetric mode) and run CALLS CUR-form
    matvecs (pskel_matvec) with 16 complex64 right-hand sides, printing the device time of each.
    Under a profiler each call is one matvec_group_kernel launch after a memset."""
    import torch
    from pskel import mesh as pmesh
    from pskel import octree
    from pskel.engine import Engine
    from pskel.predictor import Predictor
    m = pmesh.icosphere(2.0, subdiv)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=30 if subdiv <= 4 else 40)
    r0 = Predictor.load().sample_counts(part, 2 * np.pi, 1e-4)
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        eng.compress(1e-4, **dict(PRODUCT, r0=r0))
        g = torch.Generator(device="cuda").manual_seed(0)
        X = torch.randn((m.N, 16), dtype=torch.complex64, device="cuda", generator=g)
        for i in range(calls):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            eng.matvec(X)
            e1.record()
            torch.cuda.synchronize()
            print(f"matvec call {i}: {e0.elapsed_time(e1):.4f} ms", flush=True)


def recompress_case(calls, subdiv=4):
    """Compress the sphere (icosphere R = 2 lambda, SUBDIV subdivisions: 4 -> 7,680 RWG with
    0.5-lambda leaves merged to >= 30, 5 -> 30,720 RWG merged to >= 40 with the learned first
    sample counts, the bench workload) at tol 1e-4 (c64, symmetric mode) and recompress it CALLS
    times at thresh 1e-5 on the default (split tensor-core) path, then once on the FP64 path,
    printing the device time of each call. Under a profiler the split path's launches per call
    are rc_check_kernel, the FP64 set beside it, rc_prep_kernel, rc_tc_kernel (X, Yh),
    rc_gram_kernel, the SVD classes, rc_factor_kernel and rc_tc_kernel (C', R')."""
    from pskel import mesh as pmesh
    from pskel import octree
    from pskel.engine import Engine
    from pskel.predictor import Predictor
    m = pmesh.icosphere(2.0, subdiv)
    part = octree.partition(m, 0.5, origin=(0, 0, 0), min_group=30 if subdiv <= 4 else 40)
    r0 = Predictor.load().sample_counts(part, 2 * np.pi, 1e-4) if subdiv >= 5 else None
    with Engine() as eng:
        eng.upload_mesh(m, 2 * np.pi, 376.73, q=7)
        eng.set_blocks(part)
        eng.set_symmetric(True)
        if r0 is None:
            eng.compress(1e-4, precision="c64", tau=1e-7, seed=0)
        else:
            eng.compress(1e-4, precision="c64", tau=1e-7, r0=r0, oversample=0, seed=0)
        for i in range(calls + 1):
            path = "auto" if i < calls else "fp64"
            ks = eng.recompress(1e-5, path=path)
            print(f"recompress call {i} ({path}): {eng.recompress_ms():.3f} ms, split blocks "
                  f"{eng.recompress_split_blocks()} of {primary_blocks(eng)}, k mean "
                  f"{ks.mean():.2f}", flush=True)


def extras_case():
    """Octree, ACA, near-field fill and one H-matrix product on the 7,680-RWG sphere."""
    import time

    import torch

    from pskel.solve import HMatrix
    from pskel import mesh as pmesh
    from pskel import octree
    from pskel.engine import Engine
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
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="sphere30k")
    ap.add_argument("--save", default=None, help="write per-block stats (npz)")
    ap.add_argument("--no-plain-errors", action="store_true",
                    help="skip the dense-fill error check of the plain baseline's blocks")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--large", action="store_true",
                    help="skip the per-block plain run, the ablations beside plain batched, ACA and "
                         "the mixed-precision report (automatic for sphere122k)")
    ap.add_argument("--no-config3", action="store_true",
                    help="skip the mixed-precision report (store formats against the dense product)")
    ap.add_argument("--fill-variant", default=None,
                    help="fill variant instead of the autotuner's choice: tri<w> or tri32_<w> "
                         "(w = 0 balanced, 4, 8, 16) or entry<s>")
    ap.add_argument("--pipeline", type=int, default=0,
                    help="chunks of the pipelined first round (1: off) instead of the autotuner's choice")
    ap.add_argument("--product-only", action="store_true",
                    help="time the product steps only (no baselines, ablations, checks): the "
                         "command the kernel launch list is captured from")
    ap.add_argument("--profile-case", choices=("fill", "store", "extras", "recompress", "matvec"), default=None,
                    help="run one small profiling workload on the 7,680-RWG sphere instead of the "
                         "benchmark (the cases the kernel profiles are captured from)")
    ap.add_argument("--precision", default="c64", help="profiling case fill: c64 or c128")
    ap.add_argument("--calls", type=int, default=3, help="profiling cases: calls of the kernel")
    ap.add_argument("--split", type=int, default=8, help="profiling case fill: fill variant")
    ap.add_argument("--geom32", type=int, default=0, help="profiling case fill: FP32 pair geometry")
    ap.add_argument("--tri-cols", type=int, default=8,
                    help="profiling case fill: columns per triangle-moment tile (0: balanced per job)")
    ap.add_argument("--subdiv", type=int, default=4,
                    help="profiling cases recompress, store and matvec: sphere subdivisions (4: 7,680 RWG, 5: 30,720)")
    args = ap.parse_args()
    if args.profile_case:
        if args.profile_case == "fill":
            fill_case(args.precision, args.calls, args.split, args.geom32, args.tri_cols)
        elif args.profile_case == "store":
            store_case(args.calls, args.subdiv)
        elif args.profile_case == "matvec":
            matvec_case(args.calls, args.subdiv)
        elif args.profile_case == "recompress":
            recompress_case(args.calls, args.subdiv)
        else:
            extras_case()
        return
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        times, last = [], None
        for i in range(max(1, args.warmup) + max(1, args.steps)):
            cb = cpu_baseline(args.workload, n_sample=48, seed=i)
            if i >= max(1, args.warmup):
                times.append(cb["value"])
            last = cb
        v = float(np.median(times))
        line = dict(impl="reference", metric=METRIC, value=round(v, 1), unit="ms", n_gpus=world,
                    steps=args.steps, warmup=args.warmup, ms_per_step=round(v, 1),
                    higher_is_better=False, scaling="weak", vs_baseline=None, dtype="c128",
                    data="synthetic: " + WORKLOADS[args.workload]["desc"],
                    config=dict(workload=args.workload, tol=TOL, quadrature="7-point per triangle"),
                    cpu_baseline=dict(last, value=round(v, 1)),
                    extrapolated=True, sample_blocks_per_step=48,
                    note="each step times 48 random blocks over all host cores and extrapolates to "
                         "the whole block list; value = median over the steps",
                    e2e=dict(value=round(v, 1), unit="ms", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
        print(json.dumps(line), flush=True)
        return

    import torch
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = run_ours(args, rank, world, local)
    if world == 1 and rank == 0 and not (args.no_cpu_baseline or args.product_only):
        out["cpu_baseline"] = cpu_baseline(args.workload)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
