"""Python front end of the pskel_* handle API (resident mesh, batched far-block compression).

    eng = Engine()
    eng.upload_mesh(mesh, k=2*pi, eta=376.73, q=7)
    eng.set_blocks(partition)
    stats = eng.compress(tol=1e-4, precision="c64", r0=predicted)   # per-block outcome
    C, U, R, I, J = eng.get_block(b)
    err = eng.true_errors()                                          # vs dense FP64 fill
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

C128, C64 = 0, 1
START_REFERENCE, START_GIVEN = 0, 1


def _prec(p) -> int:
    if p in (C128, "c128", "complex128", "f64"):
        return C128
    if p in (C64, "c64", "complex64", "f32"):
        return C64
    raise ValueError(f"precision {p!r}")


STAT_DTYPE = np.dtype([("m", "i4"), ("n", "i4"), ("r", "i4"), ("rank", "i4"),
                       ("rank_recompressed", "i4"), ("rounds", "i4"), ("status", "i4"),
                       ("est", "f8")], align=True)


def stats_array(stats) -> np.ndarray:
    """ctypes pskel_block_stat_t array -> numpy structured array (C layout, aligned)."""
    assert ctypes.sizeof(_lib.BlockStat) == STAT_DTYPE.itemsize
    return np.frombuffer(bytes(stats), dtype=STAT_DTYPE).copy()


class Engine:
    def __init__(self, device: int = 0):
        self._lib = _lib.lib()
        h = ctypes.c_void_p()
        _lib.check(self._lib.pskel_create(ctypes.byref(h), device))
        self._h = h
        self.mesh = None
        self.partition = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pskel_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------ mesh / blocks
    def upload_mesh(self, mesh, k: float, eta: float, q: int = 7):
        a = mesh.as_f64()
        p = lambda x: x.ctypes.data_as(_lib.D)
        em = _lib.EM(k=float(k), eta=float(eta), q_test=int(q), q_src=int(q))
        _lib.check(self._lib.pskel_upload_mesh(self._h, p(a["vertex"]), mesh.Nv, p(a["topol"]),
                                               mesh.Nt, p(a["edges"]), mesh.N, p(a["ln"]),
                                               p(a["cent"]), ctypes.byref(em)))
        self.mesh = mesh
        self.k, self.eta, self.q = k, eta, q

    def set_blocks(self, part=None, *, group_ptr=None, group_ids=None, gt=None, gs=None):
        if part is not None:
            group_ptr, group_ids, gt, gs = part.group_ptr, part.group_ids, part.gt, part.gs
        gp = np.ascontiguousarray(group_ptr, dtype=np.int32)
        gi = np.ascontiguousarray(group_ids, dtype=np.int32)
        t = np.ascontiguousarray(gt, dtype=np.int32)
        s = np.ascontiguousarray(gs, dtype=np.int32)
        P = lambda x: x.ctypes.data_as(_lib.I32)
        _lib.check(self._lib.pskel_set_blocks(self._h, P(gp), P(gi), len(gp) - 1, P(t), P(s), len(t)))
        self.partition = part
        self._gp, self._gi, self._gt, self._gs = gp, gi, t, s

    def fill_near_device(self, rows_dev: int, nr: int, cols_dev: int, nc: int, out_dev: int,
                         ld: int, rinteg_s: float, ranal_s: float, rinteg_f: float,
                         q_far: int = 1):
        """Near-field fill (complex128) into device buffers given as raw device pointers, with
        the reference element routine's radii (see pskel_fill_near_device)."""
        _lib.check(self._lib.pskel_fill_near_device(
            self._h, ctypes.c_void_p(rows_dev), nr, ctypes.c_void_p(cols_dev), nc,
            ctypes.c_void_p(out_dev), ld, float(rinteg_s), float(ranal_s), float(rinteg_f),
            int(q_far)))

    def octree(self, leaf: float, origin=None, admissibility: float = 2.0, min_group: int = 1,
               symmetric: bool = False):
        """Octree partition of the uploaded mesh built on the device: the same
        ``octree.Partition`` as ``octree.partition(mesh, ...)`` on the host, bit for bit
        (extents to rounding)."""
        from . import octree as _oct
        ng, nb = ctypes.c_int(), ctypes.c_longlong()
        o = None
        if origin is not None:
            o = np.ascontiguousarray(origin, dtype=np.float64)
            if o.shape != (3,):
                raise ValueError("origin: 3 coordinates")
            o = o.ctypes.data_as(_lib.D)
        _lib.check(self._lib.pskel_octree_build(self._h, float(leaf), o, float(admissibility),
                                                int(min_group), int(bool(symmetric)),
                                                ctypes.byref(ng), ctypes.byref(nb)))
        g, b = ng.value, nb.value
        gp = np.empty(g + 1, dtype=np.int32)
        gi = np.empty(self.mesh.N, dtype=np.int32)
        cen = np.empty((g, 3), dtype=np.float64)
        ext = np.empty(g, dtype=np.float64)
        gt = np.empty(b, dtype=np.int32)
        gs = np.empty(b, dtype=np.int32)
        P = lambda x: x.ctypes.data_as(_lib.I32)
        _lib.check(self._lib.pskel_octree_get(self._h, P(gp), P(gi), cen.ctypes.data_as(_lib.D),
                                              ext.ctypes.data_as(_lib.D), P(gt), P(gs)))
        return _oct.Partition(group_ptr=gp, group_ids=gi, centres=cen, extents=ext, gt=gt, gs=gs,
                              leaf=float(leaf))

    @property
    def n_blocks(self) -> int:
        return len(self._gt)

    def block_ids(self, b: int):
        """0-based RWG ids of the rows and columns of block b."""
        gt, gs = self._gt[b], self._gs[b]
        return (self._gi[self._gp[gt]:self._gp[gt + 1]], self._gi[self._gp[gs]:self._gp[gs + 1]])

    # ------------------------------------------------------------------ compression
    def compress(self, tol: float, *, precision="c128", tau: float = 1e-8, tau_relative=True,
                 r0=None, oversample: int = 10, extra_rows: int = 16, extra_cols: int = 16,
                 est_safety: float = 2.0, est_verify: float = 2.0, full_tau: float = 1e-10,
                 max_rounds: int = 12,
                 seed: int = 0,
                 use_graph: bool = False, recompress: bool = False,
                 recompress_tol: float = 0.0, per_block: bool = False,
                 round_growth: float = 2.0) -> np.ndarray:
        """Compress every block; returns a structured array of per-block stats
        (m, n, r, rank, rank_recompressed, rounds, status, est).

        A block passes when its randomized estimate est <= tol / est_safety; a block that
        passes with est above tol / (est_safety * est_verify) is re-checked on a second set of
        extra rows and columns and passes on the pooled estimate (est_verify <= 1: no
        re-check). A block sampled on its whole smaller side (r = min(m, n)) uses the pinv
        threshold min(tau, full_tau) (relative; full_tau = 0: tau). A block that fails is
        compressed again with max(r + 1, ceil(round_growth * r)) samples (2: the reference's
        doubling)."""
        self.set_round_growth(round_growth)
        o = _lib.Opts(tol=tol, tau=tau, tau_relative=int(bool(tau_relative)),
                      precision=_prec(precision),
                      start=START_GIVEN if r0 is not None else START_REFERENCE,
                      oversample=int(oversample), extra_rows=int(extra_rows),
                      extra_cols=int(extra_cols), max_rounds=int(max_rounds),
                      recompress=int(recompress), seed=int(seed),
                      recompress_tol=float(recompress_tol), est_safety=float(est_safety),
                      use_graph=int(bool(use_graph)), per_block=int(bool(per_block)),
                      est_verify=float(est_verify), full_tau=float(full_tau))
        nb = self.n_blocks
        stats = (_lib.BlockStat * nb)()
        if r0 is not None:
            r0a = np.ascontiguousarray(r0, dtype=np.int32)
            if len(r0a) != nb:
                raise ValueError("r0 must have one entry per block")
            rp = r0a.ctypes.data_as(_lib.I32)
        else:
            r0a = None
            rp = None
        _lib.check(self._lib.pskel_compress_blocks(self._h, ctypes.byref(o), rp, stats))
        self._precision = o.precision
        return stats_array(stats)

    def timing(self) -> dict:
        """Device ms per phase of the last compress() and its work counters."""
        t = np.zeros(12)
        _lib.check(self._lib.pskel_last_timing(self._h, t.ctypes.data_as(_lib.D), 12))
        return dict(zip(("sample", "fill", "pinv", "estimate", "recompress", "total",
                         "fill_entries", "point_pairs", "fill_launches", "rounds",
                         "sweeps_mean", "sweeps_max"), t.tolist()))

    def get_block(self, b: int, stats=None):
        rows, cols = self.block_ids(b)
        m, n = len(rows), len(cols)
        if stats is None:
            raise ValueError("pass the stats array returned by compress()")
        r = int(stats["r"][b])
        C = np.zeros((m, r), dtype=np.complex128, order="F")
        U = np.zeros((r, r), dtype=np.complex128, order="F")
        R = np.zeros((r, n), dtype=np.complex128, order="F")
        I = np.zeros(r, dtype=np.int32)
        J = np.zeros(r, dtype=np.int32)
        vp = lambda x: ctypes.c_void_p(x.ctypes.data)
        _lib.check(self._lib.pskel_get_block(self._h, b, vp(C), vp(U), vp(R),
                                             I.ctypes.data_as(_lib.I32), J.ctypes.data_as(_lib.I32)))
        return C, U, R, I, J

    def true_errors(self, blocks=None) -> np.ndarray:
        """Each block's ||Z - C U R||_F / ||Z||_F against its dense FP64 fill (all blocks, or
        the listed ones in that order)."""
        if blocks is None:
            err = np.zeros(self.n_blocks)
            _lib.check(self._lib.pskel_true_errors(self._h, err.ctypes.data_as(_lib.D)))
            return err
        bl = np.ascontiguousarray(blocks, dtype=np.int32)
        err = np.zeros(len(bl))
        _lib.check(self._lib.pskel_true_errors_blocks(self._h, bl.ctypes.data_as(_lib.I32), len(bl),
                                                      err.ctypes.data_as(_lib.D)))
        return err

    def dense_far_matvec(self, X):
        """Dense reference of the far-field product, every block filled in complex FP64:
        X is a complex128 CUDA tensor (RWG count, nrhs); returns Y of the same shape."""
        import torch
        if X.dim() == 1:
            return self.dense_far_matvec(X[:, None])[:, 0]
        if X.dtype != torch.complex128 or not X.is_cuda:
            raise ValueError("X must be a complex128 CUDA tensor")
        ne, nrhs = X.shape
        Xc = X.t().contiguous()
        Y = torch.empty_like(Xc)
        torch.cuda.synchronize(X.device)
        _lib.check(self._lib.pskel_dense_far_matvec(self._h, ctypes.c_void_p(Xc.data_ptr()), ne,
                                                    ctypes.c_void_p(Y.data_ptr()), ne, nrhs))
        return Y.t()

    def matvec(self, X, precision=None):
        """Compressed far-field product Y = sum_b C_b U_b R_b X over all blocks of the last
        compress(). X: torch CUDA tensor (RWG count, nrhs <= 64), complex128 or complex64
        (the arithmetic precision); returns Y of the same shape and dtype on the same stream."""
        import torch
        if X.dim() == 1:
            return self.matvec(X[:, None], precision)[:, 0]
        if X.dtype not in (torch.complex128, torch.complex64) or not X.is_cuda:
            raise ValueError("X must be a complex CUDA tensor")
        prec = C128 if X.dtype == torch.complex128 else C64
        ne, nrhs = X.shape
        Xc = X.t().contiguous()                   # column-major (ne x nrhs), ld = ne
        Y = torch.empty_like(Xc)
        s = torch.cuda.current_stream(X.device).cuda_stream
        _lib.check(self._lib.pskel_matvec(self._h, ctypes.c_void_p(Xc.data_ptr()), ne,
                                          ctypes.c_void_p(Y.data_ptr()), ne, nrhs, prec,
                                          ctypes.c_void_p(s)))
        return Y.t()

    RECOMPRESS_PATHS = {"auto": 0, "fp64": 1, "split": 2}

    def recompress(self, thresh: float, path: str | None = None) -> np.ndarray:
        """SVD-truncate every block's C U R to C' diag(S) R' (S > thresh * S_max); returns the
        kept rank per block. path: None keeps the context's setting, else "auto" (the split
        tensor-core path for complex-FP32 compressions at thresh >= 1e-5, FP64 otherwise),
        "fp64" or "split" (every eligible block, any threshold)."""
        if path is not None:
            _lib.check(self._lib.pskel_set_recompress_path(self._h, self.RECOMPRESS_PATHS[path]))
        k = np.zeros(self.n_blocks, dtype=np.int32)
        _lib.check(self._lib.pskel_recompress(self._h, float(thresh), k.ctypes.data_as(_lib.I32)))
        self._recomp_k = k
        return k

    def recompress_split_blocks(self) -> int:
        """Blocks of the last recompress() that took the split tensor-core path."""
        n = ctypes.c_int(0)
        _lib.check(self._lib.pskel_recompress_split_blocks(self._h, ctypes.byref(n)))
        return int(n.value)

    def recompress_ms(self) -> float:
        """Device time of the last recompress() (ms, between the library's events on its
        stream)."""
        return float(self.timing()["recompress"])

    def get_recompressed(self, b: int):
        """(C', S, R') of block b after recompress()."""
        rows, cols = self.block_ids(b)
        k = int(self._recomp_k[b])
        Cp = np.zeros((len(rows), k), dtype=np.complex128, order="F")
        S = np.zeros(k)
        Rp = np.zeros((k, len(cols)), dtype=np.complex128, order="F")
        vp = lambda x: ctypes.c_void_p(x.ctypes.data)
        _lib.check(self._lib.pskel_get_recompressed(self._h, b, vp(Cp), S.ctypes.data_as(_lib.D),
                                                    vp(Rp)))
        return Cp, S, Rp

    STORE_MODES = {"bf16x3": 0, "tf32": 1, "tf32x3": 2}

    def build_store(self, mode: str = "bf16x3") -> int:
        """Compressed store of the recompressed blocks (after recompress()) in the operand
        format mode: "bf16x3" (bf16 hi + lo, three products), "tf32" (one TF32 plane, one
        product) or "tf32x3" (TF32 hi + lo, three products); returns its bytes."""
        nbytes = ctypes.c_longlong()
        _lib.check(self._lib.pskel_store_build_mode(self._h, self.STORE_MODES[mode],
                                                    ctypes.byref(nbytes)))
        return int(nbytes.value)

    def store_matvec(self, X):
        """Tensor-core matvec over the compressed store: X is a complex64 CUDA tensor
        (RWG count, nrhs <= 16); returns Y of the same shape on the current stream."""
        import torch
        if X.dim() == 1:
            return self.store_matvec(X[:, None])[:, 0]
        if X.dtype != torch.complex64 or not X.is_cuda:
            raise ValueError("X must be a complex64 CUDA tensor")
        ne, nrhs = X.shape
        if X.stride(0) <= 0 or X.stride(1) <= 0:
            X = X.contiguous()
        # X as it is laid out (no transposed copy); Y column-major (the phase-2 atomics of one
        # right-hand side then land on consecutive RWG ids), returned as its transposed view
        Yt = torch.empty((nrhs, ne), dtype=torch.complex64, device=X.device)
        s = torch.cuda.current_stream(X.device).cuda_stream
        _lib.check(self._lib.pskel_store_matvec_strided(
            self._h, ctypes.c_void_p(X.data_ptr()), X.stride(0), X.stride(1),
            ctypes.c_void_p(Yt.data_ptr()), 1, ne, nrhs, ctypes.c_void_p(s)))
        return Yt.t()

    def aca_compress(self, tol: float, kmax: int = 128) -> dict:
        """Adaptive cross approximation of every far block (see pskel_aca_compress); returns
        ranks, statuses and the kernel time in ms."""
        nb = self.n_blocks
        k = np.zeros(nb, dtype=np.int32)
        st = np.zeros(nb, dtype=np.int32)
        _lib.check(self._lib.pskel_aca_compress(self._h, float(tol), int(kmax),
                                                k.ctypes.data_as(_lib.I32), st.ctypes.data_as(_lib.I32)))
        self._aca_k = k
        return dict(k=k, status=st)

    def aca_get_block(self, b: int):
        """(U, V, I, J) of ACA block b: Z(rows, cols) ~ U V, pivots local to the block."""
        rows, cols = self.block_ids(b)
        k = int(self._aca_k[b])
        U = np.zeros((len(rows), k), dtype=np.complex128, order="F")
        V = np.zeros((k, len(cols)), dtype=np.complex128, order="F")
        I = np.zeros(max(k, 1), dtype=np.int32)
        J = np.zeros(max(k, 1), dtype=np.int32)
        vp = lambda x: ctypes.c_void_p(x.ctypes.data)
        _lib.check(self._lib.pskel_aca_get_block(self._h, int(b), vp(U), vp(V), I.ctypes.data_as(_lib.I32),
                                                 J.ctypes.data_as(_lib.I32)))
        return U, V, I[:k], J[:k]

    def aca_true_errors(self) -> np.ndarray:
        err = np.zeros(self.n_blocks)
        _lib.check(self._lib.pskel_aca_true_errors(self._h, err.ctypes.data_as(_lib.D)))
        return err

    def save_store(self, path: str, thresh: float = 0.0):
        """Write the recompressed far field (after recompress()) to a store file."""
        _lib.check(self._lib.pskel_store_save(self._h, str(path).encode(), float(thresh)))

    def load_store(self, path: str) -> int:
        """Load a store file (mesh uploaded first); returns the block count. The groups and
        blocks are taken from the file."""
        nb = ctypes.c_int()
        _lib.check(self._lib.pskel_store_load(self._h, str(path).encode(), ctypes.byref(nb)))
        from . import storefile
        hdr = storefile.read(path, factors=False, check=False)  # the library checked the hash
        self._gp, self._gi, self._gt, self._gs = hdr["group_ptr"], hdr["group_ids"], hdr["gt"], hdr["gs"]
        self._recomp_k = hdr["k"]
        self.partition = None
        return int(nb.value)

    def store_status(self) -> int:
        """Error word of the last store_matvec (0 = every pipeline wait completed)."""
        w = np.zeros(1, dtype=np.int32)
        _lib.check(self._lib.pskel_store_status(self._h, w.ctypes.data_as(_lib.I32)))
        return int(w[0])

    def set_fill_split(self, split_c128: int = -1, split_c64: int = -1):
        """Fill-kernel variant: 8 triangle moments (default), 0 two rows per thread, 1/2/4
        lanes per entry with a shuffle reduction, -1 unchanged."""
        _lib.check(self._lib.pskel_set_fill_split(self._h, int(split_c128), int(split_c64)))

    def set_tri_cols(self, cols: int):
        """Columns per CTA tile of the triangle-moment fill (4, 8 or 16; 0: per job, the width
        up to 16 that fills the CTA best)."""
        _lib.check(self._lib.pskel_set_tri_cols(self._h, int(cols)))

    def set_round_growth(self, factor: float):
        """Sample count factor from one round to the next (default 2, the reference's doubling)."""
        _lib.check(self._lib.pskel_set_round_growth(self._h, float(factor)))

    def set_pipeline(self, chunks: int):
        """Chunks of a pipelined compression round (1 = off; default 2): the fill of one chunk
        overlaps the SVD, pinv and estimate of the previous one."""
        _lib.check(self._lib.pskel_set_pipeline(self._h, int(chunks)))

    def set_symmetric(self, on: bool = True):
        """Compress one block of each (t, s) / (s, t) pair and take the other as its transpose
        (Galerkin symmetry Z = Z^T)."""
        _lib.check(self._lib.pskel_set_symmetric(self._h, int(bool(on))))
        self._symmetric = bool(on)

    def mirror_of(self) -> np.ndarray:
        """Per block: the index of the block with swapped groups (-1 if none)."""
        where = {(int(t), int(s)): b for b, (t, s) in enumerate(zip(self._gt, self._gs))}
        return np.array([where.get((int(s), int(t)), -1) for t, s in zip(self._gt, self._gs)])

    def set_fill_geometry(self, fp32_offsets: bool):
        """Complex-FP32 triangle-moment fill: FP32 pair geometry from per-item offsets (True)
        or FP64 differences and phase (False, default)."""
        _lib.check(self._lib.pskel_set_fill_geometry(self._h, int(bool(fp32_offsets))))

    def fill_device(self, rows_dev: int, nr: int, cols_dev: int, nc: int, out_dev: int, ld: int,
                    precision="c128"):
        """Fill into device buffers given as raw device pointers (e.g. torch data_ptr())."""
        _lib.check(self._lib.pskel_fill_device(self._h, ctypes.c_void_p(rows_dev), nr,
                                               ctypes.c_void_p(cols_dev), nc,
                                               ctypes.c_void_p(out_dev), ld, _prec(precision)))
