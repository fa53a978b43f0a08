"""The reference's Julia driver functions for the GPU CUR path, restated in Python over the
drop-in C ABI (same function names, argument meaning, outputs and error behaviour).

Reference: codes/GPU_implementation/seed/compres_single_block_spheres_for_sweep2.jl (``sw2``)
and codes/GPU_implementation/seed/compres_single_block_spheres.jl (``big``). Julia's 1-based
integer ranges become numpy integer arrays holding the same 1-based ids. The reference samples
with an unseeded global RNG; here every sampling function takes a numpy ``Generator``.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _lib
from .mesh import RWGMesh


@dataclasses.dataclass
class EMData:
    """``EM_data_struct`` (sw2:29-39)."""
    lambda_: float
    k: float
    eta: float
    field: int = 1
    Rint_s: float = 1.0
    Rint_f: float = 1.0
    Ranal_s: float = 1.0
    corr_solid: int = 0
    flag: int = 0

    @staticmethod
    def for_wavelength(lam: float, eta: float = 120 * np.pi, rint: float = 1.0) -> "EMData":
        return EMData(lam, 2 * np.pi / lam, eta, 1, rint, rint, rint, 0, 0)


def _p(a):
    return a.ctypes.data_as(_lib.D)


def _vp(a):
    return ctypes.c_void_p(a.ctypes.data)


def _marshal(obj: RWGMesh):
    """Float64 column-major copies of the mesh, as the Julia wrappers build before ccall
    (sw2:380-388), plus the size arguments (topol's sizes are passed for trian, sw2:397-398)."""
    a = obj.as_f64()
    sizes = [obj.N, 0, 0, 3, obj.Nv, 3, obj.Nt, 3, obj.Nt, 4, obj.N, 3, obj.Nt, 1, obj.Nt,
             obj.N, 3, obj.Nt]
    return a, sizes


def _ids(r):
    return np.ascontiguousarray(np.asarray(r, dtype=np.int64), dtype=np.float64)


def _em_args(EM: EMData):
    return [int(EM.field), float(EM.k), float(EM.eta), float(EM.Rint_s), float(EM.Ranal_s),
            float(EM.Rint_f), int(EM.corr_solid), int(EM.flag)]


def _mesh_args(a):
    return [_p(a[k]) for k in ("vertex", "topol", "trian", "edges", "un", "ds", "ln", "cent")]


def user_impedance_cuda5(r1, r2, obj: RWGMesh, EM_data: EMData):
    """Dense Z(r1, r2) on the GPU; returns (Ztotal, kernel_ms) (sw2:365-481)."""
    L = _lib.lib()
    a, sizes = _marshal(obj)
    r1 = _ids(r1)
    r2 = _ids(r2)
    sizes[1], sizes[2] = len(r1), len(r2)
    Z = np.zeros((len(r1), len(r2)), dtype=np.complex128, order="F")
    ms = L.impedance_matrix_cuda_elbyel4(_vp(Z), *_em_args(EM_data), _p(r1), _p(r2),
                                         *_mesh_args(a), *sizes, len(r1), len(r2), 1, 1,
                                         len(r1), len(r2))
    if np.isnan(ms):
        code, msg = _lib.last_error()
        raise _lib.PskelError(code, msg)
    return Z, ms


def user_impedance_cuda4(r1, r2, obj: RWGMesh, EM_data: EMData):
    """Dense Z(r1, r2) through impedance_matrix_cuda_elbyel3 (big:1635-1763)."""
    L = _lib.lib()
    a, sizes = _marshal(obj)
    r1 = _ids(r1)
    r2 = _ids(r2)
    sizes[1], sizes[2] = len(r1), len(r2)
    Z = np.zeros((len(r1), len(r2)), dtype=np.complex128, order="F")
    ok = L.impedance_matrix_cuda_elbyel3(_vp(Z), *_em_args(EM_data), _p(r1), _p(r2),
                                         *_mesh_args(a), *sizes, 1, 1, 1, 1, len(r1), len(r2))
    if ok != 1:
        code, msg = _lib.last_error()
        raise _lib.PskelError(code, msg)
    return Z


def user_impedance_cuda3(r1, r2, obj: RWGMesh, EM_data: EMData):
    """Dense Z(r1, r2) through the split re/im impedance_matrix_cuda_elbyel2
    (big:1507-1633)."""
    L = _lib.lib()
    a, sizes = _marshal(obj)
    r1 = _ids(r1)
    r2 = _ids(r2)
    sizes[1], sizes[2] = len(r1), len(r2)
    Zr = np.zeros((len(r1), len(r2)), order="F")
    Zi = np.zeros_like(Zr)
    ok = L.impedance_matrix_cuda_elbyel2(_p(Zr), _p(Zi), *_em_args(EM_data), _p(r1), _p(r2),
                                         *_mesh_args(a), *sizes, 1, 1, 1, 1, len(r1), len(r2))
    if ok != 1:
        code, msg = _lib.last_error()
        raise _lib.PskelError(code, msg)
    return Zr + 1j * Zi


def sample_sorted(rng: np.random.Generator, NN: int, r: int) -> np.ndarray:
    """``sort(sample(1:NN, r, replace=false))`` (sw2:492-494), 1-based."""
    return np.sort(rng.choice(NN, r, replace=False)) + 1


def pure_cuda_compression2(vtest, Avtest_old, current_size, pinv_tol, r1, r2, tol,
                           obj: RWGMesh, EM_data: EMData, rng=None, samples=None):
    """One GPU CUR round (sw2:484-670). Returns (C, U, R, row_samples, col_samples,
    Avtest_new, err_here, time_ms); row/col samples are global 1-based ids.
    ``samples`` = (row_local, col_local) 1-based positions overrides the random draw."""
    L = _lib.lib()
    r1 = np.asarray(r1, dtype=np.int64)
    r2 = np.asarray(r2, dtype=np.int64)
    MM, NN = len(r1), len(r2)
    r = int(current_size)
    if samples is None:
        rng = rng if rng is not None else np.random.default_rng()
        col_local = sample_sorted(rng, NN, r)
        row_local = sample_sorted(rng, MM, r)
    else:
        row_local, col_local = (np.asarray(s, dtype=np.int64) for s in samples)
    col_samples = r2[col_local - 1]
    row_samples = r1[row_local - 1]
    a, sizes = _marshal(obj)
    fr1, fr2 = _ids(r1), _ids(r2)
    sizes[1], sizes[2] = MM, NN
    C = np.zeros((MM, r), dtype=np.complex128, order="F")
    U = np.zeros((r, r), dtype=np.complex128, order="F")
    R = np.zeros((r, NN), dtype=np.complex128, order="F")
    v = np.ascontiguousarray(vtest, dtype=np.complex128)
    yo = np.ascontiguousarray(Avtest_old, dtype=np.complex128)
    yn = np.zeros(MM, dtype=np.complex128)
    t = np.zeros(1)
    cs, rs = _ids(col_samples), _ids(row_samples)
    Zdummy = np.zeros(1, dtype=np.complex128)
    err = L.cuda_complete_compression(
        _vp(C), _vp(U), _vp(R), r, _p(t), float(pinv_tol), _vp(yo), _vp(yn), _vp(v), _p(cs),
        _p(rs), *([1] * 12), _vp(Zdummy), *_em_args(EM_data), _p(fr1), _p(fr2),
        *_mesh_args(a), *sizes, MM, NN, 1, 1, MM, NN)
    if np.isnan(err):
        code, msg = _lib.last_error()
        raise _lib.PskelError(code, msg)
    return C, U, R, row_samples, col_samples, yn, err, float(t[0])


def _next_size(cur, D):
    return 2 * cur if 2 * cur <= D else D


def cuda_cur_compress3(r1, r2, tol, obj: RWGMesh, EM_data: EMData, rng=None):
    """Adaptive GPU CUR (sw2:878-973): start at D/10, double until the successive-estimate
    error is below tol or the size reaches D. Returns (C, U, R, row_samples, col_samples,
    err_app, time_total_ms)."""
    rng = rng if rng is not None else np.random.default_rng()
    pinv_tol = 1e-10
    M, N = len(r1), len(r2)
    vtest = rng.random(N) + 1j * rng.random(N)
    D = min(M, N)
    cur = 1 if D < 10 else D // 10
    err_app = np.inf
    Avtest_old = np.ones(M, dtype=complex)
    out = pure_cuda_compression2(vtest, Avtest_old, cur, pinv_tol, r1, r2, tol, obj, EM_data, rng)
    time_total = out[7]
    Avtest_old = out[5].copy()
    cur = 2 * cur if 2 * cur < D else D
    row_samples = col_samples = None
    C = U = R = None
    while err_app > tol:
        C, U, R, row_samples, col_samples, yn, err_app, tp = pure_cuda_compression2(
            vtest, Avtest_old, cur, pinv_tol, r1, r2, tol, obj, EM_data, rng)
        time_total += tp
        Avtest_old = yn.copy()
        if cur == D:
            break
        cur = _next_size(cur, D)
    return C, U, R, row_samples, col_samples, err_app, time_total


def compute_error_cuda(C, U, R, Avtest_old, vtest):
    """``compute_error_compression`` through the C ABI (sw2:978-998); returns
    (err, Avtest_new)."""
    L = _lib.lib()
    C = np.asfortranarray(C, dtype=np.complex128)
    U = np.asfortranarray(U, dtype=np.complex128)
    R = np.asfortranarray(R, dtype=np.complex128)
    M1, N1 = C.shape
    M2 = R.shape[1]
    yo = np.ascontiguousarray(Avtest_old, dtype=np.complex128).reshape(-1)
    v = np.ascontiguousarray(vtest, dtype=np.complex128).reshape(-1)
    yn = np.zeros(M1, dtype=np.complex128)
    err = L.compute_error_compression(_vp(C), _vp(U), _vp(R), _vp(yo), _vp(yn), _vp(v), M1, N1, M2)
    if np.isnan(err):
        code, msg = _lib.last_error()
        raise _lib.PskelError(code, msg)
    return err, yn


def cuda_cur_pinv2(A, nsamples, tolerance, rng=None, samples=None):
    """CUR of a dense matrix through aux_pinv_compression (sw2:748-792). Returns
    (C, U, R, row_samples, col_samples) with 1-based sample positions."""
    L = _lib.lib()
    A = np.asfortranarray(A, dtype=np.complex128)
    m, n = A.shape
    if samples is None:
        rng = rng if rng is not None else np.random.default_rng()
        cols = sample_sorted(rng, n, nsamples)
        rows = sample_sorted(rng, m, nsamples)
    else:
        rows, cols = (np.asarray(s, dtype=np.int64) for s in samples)
    rs = np.ascontiguousarray(rows, dtype=np.int64)
    cs = np.ascontiguousarray(cols, dtype=np.int64)
    C = np.zeros((m, nsamples), dtype=np.complex128, order="F")
    U = np.zeros((nsamples, nsamples), dtype=np.complex128, order="F")
    R = np.zeros((nsamples, n), dtype=np.complex128, order="F")
    ok = L.aux_pinv_compression(_vp(C), _vp(U), _vp(R), _vp(A), rs.ctypes.data_as(_lib.I64),
                                cs.ctypes.data_as(_lib.I64), nsamples, m, n, float(tolerance))
    if ok != 1:
        code, msg = _lib.last_error()
        raise _lib.PskelError(code, msg)
    return C, U, R, rows, cols


def cuda_pinv(A, treshold):
    """``cuda_pinv`` (cur_external_cuda.cu:217-367): returns (pinvA, U, S, Vt_scaled)."""
    L = _lib.lib()
    A = np.asfortranarray(A, dtype=np.complex128)
    M, N = A.shape
    mn = min(M, N)
    P = np.zeros((N, M), dtype=np.complex128, order="F")
    U = np.zeros((M, mn), dtype=np.complex128, order="F")
    S = np.zeros(mn)
    Vt = np.zeros((N, N), dtype=np.complex128, order="F")
    ok = L.cuda_pinv(_vp(P), _vp(U), _p(S), _vp(Vt), _vp(A), M, N, float(treshold))
    if ok != 1:
        code, msg = _lib.last_error()
        raise _lib.PskelError(code, msg)
    return P, U, S, Vt


def cuda_svd(A):
    """``cuda_svd`` (cur_external_cuda.cu:400-517): thin SVD (U, S, Vt)."""
    L = _lib.lib()
    A = np.asfortranarray(A, dtype=np.complex128)
    M, N = A.shape
    mn = min(M, N)
    U = np.zeros((M, mn), dtype=np.complex128, order="F")
    S = np.zeros(mn)
    Vt = np.zeros((N, N), dtype=np.complex128, order="F")
    ok = L.cuda_svd(_vp(U), _p(S), _vp(Vt), _vp(A), M, N)
    if ok != 1:
        code, msg = _lib.last_error()
        raise _lib.PskelError(code, msg)
    return U, S, Vt


def cuda_filter(V, treshold):
    """``cuda_filter`` (cur_external_cuda.cu:382-398): 0 below the threshold, 1/v above."""
    L = _lib.lib()
    V = np.ascontiguousarray(V, dtype=np.float64).copy()
    ok = L.cuda_filter(_p(V), float(treshold), len(V))
    if ok != 1:
        code, msg = _lib.last_error()
        raise _lib.PskelError(code, msg)
    return V
