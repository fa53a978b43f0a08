"""ctypes front end of the C oracle (``element_oracle.c``, ``near_oracle.c``,
``sampler_oracle.c``).

TEST INFRASTRUCTURE ONLY: the C restatement of the element integral (far and near rules) and
of the seeded sampler. ``build()`` runs ``make -C oracle`` when the library is missing.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def build() -> str:
    path = os.path.join(_HERE, "liboracle.so")
    srcs = [os.path.join(_HERE, f) for f in ("element_oracle.c", "sampler_oracle.c", "near_oracle.c")]
    if not os.path.exists(path) or any(os.path.getmtime(s) > os.path.getmtime(path) for s in srcs):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return path


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(build())
        _LIB.oracle_fill.restype = ctypes.c_int
        _LIB.oracle_fill.argtypes = [_D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_int, _D, _D, ctypes.c_int, ctypes.c_int,
                                     _D, _D, _D, _D, _D, ctypes.c_int]
        _LIB.oracle_element_composite.restype = ctypes.c_int
        _LIB.oracle_element_composite.argtypes = [_D, _D, ctypes.c_double, ctypes.c_double,
                                                  ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  _D, _D, _D, _D, _D]
        _LIB.oracle_fill_near.restype = ctypes.c_int
        _LIB.oracle_fill_near.argtypes = ([_D, _D] + [ctypes.c_double] * 5 + [ctypes.c_int] * 2 +
                                          [_D, _D, ctypes.c_int, ctypes.c_int] + [_D] * 5 +
                                          [ctypes.c_int, ctypes.c_int])
        _LIB.oracle_self_moments_tri.restype = ctypes.c_int
        _LIB.oracle_self_moments_tri.argtypes = [_D, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                 _D, _D]
        _LIB.oracle_philox_word.restype = ctypes.c_uint32
        _LIB.oracle_philox_word.argtypes = [ctypes.c_uint32] * 4 + [ctypes.c_uint64]
        _U32 = ctypes.POINTER(ctypes.c_uint32)
        _LIB.oracle_philox4.restype = None
        _LIB.oracle_philox4.argtypes = [_U32, _U32, _U32]
        _LIB.oracle_sample.restype = ctypes.c_int
        _LIB.oracle_sample.argtypes = [_I, ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64]
        _LIB.oracle_sample_extra.restype = ctypes.c_int
        _LIB.oracle_sample_extra.argtypes = [_I, ctypes.c_int, _I, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                             ctypes.c_uint64]
    return _LIB


def _p(a):
    return a.ctypes.data_as(_D)


def fill(mesh, rows, cols, k: float, eta: float, q_test: int = 1, q_src: int = 1) -> np.ndarray:
    """Z(rows, cols) in complex128 for 1-based RWG ids (oracle restatement)."""
    a = mesh.as_f64()
    r1 = np.ascontiguousarray(rows, dtype=np.float64)
    r2 = np.ascontiguousarray(cols, dtype=np.float64)
    zr = np.zeros((len(r1), len(r2)), order="F")
    zi = np.zeros_like(zr)
    rc = lib().oracle_fill(_p(zr), _p(zi), k, eta, q_test, q_src, _p(r1), _p(r2), len(r1), len(r2),
                           _p(a["vertex"]), _p(a["topol"]), _p(a["edges"]), _p(a["ln"]),
                           _p(a["cent"]), mesh.N)
    if rc != 0:
        raise ValueError("oracle_fill: bad argument")
    return zr + 1j * zi


def fill_near(mesh, rows, cols, k: float, eta: float, rinteg_s: float, ranal_s: float,
              rinteg_f: float, q_far: int = 1, n_self: int = 0) -> np.ndarray:
    """Z(rows, cols) in complex128 for 1-based RWG ids with the near-field rule
    (``near_oracle.c``): 4-point rules inside the integration radii, exact static 1/R inside
    Ranal_s, the converged same-triangle term; q_far = 1 (centroid) or 7 outside the radii."""
    a = mesh.as_f64()
    r1 = np.ascontiguousarray(rows, dtype=np.float64)
    r2 = np.ascontiguousarray(cols, dtype=np.float64)
    zr = np.zeros((len(r1), len(r2)), order="F")
    zi = np.zeros_like(zr)
    rc = lib().oracle_fill_near(_p(zr), _p(zi), k, eta, rinteg_s, ranal_s, rinteg_f, q_far, n_self,
                                _p(r1), _p(r2), len(r1), len(r2), _p(a["vertex"]), _p(a["topol"]),
                                _p(a["edges"]), _p(a["ln"]), _p(a["cent"]), mesh.N, mesh.Nt)
    if rc != 0:
        raise ValueError("oracle_fill_near: bad argument")
    return zr + 1j * zi


def self_moments(mesh, t: int, k: float, n: int = 0) -> np.ndarray:
    """Same-triangle moments of triangle t (0-based): <G>, <x G> (3), <y G> (3), <x.y G>."""
    a = mesh.as_f64()
    out = np.zeros(16)
    lib().oracle_self_moments_tri(_p(out), t, k, n, _p(a["vertex"]), _p(a["topol"]))
    return out[0::2] + 1j * out[1::2]


def element_composite(mesh, m: int, n: int, k: float, eta: float, level: int) -> complex:
    a = mesh.as_f64()
    work = np.zeros(2 * 3 * 4 ** level)
    zr = np.zeros(1)
    zi = np.zeros(1)
    lib().oracle_element_composite(_p(zr), _p(zi), k, eta, m, n, level, _p(a["vertex"]),
                                   _p(a["topol"]), _p(a["edges"]), _p(a["ln"]), _p(work))
    return complex(zr[0], zi[0])


def philox_word(i: int, block: int, rnd: int, stream: int, seed: int) -> int:
    return int(lib().oracle_philox_word(i, block, rnd, stream, seed))


def philox4(ctr, key) -> list:
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib().oracle_philox4(c, k, o)
    return [int(x) for x in o]


def sample(r: int, D: int, block: int, rnd: int, stream: int, seed: int) -> np.ndarray:
    out = np.zeros(max(r, 1), dtype=np.int32)
    if lib().oracle_sample(out.ctypes.data_as(_I), r, D, block, rnd, stream, seed) != 0:
        raise ValueError("oracle_sample: r > D")
    return out[:r].copy()


def sample_extra(p: int, I: np.ndarray, m: int, block: int, rnd: int, seed: int,
                 stream: int = 2) -> np.ndarray:
    I = np.ascontiguousarray(I, dtype=np.int32)
    out = np.zeros(max(p, 1), dtype=np.int32)
    n = lib().oracle_sample_extra(out.ctypes.data_as(_I), p, I.ctypes.data_as(_I), len(I), m,
                                  block, rnd, stream, seed)
    return out[:max(n, 0)].copy()
