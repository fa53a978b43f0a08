"""Generate the golden element fixtures from the reference's own shipped CPU element routine.

Runs ONLY where the reference checkout is present (it is not on the GPU box): it loads
``codes/GPU_implementation/seed/functionsExternal.so`` with ctypes and calls its exported
``impedance_matrix`` with the argument list of the reference's Julia wrapper
(``codes/GPU_implementation/seed/compres_single_block_spheres.jl:800-840``; topol's sizes are
passed for trian, as at ``:783-784``). The library is executed as a black box only.

Each fixture stores the mesh arrays it was computed on (so the mesh generator is pinned
too), the EM parameters, the 1-based row/column id lists and the complex128 result.

Usage:  python tests/golden/make_golden.py REFERENCE_ROOT [near]

REFERENCE_ROOT is the root of a checkout of the reference repository (required).
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gpu-randomized-pseudoskeleton_b200"))
from pskel import mesh as pmesh  # noqa: E402

_D = ctypes.POINTER(ctypes.c_double)


def reference_root() -> str:
    if len(sys.argv) < 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: make_golden.py REFERENCE_ROOT [near]  (root of a reference checkout)")
    return sys.argv[1]


def load(ref_root: str):
    so = os.path.join(ref_root, "codes/GPU_implementation/seed/functionsExternal.so")
    lib = ctypes.CDLL(so)
    f = lib.impedance_matrix
    f.restype = ctypes.c_int64
    f.argtypes = ([_D, _D, ctypes.c_int] + [ctypes.c_double] * 5 + [ctypes.c_int] * 2 +
                  [_D] * 10 + [ctypes.c_int] * 18)
    return f


def call(f, m, r1, r2, k, eta, rs, ra, rf):
    a = m.as_f64()
    r1 = np.ascontiguousarray(r1, dtype=np.float64)
    r2 = np.ascontiguousarray(r2, dtype=np.float64)
    zr = np.zeros((len(r1), len(r2)), order="F")
    zi = np.zeros_like(zr)
    p = lambda x: x.ctypes.data_as(_D)
    f(p(zr), p(zi), 1, k, eta, rs, ra, rf, 0, 0, p(r1), p(r2), p(a["vertex"]), p(a["topol"]),
      p(a["trian"]), p(a["edges"]), p(a["un"]), p(a["ds"]), p(a["ln"]), p(a["cent"]),
      m.N, len(r1), len(r2), 3, m.Nv, 3, m.Nt, 3, m.Nt, 4, m.N, 3, m.Nt, 1, m.Nt, m.N, 3, m.Nt)
    return zr + 1j * zi


def save(name, m, r1, r2, k, eta, rint, Z):
    np.savez_compressed(
        os.path.join(HERE, name), vertex=m.vertex, topol=m.topol, trian=m.trian, edges=m.edges,
        un=m.un, ds=m.ds, ln=m.ln, cent=m.cent, rows=np.asarray(r1, dtype=np.int64),
        cols=np.asarray(r2, dtype=np.int64), k=k, eta=eta, rint=rint, Z=Z)
    print(name, Z.shape, float(np.abs(Z).max()))


def main():
    f = load(reference_root())
    eta = 120 * np.pi
    rng = np.random.default_rng(20261203)

    # (1) the reference's own setup (R=1 m spheres 12 m apart, Rint=1, lambda=2): every
    #     element on the centroid path; full 48x48 block of the Ne=48 pair.
    m = pmesh.two_spheres(1.0, 12.0, 48)
    k = 2 * np.pi / 2.0
    r1 = np.arange(1, 49)
    r2 = np.arange(49, 97)
    save("so_two_spheres_ne48.npz", m, r1, r2, k, eta, 1.0, call(f, m, r1, r2, k, eta, 1.0, 1.0, 1.0))

    # (2) Ne=768 per sphere (the reference's case_code 1 uses 12*4^3 = 768), random
    #     unsorted id lists with a repeat, lambda = 4.
    m = pmesh.two_spheres(1.0, 12.0, 768)
    k = 2 * np.pi / 4.0
    r1 = rng.choice(np.arange(1, 769), 40, replace=False)
    r1[5] = r1[0]
    r2 = rng.choice(np.arange(769, 1537), 36, replace=False)
    save("so_two_spheres_ne768_sub.npz", m, r1, r2, k, eta, 1.0, call(f, m, r1, r2, k, eta, 1.0, 1.0, 1.0))

    # (3) the two-plate single-block workload with every radius 0 (centroid rule on every
    #     pair), lambda = 1.
    m = pmesh.two_plates(1.0, 20, 3.0)
    k = 2 * np.pi
    r1 = np.sort(rng.choice(np.arange(1, 1161), 48, replace=False))
    r2 = np.sort(rng.choice(np.arange(1161, 2321), 48, replace=False))
    save("so_two_plates_centroid_sub.npz", m, r1, r2, k, 376.73, 0.0,
         call(f, m, r1, r2, k, 376.73, 0.0, 0.0, 0.0))

    # (4) close spheres (3 m apart), radii 0: centroid rule at short range, lambda = 2.
    m = pmesh.two_spheres(1.0, 3.0, 192)
    k = np.pi
    r1 = np.arange(1, 193, 4)
    r2 = np.arange(193, 385, 4)
    save("so_two_spheres_close_centroid.npz", m, r1, r2, k, eta, 0.0, call(f, m, r1, r2, k, eta, 0.0, 0.0, 0.0))


def save_near(name, m, r1, r2, k, eta, radii, Z):
    np.savez_compressed(
        os.path.join(HERE, name), vertex=m.vertex, topol=m.topol, trian=m.trian, edges=m.edges,
        un=m.un, ds=m.ds, ln=m.ln, cent=m.cent, rows=np.asarray(r1, dtype=np.int64),
        cols=np.asarray(r2, dtype=np.int64), k=k, eta=eta, radii=np.asarray(radii, dtype=np.float64),
        Z=Z)
    print(name, Z.shape, float(np.abs(Z).max()))


def main_near():
    """Near-field fixtures: blocks whose RWG pairs include same-triangle, adjacent and nearby
    triangle pairs, with the integration radii (Rinteg_s, Ranal_s, Rinteg_f) switching the
    library onto its near-field rules."""
    f = load(reference_root())
    eta = 376.73
    # (n1, n2) one plate of the two-plate workload (lambda = 1): RWG 1-48 against 1-64
    m = pmesh.two_plates(1.0, 20, 3.0)
    k = 2 * np.pi
    r1, r2 = np.arange(1, 49), np.arange(1, 65)
    for tag, radii in (("r03", (0.3, 0.3, 0.3)), ("mixed", (0.2, 0.4, 0.1))):
        save_near(f"near_plate_{tag}.npz", m, r1, r2, k, eta, radii, call(f, m, r1, r2, k, eta, *radii))
    # (n3, n4) a coarse sphere (R = 1, 480 RWG, lambda = 2): 40 RWG against their 60 nearest
    m = pmesh.icosphere(1.0, 2)
    k = np.pi
    c = m.basis_centres().T
    r1 = np.arange(1, 41)
    d = np.linalg.norm(c[:, None, :] - c[None, :40, :], axis=2).min(axis=1)
    r2 = np.sort(np.argsort(d, kind="stable")[:60] + 1)
    for tag, radii in (("r05", (0.5, 0.5, 0.5)), ("noanal", (1.0, 0.0, 1.0))):
        save_near(f"near_sphere_{tag}.npz", m, r1, r2, k, eta, radii, call(f, m, r1, r2, k, eta, *radii))


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[2] == "near":
        main_near()
        sys.exit(0)
    main()
