"""H-matrix product and iterative solve of the EFIE system on the device.

The reference assembles whole matrices from precomputed block lists
(compres_single_block_spheres.jl:1404-1505) and solves them densely or by characteristic basis
functions (solve_by_CBF, compres_single_block_spheres.jl:983-1017, called as
``solve_by_CBF(-Ze, Ei)`` at :3939); its excitation is test_fields
(compres_single_block_spheres_for_sweep2.jl:60-85). Here:

* the far blocks of an octree partition are compressed by the engine (CUR, resident on the GPU);
* the near blocks (every other group pair, diagonal included) are filled densely with the
  near-field rule (``pskel_near_build``);
* ``HMatrix.matvec`` is Z X = sum_far C U R X + Z_near X (``pskel_matvec`` + ``pskel_near_matvec``,
  both on the caller's stream);
* ``gmres`` solves (-Z) x = E with restarted GMRES (Arnoldi with classical Gram-Schmidt applied
  twice, Givens rotations); the vectors stay on the device, the small Hessenberg problem on the
  host.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib


def near_pairs(part) -> tuple[np.ndarray, np.ndarray]:
    """Every ordered group pair (t, s) of the partition that is not in its far list (both
    orders of a far pair count as far), diagonal included, in row-major order."""
    G = part.n_groups
    far = np.zeros((G, G), dtype=bool)
    far[part.gt, part.gs] = True
    far[part.gs, part.gt] = True
    t, s = np.nonzero(~far)
    return t.astype(np.int32), s.astype(np.int32)


class HMatrix:
    """Near blocks (dense, complex FP64) + far blocks (compressed) of one engine."""

    def __init__(self, eng, part, radii=(0.0, 0.0, 0.0), q_far: int = 7):
        self.eng = eng
        self.N = eng.mesh.N
        nt, ns = near_pairs(part)
        self.n_near = len(nt)
        nb = ctypes.c_longlong()
        P = lambda x: x.ctypes.data_as(_lib.I32)
        t0 = time.perf_counter()
        _lib.check(eng._lib.pskel_near_build(eng._h, P(nt), P(ns), len(nt), float(radii[0]),
                                             float(radii[1]), float(radii[2]), int(q_far),
                                             ctypes.byref(nb)))
        self.near_build_s = time.perf_counter() - t0
        self.near_bytes = int(nb.value)
        self._nt, self._ns = nt, ns

    def matvec(self, X, far: bool = True, near: bool = True):
        """Z X for a complex128 CUDA tensor X (N or N x nrhs, nrhs <= 16), on the current
        stream."""
        import torch
        vec = X.dim() == 1
        Xm = X[:, None] if vec else X
        if Xm.dtype != torch.complex128 or not Xm.is_cuda or Xm.shape[0] != self.N:
            raise ValueError("X must be a complex128 CUDA tensor with N rows")
        Xc = Xm.t().contiguous()  # column-major N x nrhs
        nrhs = Xm.shape[1]
        Y = torch.empty((nrhs, self.N), dtype=torch.complex128, device=Xm.device)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        vp = lambda t: ctypes.c_void_p(t.data_ptr())
        if far:
            _lib.check(self.eng._lib.pskel_matvec(self.eng._h, vp(Xc), self.N, vp(Y), self.N, nrhs,
                                                  0, st))
        if near:
            _lib.check(self.eng._lib.pskel_near_matvec(self.eng._h, vp(Xc), self.N, vp(Y), self.N,
                                                       nrhs, 1 if far else 0, st))
        Y = Y.t()
        return Y[:, 0] if vec else Y


def plane_wave(eng, theta_deg: float = 0.0, phi_deg: float = 0.0, rot_deg: float = 0.0):
    """Excitation E (complex128 CUDA tensor, N) of test_fields on the engine's mesh."""
    import torch
    E = torch.empty(eng.mesh.N, dtype=torch.complex128, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(eng._lib.pskel_plane_wave(eng._h, float(theta_deg), float(phi_deg), float(rot_deg),
                                         ctypes.c_void_p(E.data_ptr()), st))
    return E


def gmres(A, b, tol: float = 1e-6, restart: int = 60, maxiter: int = 2000, x0=None, M=None):
    """Restarted GMRES for A x = b (A: callable on CUDA complex128 vectors), right-preconditioned
    by M when given (A M y = b, x = M y, so the residual is that of the original system).
    Returns (x, relative residual history, matvec count); stops when the true residual
    ||b - A x|| <= tol ||b|| (checked at every restart) or after maxiter products."""
    import torch
    if M is not None:
        if x0 is None:
            y, hist, nmv = gmres(lambda v: A(M(v)), b, tol, restart, maxiter, None, None)
            return M(y), hist, nmv
        # x0 is a guess of x, not of y: solve A M y = b - A x0 for the correction from y = 0,
        # to the same absolute residual tol ||b||, and return x0 + M y
        bn = float(torch.linalg.vector_norm(b))
        r0 = b - A(x0)
        rn = float(torch.linalg.vector_norm(r0))
        if rn <= tol * bn:
            return x0.clone(), [rn / bn if bn > 0 else 0.0], 1
        y, hist, nmv = gmres(lambda v: A(M(v)), r0, tol * bn / rn, restart, maxiter - 1, None, None)
        return x0 + M(y), [h * rn / bn for h in hist], nmv + 1
    n = b.shape[0]
    bn = float(torch.linalg.vector_norm(b))
    if bn == 0.0:
        return torch.zeros_like(b), [0.0], 0
    nmv = 0
    if x0 is None:
        x = torch.zeros_like(b)
        r = b.clone()
    else:
        x = x0.clone()
        r = b - A(x)
        nmv += 1
    beta = float(torch.linalg.vector_norm(r))
    hist = [beta / bn]
    while beta > tol * bn and nmv < maxiter:
        V = torch.empty((restart + 1, n), dtype=b.dtype, device=b.device)
        V[0] = r / beta
        H = np.zeros((restart + 1, restart), dtype=np.complex128)
        cs = np.zeros(restart, dtype=np.complex128)
        sn = np.zeros(restart, dtype=np.complex128)
        g = np.zeros(restart + 1, dtype=np.complex128)
        g[0] = beta
        j_end = 0
        for j in range(restart):
            w = A(V[j])
            nmv += 1
            # classical Gram-Schmidt applied twice (as accurate as the modified form, two
            # batched products instead of j + 1 dot products and host round trips)
            Vj = V[:j + 1]
            h = Vj.conj() @ w
            w = w - h @ Vj
            h2 = Vj.conj() @ w
            w = w - h2 @ Vj
            H[:j + 1, j] = (h + h2).cpu().numpy()
            hn = float(torch.linalg.vector_norm(w))
            H[j + 1, j] = hn
            if hn != 0.0:
                V[j + 1] = w / hn
            for i in range(j):  # apply the earlier rotations to the new column
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -np.conj(sn[i]) * H[i, j] + np.conj(cs[i]) * H[i + 1, j]
                H[i, j] = t
            # complex Givens rotation G = [[cs, sn], [-conj(sn), conj(cs)]] with
            # G [a; c] = [den; 0]: cs = conj(a) / den, sn = conj(c) / den
            a, c = H[j, j], H[j + 1, j]
            den = np.sqrt(abs(a) ** 2 + abs(c) ** 2)
            cs[j] = np.conj(a) / den if den else 1.0
            sn[j] = np.conj(c) / den if den else 0.0
            H[j, j] = den
            H[j + 1, j] = 0.0
            g[j + 1] = -np.conj(sn[j]) * g[j]
            g[j] = cs[j] * g[j]
            j_end = j + 1
            if abs(g[j + 1]) <= tol * bn or nmv >= maxiter or hn == 0.0:
                break
        y = np.linalg.solve(np.triu(H[:j_end, :j_end]), g[:j_end])
        x = x + torch.as_tensor(y, device=b.device) @ V[:j_end]
        r = b - A(x)
        nmv += 1
        beta = float(torch.linalg.vector_norm(r))
        hist.append(beta / bn)
    return x, hist, nmv
