"""numpy restatement of the reference's CUR (pseudoskeleton) path: TEST INFRASTRUCTURE ONLY.

Each function names the reference lines it follows (paths relative to the reference repo;
``sw2`` = codes/GPU_implementation/seed/compres_single_block_spheres_for_sweep2.jl,
``cu1`` = codes/GPU_implementation/seed/user_impedance_for_julia_cuda.cu).

``fill(rows, cols)`` arguments are callables returning the complex128 block Z(rows, cols) for
1-based RWG ids (normally :func:`oracle.element.fill` bound to a mesh). SVDs use LAPACK gesdd
through numpy, as Julia's ``svd`` does (the reference pins no LAPACK version).
"""
from __future__ import annotations

import numpy as np

from . import element as el


def invert_svec(s: np.ndarray, tol: float) -> np.ndarray:
    """1/s where s >= tol, else 0 (sw2:1001-1009; the GPU twin kernel_Sinv, cu1:1435-1445,
    zeroes s < tol)."""
    out = np.zeros_like(s)
    keep = s >= tol
    out[keep] = 1.0 / s[keep]
    return out


def my_pinv(A: np.ndarray, tol: float = 1e-10, relative: bool = False) -> np.ndarray:
    """Truncated pseudo-inverse V diag(1/s) U^H (sw2:1011-1022). ``relative`` keeps
    s >= tol * s_max instead of the reference's absolute s >= tol."""
    U, s, Vh = np.linalg.svd(A, full_matrices=False)
    thr = tol * (s[0] if (relative and s.size) else 1.0)
    return (Vh.conj().T * invert_svec(s, thr)) @ U.conj().T


def pinv_rank(A: np.ndarray, tol: float, relative: bool) -> int:
    s = np.linalg.svd(A, compute_uv=False)
    thr = tol * (s[0] if (relative and s.size) else 1.0)
    return int(np.sum(s >= thr))


def cur_from_indices(fill, rows, cols, I, J, tol=1e-10, relative=False):
    """One CUR round with given local index sets (cu1:1742-1924, sw2:705-745):
    C = Z(rows, cols[J]), U = pinv(Z(rows[I], cols[J])), R = Z(rows[I], cols)."""
    rows = np.asarray(rows)
    cols = np.asarray(cols)
    C = fill(rows, cols[J])
    core = fill(rows[I], cols[J])
    R = fill(rows[I], cols)
    return C, my_pinv(core, tol, relative), R


def compressed_matvec(C, U, R, v):
    """C (U (R v)) (cu1:1929-1960)."""
    return C @ (U @ (R @ v))


def estimate_error(C, U, R, y_old, v):
    """Successive-estimate error ||y_old - y_new|| / ||y_new|| (cu1:1929-1963,
    compute_error_compression cu1:1449-1556)."""
    y_new = compressed_matvec(C, U, R, v)
    return float(np.linalg.norm(y_old - y_new) / np.linalg.norm(y_new)), y_new


def next_size(cur: int, D: int) -> int:
    """Doubling rule with clamp to D (sw2:958-966)."""
    return 2 * cur if 2 * cur <= D else D


def start_size(D: int) -> int:
    """D/10, or 1 below D=10 (sw2:890-895)."""
    return 1 if D < 10 else D // 10


def cur_compress2(fill, rows, cols, tol, rng, pinv_tol=1e-10):
    """CPU adaptive CUR (sw2:794-876), including its quirk: ``Avtest_old`` is the
    first-round estimate and is never refreshed inside the loop (sw2:836-845)."""
    M, N = len(rows), len(cols)
    v = rng.random(N) + 1j * rng.random(N)
    D = min(M, N)
    cur = start_size(D)
    I = np.sort(rng.choice(M, cur, replace=False))
    J = np.sort(rng.choice(N, cur, replace=False))
    C, U, R = cur_from_indices(fill, rows, cols, I, J, pinv_tol)
    y_old = compressed_matvec(C, U, R, v)
    cur = 2 * cur if 2 * cur < D else D
    err = np.inf
    sizes = []
    while err > tol:
        I = np.sort(rng.choice(M, cur, replace=False))
        J = np.sort(rng.choice(N, cur, replace=False))
        C, U, R = cur_from_indices(fill, rows, cols, I, J, pinv_tol)
        sizes.append(cur)
        y_new = compressed_matvec(C, U, R, v)
        err = float(np.linalg.norm(y_old - y_new) / np.linalg.norm(y_new))
        if cur == D:
            break
        cur = next_size(cur, D)
    return C, U, R, err, sizes


def cuda_cur_compress3(fill, rows, cols, tol, rng, pinv_tol=1e-10):
    """GPU adaptive CUR driver semantics (sw2:878-973): first round against
    Avtest_old = ones(M); the first round's error is ignored (assigned to err_here, sw2:905),
    later rounds refresh Avtest_old (sw2:943)."""
    M, N = len(rows), len(cols)
    v = rng.random(N) + 1j * rng.random(N)
    D = min(M, N)
    cur = start_size(D)
    y_old = np.ones(M, dtype=complex)
    I = np.sort(rng.choice(M, cur, replace=False))
    J = np.sort(rng.choice(N, cur, replace=False))
    C, U, R = cur_from_indices(fill, rows, cols, I, J, pinv_tol)
    _, y_old = estimate_error(C, U, R, y_old, v)
    cur = 2 * cur if 2 * cur < D else D
    err = np.inf
    sizes = []
    while err > tol:
        I = np.sort(rng.choice(M, cur, replace=False))
        J = np.sort(rng.choice(N, cur, replace=False))
        C, U, R = cur_from_indices(fill, rows, cols, I, J, pinv_tol)
        sizes.append(cur)
        err, y_old = estimate_error(C, U, R, y_old, v)
        if cur == D:
            break
        cur = next_size(cur, D)
    return C, U, R, err, sizes


def _residual_sums(approx, Z):
    """(||Z - approx||_F^2, ||Z||_F^2)."""
    return float(np.linalg.norm(Z - approx) ** 2), float(np.linalg.norm(Z) ** 2)


def extra_row_sums(C, U, R, Zx, Ix):
    """Residual and norm sums on extra rows Ix (local ids, not in I)."""
    if len(Ix) == 0:
        return 0.0, 0.0
    return _residual_sums((C[Ix, :] @ U) @ R, Zx)


def extra_col_sums(C, U, R, Zc, Jx):
    """Residual and norm sums on extra columns Jx (local ids, not in J)."""
    if len(Jx) == 0:
        return 0.0, 0.0
    return _residual_sums(C @ (U @ R[:, Jx]), Zc)


def est_from_sums(nr, dr, nc, dc):
    """The larger of the relative errors on the extra rows and on the extra columns (0 for a
    side without extra samples)."""
    er = np.sqrt(nr / dr) if dr > 0 else 0.0
    ec = np.sqrt(nc / dc) if dc > 0 else 0.0
    return float(max(er, ec))


def extra_row_estimate(C, U, R, Zx, Ix):
    """Relative error on extra rows Ix (local ids, not in I):
    ||Z(Ix,:) - C(Ix,:) U R||_F / ||Z(Ix,:)||_F; 0 when there are none."""
    return est_from_sums(*extra_row_sums(C, U, R, Zx, Ix), 0.0, 0.0)


def extra_col_estimate(C, U, R, Zc, Jx):
    """Relative error on extra columns Jx (local ids, not in J):
    ||Z(:,Jx) - C U R(:,Jx)||_F / ||Z(:,Jx)||_F; 0 when there are none."""
    return est_from_sums(0.0, 0.0, *extra_col_sums(C, U, R, Zc, Jx))


def plain_adaptive(fill, rows, cols, tol, block_id, seed, extra_rows=16, extra_cols=16,
                   safety=2.0, tau=1e-8, relative=True, r0=None, max_rounds=12, verify=2.0,
                   full_tau=1e-10):
    """Plain adaptive pseudoskeleton with seeded sampling and the randomized estimate: start at
    r0 (default D/10), double until max(extra-row, extra-column relative error) <= tol/safety
    or r = D. Index sets come from the same Philox/Floyd definition as the device sampler
    (streams 0 rows, 1 columns, 2 extra rows, 3 extra columns).

    Two refinements of the library's engine, restated here so that the oracle takes the same
    decisions: a block with r = D uses the relative pinv threshold min(tau, full_tau) (full_tau
    = 0: tau); the core's numbers are also R's at the sampled columns (the library writes C's
    values there; with a common fill they are the same); a block that passes with est above
    tol / (safety * verify) is re-checked on fresh
    extra rows and columns (streams 4 and 5, outside I, Ix and J, Jx) and passes only if the
    estimate pooled over both sets does (verify <= 1: no re-check)."""
    rows = np.asarray(rows)
    cols = np.asarray(cols)
    M, N = len(rows), len(cols)
    D = min(M, N)
    r = start_size(D) if r0 is None else min(max(int(r0), 1), D)
    rnd = 0
    while True:
        I = el.sample(r, M, block_id, rnd, 0, seed)
        J = el.sample(r, N, block_id, rnd, 1, seed)
        Ix = el.sample_extra(extra_rows, I, M, block_id, rnd, seed, stream=2)
        Jx = el.sample_extra(extra_cols, J, N, block_id, rnd, seed, stream=3)
        if r >= D and full_tau > 0:
            t_r, rel_r = (min(tau, full_tau) if relative else full_tau), True
        else:
            t_r, rel_r = tau, relative
        C, U, R = cur_from_indices(fill, rows, cols, I, J, t_r, rel_r)
        Zx = fill(rows[Ix], cols) if len(Ix) else np.zeros((0, N), complex)
        Zc = fill(rows, cols[Jx]) if len(Jx) else np.zeros((M, 0), complex)
        sums = extra_row_sums(C, U, R, Zx, Ix) + extra_col_sums(C, U, R, Zc, Jx)
        est = est_from_sums(*sums)
        last = r >= D or rnd + 1 >= max_rounds
        ok = est <= tol / safety
        more = M - r - len(Ix) > 0 or N - r - len(Jx) > 0
        verified = False
        if ok and verify > 1 and est > tol / (safety * verify) and more and not last:
            Ix2 = el.sample_extra(extra_rows, np.union1d(I, Ix), M, block_id, rnd, seed, stream=4)
            Jx2 = el.sample_extra(extra_cols, np.union1d(J, Jx), N, block_id, rnd, seed, stream=5)
            Zx2 = fill(rows[Ix2], cols) if len(Ix2) else np.zeros((0, N), complex)
            Zc2 = fill(rows, cols[Jx2]) if len(Jx2) else np.zeros((M, 0), complex)
            s2 = extra_row_sums(C, U, R, Zx2, Ix2) + extra_col_sums(C, U, R, Zc2, Jx2)
            est = est_from_sums(*[a + b for a, b in zip(sums, s2)])
            ok = est <= tol / safety
            verified = True
        if ok or last:
            return dict(C=C, U=U, R=R, I=I, J=J, Ix=Ix, Jx=Jx, est=est, r=r, rounds=rnd + 1,
                        verified=verified)
        r = next_size(r, D)
        rnd += 1


def householder_qr(A):
    """Thin QR (LAPACK geqrf/orgqr via numpy); stands in for the unshipped ``qr_cbd``."""
    return np.linalg.qr(A, mode="reduced")


def svd_compress(C, U, R, thresh):
    """Recompression of a CUR product (A/seed/svd_compress.m:19-33 with x.u=C, x.s=U, x.v=R,
    postcompress_wrapper.m:1-5): QR of C and R^H, SVD of Rc U Rr^H, keep s/s_max > thresh.
    Returns (C', S', R') with C' S' R' ~= C U R."""
    qu, ru = householder_qr(C)
    qv, rv = householder_qr(R.conj().T)
    core = ru @ U @ rv.conj().T
    u, s, vh = np.linalg.svd(core, full_matrices=False)
    if s.size == 0 or s[0] == 0:
        return C[:, :0], np.zeros((0, 0)), R[:0, :]
    keep = (s / s[0]) > thresh
    return qu @ u[:, keep], np.diag(s[keep]), (qv @ vh.conj().T[:, keep]).conj().T


def rel_fro_error(Z, C, U, R):
    return float(np.linalg.norm(Z - C @ U @ R) / np.linalg.norm(Z))
