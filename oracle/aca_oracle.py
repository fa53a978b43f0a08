"""Adaptive cross approximation restated from the reference (TEST INFRASTRUCTURE ONLY).

``ACA_julia`` (codes/ACA_vs_CUR/seed/ACA_julia.jl:2-112; Zhao, Vouvakis and Lee, IEEE Trans.
EMC 47(4), 2005, as cited at codes/ACA_vs_CUR/seed/ACA.m:13-16): partially pivoted ACA on an
m x n block whose rows and columns are computed on demand. Row pivot 1 is the first row; each
step takes the residual of the current row, its largest unused entry as the column pivot,
scales the row by it (V), takes the residual of that column (U), updates the running estimate of
||U V||_F^2, and stops when ||U_k|| ||V_k|| <= tol ||U V||_F (from the second step on), on a zero
pivot, or after min(m, n) steps; the next row pivot is the largest unused entry of the column
residual. Ties in the pivot searches go to the first index (Julia's findmax).

The library's batched device ACA follows the same steps; this is the checker.
"""
from __future__ import annotations

import numpy as np


def aca(fill_row, fill_col, M: int, N: int, tol: float, kmax: int | None = None):
    """fill_row(i) -> Z[i, :] (N,), fill_col(j) -> Z[:, j] (M,), local 0-based indices.
    Returns dict(U (M x k), V (k x N), I, J, k, status) with status 0 = converged or full rank,
    1 = kmax reached, 2 = zero pivot."""
    kmax = min(M, N) if kmax is None else min(kmax, M, N)
    if M == 1 or N == 1:
        raise ValueError("single-row or single-column blocks are returned uncompressed")
    I, J = [], []
    rows_left = list(range(1, M))  # ACA_julia.jl: i = 2:M (row 1 is the first pivot)
    cols_left = list(range(N))
    # first step
    I.append(0)
    Rik = np.asarray(fill_row(0), dtype=np.complex128)
    col = int(np.argmax(np.abs(Rik[cols_left])))
    J.append(cols_left.pop(col))
    V = (Rik / Rik[J[0]])[None, :]
    Rjk = np.asarray(fill_col(J[0]), dtype=np.complex128)
    U = Rjk[:, None]
    normZ = np.linalg.norm(U) ** 2 * np.linalg.norm(V) ** 2
    status = 0
    if kmax == 1:
        return dict(U=U, V=V, I=np.array(I), J=np.array(J), k=1, status=1)
    row = int(np.argmax(np.abs(Rjk[rows_left])))
    I.append(rows_left.pop(row))
    for k in range(2, min(M, N) + 1):
        Rik = np.asarray(fill_row(I[k - 1]), dtype=np.complex128) - U[I[k - 1], :] @ V
        col = int(np.argmax(np.abs(Rik[cols_left])))
        jk = cols_left.pop(col)
        if Rik[jk] == 0:
            I.pop()
            status = 2
            break
        J.append(jk)
        Vk = Rik / Rik[jk]
        Rjk = np.asarray(fill_col(jk), dtype=np.complex128) - U @ V[:, jk]
        Uk = Rjk
        normZ = normZ + 2 * np.sum(np.real((U.conj().T @ Uk) * (V.conj() @ Vk))) + \
            np.linalg.norm(Uk) ** 2 * np.linalg.norm(Vk) ** 2
        U = np.column_stack([U, Uk])
        V = np.vstack([V, Vk])
        if np.linalg.norm(Uk) * np.linalg.norm(Vk) <= tol * np.sqrt(normZ):
            break
        if k == min(M, N):
            break
        if k == kmax:
            status = 1
            break
        row = int(np.argmax(np.abs(Rjk[rows_left])))
        I.append(rows_left.pop(row))
    return dict(U=U, V=V, I=np.array(I[:U.shape[1]]), J=np.array(J), k=U.shape[1], status=status)
