"""Algorithmic work of the hot-path kernels: the numerators of every roofline fraction the bench
reports. The counts are conventions fixed once here (they are not instruction counts):

- fill: one Green's-function evaluation between a test and a source quadrature point costs
  FLOPS_PER_PAIR = 32 flops (3 subtractions + 3 FMA for R^2 = 9, sqrt, reciprocal and sin/cos 1
  each, the complex Green's-function scaling 8, the two-term kernel combine 10); a matrix entry
  of the 7-point rule is 4 Q^2 = 196 such pairs;
- pinv of an r x r core: 84 r^3 (complex SVD with both singular-vector sets, 21 n^3 real flops x 4)
  plus 8 r^3 for forming the pseudo-inverse;
- recompression of an m x r, r x r, r x n CUR: 8 (2 m r^2 + 2 n r^2) for the two QRs, 84 r^3 for
  the core SVD, 8 (m + n) r k to rebuild C' and R';
- compressed matvec with s right-hand sides: 8 s (m r + r r + r n) flops; its bytes are the factor
  entries read once plus the vector traffic of the kernel's organisation:
  * CUR form (one pass per block): s (m + n) gathered and scattered vector entries per block;
  * compressed store (grouped GEMMs): X read once (s N entries), the intermediate T = S R' X
    written once and read once (2 s sum_b k_b entries) and Y written once (s N entries).
"""
from __future__ import annotations

import numpy as np

FLOPS_PER_PAIR = 32


def fill_flops(point_pairs: float) -> float:
    return FLOPS_PER_PAIR * float(point_pairs)


def pinv_flops(r) -> float:
    r = np.asarray(r, dtype=np.float64)
    return float((84.0 * r ** 3 + 8.0 * r ** 3).sum())


def recompress_flops(m, n, r, k) -> float:
    m, n, r, k = (np.asarray(x, dtype=np.float64) for x in (m, n, r, k))
    return float((8.0 * (2 * m * r * r + 2 * n * r * r) + 84.0 * r ** 3 + 8.0 * (m + n) * r * k).sum())


def matvec_flops(m, n, r, nrhs: int) -> float:
    m, n, r = (np.asarray(x, dtype=np.float64) for x in (m, n, r))
    return float((8.0 * nrhs * (m * r + r * r + r * n)).sum())


def matvec_bytes(m, n, r, nrhs: int, entry_bytes: float, core_bytes: float = 0.0,
                 vec_entry_bytes: float = 8.0) -> float:
    """Factor entries (m r + r n) of entry_bytes each, r^2 core entries of core_bytes each (0
    for a recompressed store, whose diagonal is folded into R'), and s (m + n) vector entries."""
    m, n, r = (np.asarray(x, dtype=np.float64) for x in (m, n, r))
    return float(((m + n) * r * entry_bytes + r * r * core_bytes + nrhs * (m + n) * vec_entry_bytes).sum())


def store_matvec_bytes(m, n, k, n_rwg: int, nrhs: int, entry_bytes: float = 8.0,
                       vec_entry_bytes: float = 8.0) -> float:
    """Algorithmic bytes of one compressed-store matvec: the factor entries (m + n) k of every
    block (entry_bytes each: bf16 hi + lo of re and im; a mirrored block's transposed factors
    sit in its own groups' tiles), X and Y once each (nrhs N entries) and T = S R' X once
    written and once read (2 nrhs sum k)."""
    m, n, k = (np.asarray(x, dtype=np.float64) for x in (m, n, k))
    factors = float(((m + n) * k * entry_bytes).sum())
    vectors = nrhs * vec_entry_bytes * (2.0 * n_rwg + 2.0 * float(k.sum()))
    return factors + vectors
