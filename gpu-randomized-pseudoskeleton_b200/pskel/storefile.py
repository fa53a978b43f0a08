"""Reader and writer of the compressed far-field store file (the layout written by
``pskel_store_save``, csrc/storefile.cu), in numpy: for inspection, for tools that consume the
factors without a GPU, and as the format's executable specification.

    char[8] "PSKELST1"; u32 version = 1; u32 flags (bit 0: mirrored blocks);
    i64 N; i32 G; i32 B; f64 thresh;
    i32 group_ptr[G+1]; i32 group_ids[group_ptr[G]]; i32 gt[B]; i32 gs[B];
    i32 (m, n, k, mirror)[B];
    for every block with mirror = -1: complex128 C'[m x k] (column-major), float64 S[k],
                                      complex128 R'[k x n] (column-major);
    u64 FNV-1a hash of all preceding bytes.

A block with mirror >= 0 is the transpose of block ``mirror``: C' = R'_p^T, S = S_p, R' = C'_p^T.
"""
from __future__ import annotations

import numpy as np

MAGIC = b"PSKELST1"
VERSION = 1


def fnv1a(data: bytes) -> int:
    """64-bit FNV-1a (byte-serial; for small files and tests)."""
    h = 1469598103934665603
    for b in data:
        h ^= b
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def write(path, N, group_ptr, group_ids, gt, gs, blocks, thresh=0.0):
    """blocks: list of (m, n, k, mirror, Cp, S, Rp) with Cp/S/Rp None for mirrored blocks."""
    parts = [MAGIC, np.array([VERSION, int(any(b[3] >= 0 for b in blocks))], "<u4").tobytes(),
             np.array([N], "<i8").tobytes(), np.array([len(group_ptr) - 1, len(gt)], "<i4").tobytes(),
             np.array([thresh], "<f8").tobytes()]
    for a in (group_ptr, group_ids, gt, gs):
        parts.append(np.asarray(a, "<i4").tobytes())
    parts.append(np.array([[b[0], b[1], b[2], b[3]] for b in blocks], "<i4").tobytes())
    for m, n, k, mir, Cp, S, Rp in blocks:
        if mir >= 0:
            continue
        parts.append(np.asarray(Cp, dtype="<c16").tobytes(order="F"))
        parts.append(np.asarray(S, "<f8").tobytes())
        parts.append(np.asarray(Rp, dtype="<c16").tobytes(order="F"))
    body = b"".join(parts)
    with open(path, "wb") as f:
        f.write(body)
        f.write(np.array([fnv1a(body)], "<u8").tobytes())


def read(path, factors: bool = True, check: bool = True) -> dict:
    """Parse a store file. factors=False skips the factor arrays; check=False skips the hash
    (byte-serial in Python: slow for large files)."""
    raw = open(path, "rb").read()
    if raw[:8] != MAGIC:
        raise ValueError("not a store file")
    version, flags = np.frombuffer(raw, "<u4", 2, 8)
    if version != VERSION:
        raise ValueError(f"store version {version}")
    N = int(np.frombuffer(raw, "<i8", 1, 16)[0])
    G, B = (int(x) for x in np.frombuffer(raw, "<i4", 2, 24))
    thresh = float(np.frombuffer(raw, "<f8", 1, 32)[0])
    o = 40
    gp = np.frombuffer(raw, "<i4", G + 1, o).astype(np.int32)
    o += 4 * (G + 1)
    gi = np.frombuffer(raw, "<i4", int(gp[-1]), o).astype(np.int32)
    o += 4 * int(gp[-1])
    gt = np.frombuffer(raw, "<i4", B, o).astype(np.int32)
    o += 4 * B
    gs = np.frombuffer(raw, "<i4", B, o).astype(np.int32)
    o += 4 * B
    rec = np.frombuffer(raw, "<i4", 4 * B, o).reshape(B, 4).astype(np.int32)
    o += 16 * B
    out = dict(N=N, flags=int(flags), thresh=thresh, group_ptr=gp, group_ids=gi, gt=gt, gs=gs,
               m=rec[:, 0].copy(), n=rec[:, 1].copy(), k=rec[:, 2].copy(), mirror=rec[:, 3].copy())
    blocks = []
    for m, n, k, mir in rec:
        if mir >= 0:
            blocks.append(None)
            continue
        if o + 16 * m * k + 8 * k + 16 * k * n > len(raw):
            raise ValueError("store file is truncated")
        Cp = np.frombuffer(raw, "<c16", m * k, o).reshape((m, k), order="F")
        o += 16 * m * k
        S = np.frombuffer(raw, "<f8", k, o)
        o += 8 * k
        Rp = np.frombuffer(raw, "<c16", k * n, o).reshape((k, n), order="F")
        o += 16 * k * n
        blocks.append((Cp, S, Rp) if factors else None)
    if o + 8 != len(raw):
        raise ValueError("store file size does not match its records")
    if check and int(np.frombuffer(raw, "<u8", 1, o)[0]) != fnv1a(raw[:o]):
        raise ValueError("store file hash mismatch")
    if factors:
        for b, mir in enumerate(out["mirror"]):
            if mir >= 0:
                Cp, S, Rp = blocks[mir]
                blocks[b] = (Rp.T.copy(), S, Cp.T.copy())
    out["blocks"] = blocks
    return out
