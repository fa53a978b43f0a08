"""Single-level octree grouping of RWG basis functions and the far-field block list.

The reference has no partitioner of its own: its only multi-block code rebuilds a matrix from
block lists produced by MATLAB (compres_single_block_spheres.jl:1109-1347; the .mat data are
not shipped). This module supplies the partition the far-field workloads are defined on:

* every RWG is assigned to the leaf box containing its basis centre (mean of its two triangle
  centroids, ``user_get_OG_basis_center.m:36-39``); boxes are cubes of side ``leaf`` aligned
  at ``origin`` (default: the mesh's bounding-box centre);
* groups = non-empty leaf boxes, listed in Morton order of their integer box coordinates;
  groups smaller than ``min_group`` are folded, smallest first, into the nearest group (by
  size-weighted centre) so that every block has at least that many rows and columns;
* far pairs = ordered group pairs (i, j), i != j, whose box centres are at least
  ``admissibility`` x the box diameter (sqrt(3) * leaf) apart.

Every floating-point step is an elementwise IEEE operation in a fixed order (distances are
sqrt((dx*dx + dy*dy) + dz*dz), no BLAS reductions), so that the device partition
(``Engine.octree``) reproduces the groups, the group centres and the far list bit for bit.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Partition:
    group_ptr: np.ndarray   # (G+1,) int32 CSR offsets
    group_ids: np.ndarray   # (N,) int32 0-based RWG ids grouped
    centres: np.ndarray     # (G, 3) group centre (box centre, size-weighted after merges)
    extents: np.ndarray     # (G,) diameter of the bounding sphere of the group's basis centres
    gt: np.ndarray          # (B,) test group of each far block
    gs: np.ndarray          # (B,) source group of each far block
    leaf: float

    @property
    def n_groups(self) -> int:
        return len(self.group_ptr) - 1

    @property
    def n_blocks(self) -> int:
        return len(self.gt)

    def sizes(self) -> np.ndarray:
        return np.diff(self.group_ptr)

    def members(self, g: int) -> np.ndarray:
        return self.group_ids[self.group_ptr[g]:self.group_ptr[g + 1]]


def _morton3(ix, iy, iz):
    def spread(v):
        v = v.astype(np.uint64) & np.uint64(0x1FFFFF)
        v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
        v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
        v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
        v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
        return v
    return spread(ix) | (spread(iy) << np.uint64(1)) | (spread(iz) << np.uint64(2))


def _dist(a, b):
    """Euclidean distance of (..., 3) points, as sqrt((dx*dx + dy*dy) + dz*dz) with every
    product and sum rounded separately."""
    dx = a[..., 0] - b[..., 0]
    dy = a[..., 1] - b[..., 1]
    dz = a[..., 2] - b[..., 2]
    return np.sqrt((dx * dx + dy * dy) + dz * dz)


def partition(mesh, leaf: float, origin=None, admissibility: float = 2.0,
              min_group: int = 1, symmetric: bool = False) -> Partition:
    c = mesh.basis_centres().T  # (N, 3)
    if origin is None:
        origin = 0.5 * (c.min(axis=0) + c.max(axis=0))
    origin = np.asarray(origin, dtype=np.float64)
    idx = np.floor((c - origin) / leaf).astype(np.int64)
    shift = idx.min(axis=0)
    ui = idx - shift
    keys = _morton3(ui[:, 0], ui[:, 1], ui[:, 2])
    order = np.lexsort((np.arange(len(keys)), keys))
    ks = keys[order]
    starts = np.concatenate([[0], np.nonzero(np.diff(ks))[0] + 1, [len(ks)]])
    groups = [order[starts[i]:starts[i + 1]] for i in range(len(starts) - 1)]
    box_centre = [origin + (idx[g[0]] + 0.5) * leaf for g in groups]
    # merge small groups: repeatedly fold the smallest group into the nearest other group
    # (size-weighted centre), until every group has at least min_group members
    if min_group > 1 and len(groups) > 1:
        members = [list(g) for g in groups]
        cen = [np.asarray(bc, dtype=np.float64) for bc in box_centre]
        alive = list(range(len(groups)))
        while len(alive) > 1:
            sizes = [len(members[i]) for i in alive]
            k = int(np.argmin(sizes))
            if sizes[k] >= min_group:
                break
            i = alive[k]
            others = [j for j in alive if j != i]
            d = _dist(np.array([cen[j] for j in others]), cen[i])
            j = others[int(np.argmin(d))]
            ni, nj = len(members[i]), len(members[j])
            cen[j] = (cen[j] * nj + cen[i] * ni) / (ni + nj)
            members[j].extend(members[i])
            alive.remove(i)
        groups = [np.sort(np.array(members[i], dtype=np.int64)) for i in alive]
        box_centre = [cen[i] for i in alive]
    ptr = np.zeros(len(groups) + 1, dtype=np.int32)
    ptr[1:] = np.cumsum([len(g) for g in groups])
    ids = np.concatenate(groups).astype(np.int32)
    centres = np.array(box_centre)
    ext = np.array([2 * np.linalg.norm(c[g] - c[g].mean(axis=0), axis=1).max() for g in groups])
    diam = np.sqrt(3.0) * leaf
    far = _dist(centres[:, None, :], centres[None, :, :]) >= admissibility * diam
    np.fill_diagonal(far, False)
    if symmetric:
        far = np.triu(far, 1)
    gt, gs = np.nonzero(far)
    return Partition(group_ptr=ptr, group_ids=ids, centres=centres, extents=ext,
                     gt=gt.astype(np.int32), gs=gs.astype(np.int32), leaf=leaf)
