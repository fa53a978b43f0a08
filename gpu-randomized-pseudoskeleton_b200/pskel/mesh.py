"""Surface meshes and RWG topology in the reference's array conventions.

Every mesh is returned as an :class:`RWGMesh` whose arrays follow the layout that the
reference's Julia drivers pass through ``ccall`` (column-major Float64, 1-based ids):

* ``vertex`` 3 x Nv, ``topol`` 3 x Nt (vertex ids),
* ``edges`` 4 x Ne: T+, T-, opposite vertex in T+, opposite vertex in T-
  (``get_edge.m:105-108``),
* ``trian`` 3 x Nt: +e where the triangle is T+ of edge e with the opposite vertex in that
  row, -e for T- (``get_edge.m:110-113``),
* ``ln`` Ne edge lengths, ``cent`` 3 x Nt centroids, ``un`` 3 x Nt unit normals of
  cross(v3-v1, v2-v1), ``ds`` 1 x Nt areas (``get_edge.m:115-131``).

Generators:

* :func:`octa_sphere` - the reference's octahedral sphere (``objects/sphere.m:13-53``,
  Julia twin ``compres_single_block_spheres_for_sweep2.jl:88-184``), Ne = 12*4^n.
* :func:`two_spheres` - two twin spheres displaced along x
  (``object_wrapper_spheres_interaction2.m:1-54``); edges 1..N/2 lie on sphere 1.
* :func:`two_plates` - two parallel square plates in xy, each an n x n grid of squares split
  along one diagonal (the single-block plate workload: 800 triangles, 1160 RWG per plate).
* :func:`icosphere` - icosahedron subdivided ``n`` times and projected to radius R
  (20*4^n triangles, 30*4^n RWG).
* :func:`ellipsoid`, :func:`cube` - seeded training geometries for the rank predictor.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class RWGMesh:
    vertex: np.ndarray  # (3, Nv) float64
    topol: np.ndarray  # (3, Nt) int64, 1-based
    trian: np.ndarray  # (3, Nt) int64, signed 1-based edge ids
    edges: np.ndarray  # (4, Ne) int64, 1-based
    un: np.ndarray  # (3, Nt)
    ds: np.ndarray  # (1, Nt)
    ln: np.ndarray  # (Ne,)
    cent: np.ndarray  # (3, Nt)
    name: str = "mesh"

    @property
    def N(self) -> int:
        return int(self.edges.shape[1])

    @property
    def Nt(self) -> int:
        return int(self.topol.shape[1])

    @property
    def Nv(self) -> int:
        return int(self.vertex.shape[1])

    def basis_centres(self) -> np.ndarray:
        """(3, Ne) centre of each RWG: mean of its two triangle centroids
        (``user_get_OG_basis_center.m:36-39``)."""
        tp = self.edges[0] - 1
        tm = self.edges[1] - 1
        return 0.5 * (self.cent[:, tp] + self.cent[:, tm])

    def as_f64(self) -> dict:
        """Arrays converted the way the Julia wrappers convert them before ``ccall``
        (``compres_single_block_spheres_for_sweep2.jl:380-388``): Fortran-ordered Float64."""
        f = lambda a: np.asfortranarray(np.asarray(a, dtype=np.float64))
        return dict(
            vertex=f(self.vertex), topol=f(self.topol), trian=f(self.trian),
            edges=f(self.edges), un=f(self.un), ds=f(self.ds.reshape(1, -1)),
            ln=np.ascontiguousarray(self.ln, dtype=np.float64), cent=f(self.cent),
        )


def get_edge(vertex: np.ndarray, topol: np.ndarray, name: str = "mesh") -> RWGMesh:
    """Build RWG topology from vertices and 1-based triangle connectivity.

    Restates ``get_edge.m:16-131`` for manifold meshes (no junctions): the 3*Nt directed
    triangle edges are listed slot-major ([v1 v2], [v2 v3], [v3 v1] for all triangles),
    sorted by (min vertex, max vertex) with a stable sort; each pair of equal rows is one
    RWG whose T+ is the later row of the pair and T- the earlier one. Boundary edges
    (a single triangle) carry no basis function.
    """
    vertex = np.ascontiguousarray(vertex, dtype=np.float64)
    topol = np.ascontiguousarray(topol, dtype=np.int64)
    nt = topol.shape[1]
    v1, v2, v3 = topol[0], topol[1], topol[2]
    t = np.arange(1, nt + 1, dtype=np.int64)
    tt = np.concatenate([t, t, t])
    e = np.stack([np.concatenate([v1, v2, v3]), np.concatenate([v2, v3, v1])])
    vv = np.concatenate([v3, v1, v2])
    ov = np.concatenate([np.full(nt, 3), np.full(nt, 1), np.full(nt, 2)]).astype(np.int64)
    e1 = np.sort(e, axis=0)
    # stable lexicographic sort of rows (first, then second vertex)
    ie2 = np.lexsort((e1[1], e1[0]))
    e2 = e1[:, ie2]
    same = np.all(e2[:, 1:] == e2[:, :-1], axis=0)
    e4 = np.concatenate([[False], same])  # row equals its predecessor
    e5 = np.concatenate([same, [False]])  # row equals its successor
    if np.any(e4 & e5):
        raise ValueError("non-manifold edge (junction): more than two triangles share an edge")
    vv1 = vv[ie2[e4]]
    vv2 = vv[ie2[e5]]
    tt1 = tt[ie2[e4]]
    tt2 = tt[ie2[e5]]
    ov1 = ov[ie2[e4]]
    ov2 = ov[ie2[e5]]
    ne = tt1.shape[0]
    edges = np.stack([tt1, tt2, vv1, vv2]).astype(np.int64)
    ids = np.arange(1, ne + 1, dtype=np.int64)
    trianp = np.zeros((3, nt), dtype=np.int64)
    trianm = np.zeros((3, nt), dtype=np.int64)
    np.add.at(trianp, (ov1 - 1, tt1 - 1), ids)
    np.add.at(trianm, (ov2 - 1, tt2 - 1), ids)
    trian = trianp - trianm
    ea = e[0, ie2[e4]] - 1
    eb = e[1, ie2[e4]] - 1
    ln = np.sqrt(np.sum((vertex[:, ea] - vertex[:, eb]) ** 2, axis=0))
    p1 = vertex[:, v1 - 1]
    p2 = vertex[:, v2 - 1]
    p3 = vertex[:, v3 - 1]
    cent = (p1 + p2 + p3) / 3.0
    c = np.cross((p3 - p1).T, (p2 - p1).T).T
    cn = np.sqrt(np.sum(c ** 2, axis=0))
    un = c / cn
    ds = (cn / 2.0).reshape(1, -1)
    return RWGMesh(vertex=vertex, topol=topol, trian=trian, edges=edges, un=un, ds=ds,
                   ln=ln, cent=cent, name=name)


def _octa_sphere_raw(R: float, Ne: int):
    n = math.log(Ne / 12) / math.log(4)
    if abs(n - round(n)) > 1e-12:
        raise ValueError("Ne must be 12*4^n")
    n = int(round(n))
    vert = [np.array(v, dtype=np.float64) * R for v in
            ([0, 0, 1], [1, 0, 0], [0, 1, 0], [-1, 0, 0], [0, -1, 0], [0, 0, -1])]
    topol = [list(c) for c in zip([1, 1, 1, 1, 6, 6, 6, 6], [3, 4, 5, 2, 2, 3, 4, 5],
                                  [2, 3, 4, 5, 3, 4, 5, 2])]
    index = {tuple(v.tolist()): i + 1 for i, v in enumerate(vert)}

    def mid(a, b):
        r = (vert[a - 1] + vert[b - 1]) / 2.0
        r = r * R / math.sqrt(float(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]))
        key = tuple(r.tolist())
        if key in index:
            return index[key]
        vert.append(r)
        index[key] = len(vert)
        return len(vert)

    nt = 8
    for _ in range(n):
        for t in range(nt):
            a, b, c = topol[t]
            v12 = mid(a, b)
            v23 = mid(b, c)
            v31 = mid(c, a)
            topol[t] = [v12, v23, v31]
            topol.append([b, v23, v12])
            topol.append([v23, c, v31])
            topol.append([v31, a, v12])
        nt *= 4
    return np.array(vert).T.copy(), np.array(topol, dtype=np.int64).T.copy()


def octa_sphere(R: float, Ne: int) -> RWGMesh:
    """Octahedral sphere of radius R with Ne = 12*4^n RWG (``objects/sphere.m:13-53``)."""
    v, t = _octa_sphere_raw(R, Ne)
    return get_edge(v, t, name="sphere")


def two_spheres(radius: float, d: float, Ne: int) -> RWGMesh:
    """Two octahedral spheres, the second shifted by d along x; joined before the RWG
    build (``object_wrapper_spheres_interaction2.m:19-41``). RWG 1..Ne lie on sphere 1."""
    v1, t1 = _octa_sphere_raw(radius, Ne)
    v2 = v1.copy()
    v2[0] += d
    nv1 = v1.shape[1]
    v = np.concatenate([v1, v2], axis=1)
    t = np.concatenate([t1, t1 + nv1], axis=1)
    return get_edge(v, t, name="two_spheres")


def _plate_raw(side: float, n: int, z: float):
    xs = np.linspace(-side / 2, side / 2, n + 1)
    gx, gy = np.meshgrid(xs, xs, indexing="ij")  # vertex (i, j) -> id i*(n+1)+j+1
    vert = np.stack([gx.ravel(), gy.ravel(), np.full(gx.size, z)])
    tris = []
    for i in range(n):
        for j in range(n):
            a = i * (n + 1) + j + 1
            b = (i + 1) * (n + 1) + j + 1
            c = (i + 1) * (n + 1) + j + 2
            d = i * (n + 1) + j + 2
            tris.append([a, b, c])  # split along the a-c diagonal
            tris.append([a, c, d])
    return vert, np.array(tris, dtype=np.int64).T.copy()


def two_plates(side: float = 1.0, n: int = 20, gap: float = 3.0) -> RWGMesh:
    """Two parallel square plates in the xy plane, centres (0,0,0) and (0,0,gap); each an
    n x n grid split along one diagonal (2n^2 triangles, 3n^2-2n interior RWG per plate).
    RWG 1..N/2 lie on the first plate."""
    v1, t1 = _plate_raw(side, n, 0.0)
    v2, t2 = _plate_raw(side, n, gap)
    nv1 = v1.shape[1]
    v = np.concatenate([v1, v2], axis=1)
    t = np.concatenate([t1, t2 + nv1], axis=1)
    return get_edge(v, t, name="two_plates")


def _icosahedron():
    p = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0],
                  [0, -1, p], [0, 1, p], [0, -1, -p], [0, 1, -p],
                  [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    return v, f


def _subdivide_unit(v: np.ndarray, f: np.ndarray, levels: int):
    """Loop-free midpoint subdivision with midpoints projected to the unit sphere."""
    for _ in range(levels):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        es = np.sort(e, axis=1)
        uniq, inv = np.unique(es, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        m = 0.5 * (v[uniq[:, 0]] + v[uniq[:, 1]])
        m /= np.linalg.norm(m, axis=1, keepdims=True)
        mid = inv + v.shape[0]
        nf = f.shape[0]
        m01, m12, m20 = mid[:nf], mid[nf:2 * nf], mid[2 * nf:]
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        f = np.concatenate([np.stack([a, m01, m20], 1), np.stack([b, m12, m01], 1),
                            np.stack([c, m20, m12], 1), np.stack([m01, m12, m20], 1)])
        v = np.concatenate([v, m])
    return v, f


def icosphere(R: float, subdivisions: int, centre=(0.0, 0.0, 0.0)) -> RWGMesh:
    """Icosahedron subdivided ``subdivisions`` times, vertices on radius R.
    5 subdivisions: 20,480 triangles and 30,720 RWG; 6: 81,920 and 122,880."""
    v, f = _icosahedron()
    v, f = _subdivide_unit(v, f, subdivisions)
    v = v * R + np.asarray(centre, dtype=np.float64)
    return get_edge(v.T.copy(), (f + 1).T.copy(), name=f"icosphere{subdivisions}")


def ellipsoid(a: float, b: float, c: float, edge: float, max_rwg: int = 1 << 30) -> RWGMesh:
    """Ellipsoid with semi-axes (a, b, c): an icosphere scaled per axis, subdivided until the
    mean edge length is at most ``edge`` or one more subdivision would exceed ``max_rwg``
    RWG functions (30 * 4^level)."""
    v0, f0 = _icosahedron()
    lev = 0
    while True:
        v, f = _subdivide_unit(v0, f0, lev)
        w = v * np.array([a, b, c])
        el = np.linalg.norm(w[f[:, 0]] - w[f[:, 1]], axis=1).mean()
        if el <= edge or lev >= 8 or 30 * 4 ** (lev + 1) > max_rwg:
            break
        lev += 1
    return get_edge(w.T.copy(), (f + 1).T.copy(), name="ellipsoid")


def cube(side: float, edge: float, max_rwg: int = 1 << 30) -> RWGMesh:
    """Closed cube of the given side, each face an n x n grid (n = ceil(side/edge), reduced
    until the 18 n^2 RWG fit in ``max_rwg``) split along one diagonal; shared face-boundary
    vertices are merged."""
    n = max(1, int(math.ceil(side / edge)))
    while n > 1 and 18 * n * n > max_rwg:
        n -= 1
    h = side / 2
    s = np.linspace(-h, h, n + 1)
    verts = {}
    vlist = []
    tris = []

    def vid(p):
        key = tuple(np.round(p, 12).tolist())
        if key not in verts:
            vlist.append(p)
            verts[key] = len(vlist)
        return verts[key]

    faces = []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            faces.append((axis, sign))
    for axis, sign in faces:
        u_ax, v_ax = [i for i in range(3) if i != axis]
        ids = np.zeros((n + 1, n + 1), dtype=np.int64)
        for i in range(n + 1):
            for j in range(n + 1):
                p = np.zeros(3)
                p[axis] = sign * h
                p[u_ax] = s[i]
                p[v_ax] = s[j]
                ids[i, j] = vid(p)
        for i in range(n):
            for j in range(n):
                a, b, c, d = ids[i, j], ids[i + 1, j], ids[i + 1, j + 1], ids[i, j + 1]
                if sign > 0:
                    tris.append([a, b, c]); tris.append([a, c, d])
                else:
                    tris.append([a, c, b]); tris.append([a, d, c])
    v = np.array(vlist).T.copy()
    t = np.array(tris, dtype=np.int64).T.copy()
    return get_edge(v, t, name="cube")
