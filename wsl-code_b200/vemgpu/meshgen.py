"""Seeded Voronoi + Lloyd meshes of the unit disk and of the annulus 0.3 < r < 1 with exact
circular-arc boundary edges.

The reference makes its CVT polygon meshes with scipy + gmsh (vem/gmesh_py/get_gmesh.py:15-77,
487-556) and reads them back as VTK polygons (vem/CurvedVEM_Darcy_gpu/mesh/straight_mesh.cpp:68).
Here, without gmsh:

1. ``n`` generators drawn uniformly in the domain with ``numpy.random.default_rng(seed)``;
2. ``lloyd`` Lloyd iterations (default 20) in C++ (libvgmesh.so, vg_lloyd);
3. generators ordered along a Hilbert curve (locality of cells, nodes and edges in memory);
4. final topology from one Delaunay triangulation of the generators plus their mirror images
   across the boundary circles: the Voronoi cell of every real generator is the ring of
   circumcentres of its triangles; an edge to a mirror generator is a boundary chord, and the
   two ends of every boundary chord are projected radially onto their circle;
5. nodes numbered by first appearance over the Hilbert-ordered cells.

The computational mesh is the polygon with the chords; every chord is returned in
``arc_nodes`` / ``arc_data`` so that the solver maps it onto the exact arc.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MESHLIB = os.path.join(HERE, "libvgmesh.so")
_ml = None


def _meshlib():
    global _ml
    if _ml is None:
        if not os.path.exists(MESHLIB):
            raise RuntimeError(f"{MESHLIB} is missing: build it with `python wsl-code_b200/build.py`")
        _ml = ctypes.CDLL(MESHLIB)
        _ml.vg_lloyd.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                 ctypes.c_int]
        _ml.vg_lloyd.restype = ctypes.c_int
    return _ml


def sample(rng, n, r_in, r_out):
    out = np.empty((0, 2))
    while len(out) < n:
        p = rng.uniform(-r_out, r_out, size=(2 * (n - len(out)) + 64, 2))
        r = np.hypot(p[:, 0], p[:, 1])
        out = np.concatenate([out, p[(r < r_out) & (r > r_in)]])
    return out[:n].copy()


def lloyd(points, r_in, r_out, iterations, threads=0):
    xy = np.ascontiguousarray(points, np.float64).copy()
    if iterations > 0:
        rc = _meshlib().vg_lloyd(len(xy), xy.ctypes.data, float(r_in), float(r_out), int(iterations), int(threads))
        if rc != 0:
            raise RuntimeError("vg_lloyd failed")
    return xy


def hilbert_order(points, bits=16):
    """Permutation sorting points along a Hilbert curve on a 2^bits grid."""
    lo = points.min(axis=0)
    span = max(float((points.max(axis=0) - lo).max()), 1e-300)
    n = (1 << bits) - 1
    x = np.minimum((points[:, 0] - lo[0]) / span * n, n).astype(np.int64)
    y = np.minimum((points[:, 1] - lo[1]) / span * n, n).astype(np.int64)
    d = np.zeros(len(points), np.int64)
    s = 1 << (bits - 1)
    while s > 0:
        rx = (x & s) > 0
        ry = (y & s) > 0
        d += s * s * ((3 * rx) ^ ry)
        # rotate
        m = ~ry
        flip = m & rx
        x = np.where(flip, s - 1 - x, x)
        y = np.where(flip, s - 1 - y, y)
        x2 = np.where(m, y, x)
        y2 = np.where(m, x, y)
        x, y = x2, y2
        s >>= 1
    return np.argsort(d, kind="stable")


def _circumcenters(P, T):
    a, b, c = P[T[:, 0]], P[T[:, 1]], P[T[:, 2]]
    bx, by = b[:, 0] - a[:, 0], b[:, 1] - a[:, 1]
    cx, cy = c[:, 0] - a[:, 0], c[:, 1] - a[:, 1]
    d = 2.0 * (bx * cy - by * cx)
    b2, c2 = bx * bx + by * by, cx * cx + cy * cy
    ux = (cy * b2 - by * c2) / d
    uy = (bx * c2 - cx * b2) / d
    return np.stack([a[:, 0] + ux, a[:, 1] + uy], axis=1)


def voronoi_polygons(points, r_in, r_out):
    """Chord-polygon Voronoi mesh of ``points`` (already relaxed and ordered)."""
    from scipy.spatial import Delaunay
    n = len(points)
    h = np.sqrt(np.pi * (r_out ** 2 - r_in ** 2) / n)
    rho = np.hypot(points[:, 0], points[:, 1])
    band = 4.0 * h
    oi = np.nonzero(rho > r_out - band)[0]
    ghosts = [points[oi] * ((2 * r_out - rho[oi]) / rho[oi])[:, None]]
    kinds = [np.zeros(n, np.int8), np.ones(len(oi), np.int8)]
    if r_in > 0:
        ii = np.nonzero(rho < r_in + band)[0]
        ghosts.append(points[ii] * ((2 * r_in - rho[ii]) / rho[ii])[:, None])
        kinds.append(np.full(len(ii), 2, np.int8))
    P = np.concatenate([points] + ghosts)
    kind = np.concatenate(kinds)
    T = Delaunay(P).simplices.astype(np.int64)
    keep = (T < n).any(axis=1)
    T = T[keep]
    cc = _circumcenters(P, T)
    tk = kind[T]
    # boundary vertices: circumcentres of triangles mixing real and mirror generators
    outer = (tk == 1).any(axis=1)
    inner = (tk == 2).any(axis=1)
    r = np.hypot(cc[:, 0], cc[:, 1])
    cc[outer] *= (r_out / r[outer])[:, None]
    if r_in > 0:
        cc[inner] *= (r_in / r[inner])[:, None]
    # rings of triangles around every real generator, counter-clockwise
    owner = T.reshape(-1)
    tid = np.repeat(np.arange(len(T)), 3)
    real = owner < n
    owner, tid = owner[real], tid[real]
    ang = np.arctan2(cc[tid, 1] - points[owner, 1], cc[tid, 0] - points[owner, 0])
    order = np.lexsort((ang, owner))
    owner, tid = owner[order], tid[order]
    counts = np.bincount(owner, minlength=n)
    if (counts < 3).any():
        raise RuntimeError("Voronoi cell with fewer than 3 vertices")
    ptr = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=ptr[1:])
    # Delaunay neighbour across each polygon edge (t_i, t_{i+1}) of the ring of p
    nxt = np.arange(len(tid)) + 1
    last = ptr[1:] - 1
    nxt[last] = ptr[:-1]
    Ta, Tb = T[tid], T[tid[nxt]]
    eq = (Ta[:, :, None] == Tb[:, None, :]).any(axis=2) & (Ta != owner[:, None])
    q = np.where(eq.any(axis=1), Ta[np.arange(len(Ta)), eq.argmax(axis=1)], -1)
    if (q < 0).any():
        raise RuntimeError("inconsistent Voronoi ring")
    # collapse Voronoi edges shorter than 1% of the mean spacing (near-cocircular generators):
    # the end points are merged globally, so neighbouring cells stay conforming; a merged group
    # that contains a boundary vertex keeps that vertex's position on the circle
    vid = np.arange(len(cc))
    ring_next_t = tid[nxt]
    d = np.hypot(*(cc[tid] - cc[ring_next_t]).T)
    short = np.nonzero(d < 1e-2 * h)[0]
    if len(short):
        from scipy.sparse import coo_matrix
        from scipy.sparse.csgraph import connected_components
        a, b = tid[short], ring_next_t[short]
        members = np.unique(np.concatenate([a, b]))
        la, lb = np.searchsorted(members, a), np.searchsorted(members, b)
        g = coo_matrix((np.ones(len(la)), (la, lb)), shape=(len(members), len(members)))
        ncomp, lab = connected_components(g, directed=False)
        root = np.full(ncomp, np.iinfo(np.int64).max)
        np.minimum.at(root, lab, members)
        vid[members] = root[lab]
        onb = (outer | inner)[members]
        pos = np.zeros((ncomp, 2))
        cnt = np.zeros(ncomp)
        np.add.at(pos, lab, cc[members])
        np.add.at(cnt, lab, 1.0)
        pos /= cnt[:, None]
        bsel = np.nonzero(onb)[0]
        pos[lab[bsel]] = cc[members[bsel]]  # any boundary member (all lie on the circle)
        cc[members] = pos[lab]
    verts = vid[tid]
    edge_kind = kind[q]  # 0 interior, 1 outer chord, 2 inner chord
    # drop repeated consecutive vertices
    keepv = verts != verts[nxt]
    cell_of = owner[keepv]
    nodes = verts[keepv]
    ekind = edge_kind[keepv]
    cnt = np.bincount(cell_of, minlength=n)
    if (cnt < 3).any():
        raise RuntimeError("degenerate Voronoi cell after merging coincident vertices")
    cptr = np.zeros(n + 1, np.int64)
    np.cumsum(cnt, out=cptr[1:])
    # renumber nodes by first appearance
    uniq, first = np.unique(nodes, return_index=True)
    rank = np.empty(len(uniq), np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(uniq))
    remap = np.full(vid.max() + 1, -1, np.int64)
    remap[uniq] = rank
    cell_nodes = remap[nodes]
    xy = np.zeros((len(uniq), 2))
    vxy = np.zeros((vid.max() + 1, 2))
    vxy[vid] = cc
    xy[remap[uniq]] = vxy[uniq]
    # arcs: chords (node_i, node_{i+1}) whose dual Delaunay edge reaches a mirror generator
    nx2 = np.arange(len(cell_nodes)) + 1
    nx2[cptr[1:] - 1] = cptr[:-1]
    b = np.nonzero(ekind > 0)[0]
    arc_nodes = np.stack([cell_nodes[b], cell_nodes[nx2[b]]], axis=1).astype(np.int32)
    radius = np.where(ekind[b] == 1, r_out, r_in)
    arc_data = np.stack([np.zeros(len(b)), np.zeros(len(b)), radius], axis=1)
    return dict(xy=xy, cell_ptr=cptr.astype(np.int32), cell_nodes=cell_nodes.astype(np.int32),
                arc_nodes=arc_nodes, arc_data=arc_data, generators=points)


def voronoi_mesh(n, domain="disk", seed=0, lloyd_iterations=20, r_in=0.3, r_out=1.0, threads=0):
    """Disk (r < r_out) or annulus (r_in < r < r_out) mesh of ``n`` Voronoi cells."""
    ri = 0.0 if domain == "disk" else float(r_in)
    rng = np.random.default_rng(seed)
    pts = sample(rng, n, ri, r_out)
    pts = lloyd(pts, ri, r_out, lloyd_iterations, threads)
    pts = pts[hilbert_order(pts)]
    m = voronoi_polygons(pts, ri, r_out)
    m.update(domain=domain, r_in=ri, r_out=r_out, seed=seed, lloyd=lloyd_iterations)
    return m


def mesh_stats(m):
    cnt = np.diff(m["cell_ptr"])
    return dict(cells=len(cnt), nodes=len(m["xy"]), arcs=len(m["arc_nodes"]),
                edge_counts={int(k): int(v) for k, v in zip(*np.unique(cnt, return_counts=True))})
