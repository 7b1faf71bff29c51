"""ORACLE — test infrastructure only (the checker, never the thing measured or shipped).

Seeded Voronoi + Lloyd meshes of the unit disk and of the annulus 0.3 < r < 1 for the CPU
reference runs (the timed CPU baseline), built from numpy and scipy alone so that the CPU runs
load none of the GPU library's code.

The reference makes its CVT meshes with scipy's Voronoi diagram and a Lloyd iteration
(vem/gmesh_py/get_gmesh.py:15-77: every generator moves to the centroid of its Voronoi region,
the region clipped to the domain) and hands the polygons to gmsh (get_gmesh.py:487-556). The same
iteration here, with the domain clipping done by mirror generators:

1. ``n`` generators drawn uniformly in the domain with ``numpy.random.default_rng(seed)``
   (rejection sampling from the bounding square);
2. every generator within four mean spacings of a boundary circle gets its mirror image across
   that circle, so that the Voronoi regions of the real generators close along the boundary;
3. Lloyd: the region of each real generator (scipy.spatial.Voronoi of generators and mirrors), its
   vertices outside the domain pulled radially onto the circle, is replaced by its centroid;
4. final mesh: the regions of the real generators; a ridge between a real generator and a mirror
   is a boundary chord, its two vertices are projected onto the circle and the chord is returned
   in ``arc_nodes`` / ``arc_data`` (centre (0, 0), radius) for the exact-arc geometry.

The result is a mesh of the same family as the GPU library's own generator (same sampling, same
relaxation, same boundary treatment); the two are not bitwise identical.
"""
import numpy as np


def sample(rng, n, r_in, r_out):
    """n points uniform in r_in < |p| < r_out (rejection from the square [-r_out, r_out]^2)."""
    out = np.empty((0, 2))
    while len(out) < n:
        p = rng.uniform(-r_out, r_out, size=(2 * (n - len(out)) + 64, 2))
        r = np.hypot(p[:, 0], p[:, 1])
        out = np.concatenate([out, p[(r < r_out) & (r > r_in)]])
    return out[:n].copy()


def _with_mirrors(points, r_in, r_out):
    n = len(points)
    h = np.sqrt(np.pi * (r_out ** 2 - r_in ** 2) / n)
    rho = np.hypot(points[:, 0], points[:, 1])
    oi = np.nonzero(rho > r_out - 4.0 * h)[0]
    parts = [points, points[oi] * ((2 * r_out - rho[oi]) / rho[oi])[:, None]]
    kinds = [np.zeros(n, np.int8), np.ones(len(oi), np.int8)]
    if r_in > 0:
        ii = np.nonzero(rho < r_in + 4.0 * h)[0]
        parts.append(points[ii] * ((2 * r_in - rho[ii]) / rho[ii])[:, None])
        kinds.append(np.full(len(ii), 2, np.int8))
    return np.concatenate(parts), np.concatenate(kinds)


def _regions(vor, n):
    """(owner, vertex) pairs of the regions of the first n points, counter-clockwise per owner;
    owners whose region is unbounded are left out."""
    reg = [vor.regions[vor.point_region[i]] for i in range(n)]
    ok = np.array([len(r) >= 3 and -1 not in r for r in reg])
    owners = np.nonzero(ok)[0]
    lens = np.array([len(reg[i]) for i in owners])
    verts = np.fromiter((v for i in owners for v in reg[i]), dtype=np.int64, count=int(lens.sum()))
    own = np.repeat(owners, lens)
    c = vor.points[own]
    ang = np.arctan2(vor.vertices[verts, 1] - c[:, 1], vor.vertices[verts, 0] - c[:, 0])
    order = np.lexsort((ang, own))
    return own[order], verts[order]


def _clip_radial(v, r_in, r_out):
    r = np.hypot(v[:, 0], v[:, 1])
    v = v.copy()
    out = r > r_out
    v[out] *= (r_out / r[out])[:, None]
    if r_in > 0:
        inn = r < r_in
        v[inn] *= (r_in / np.maximum(r[inn], 1e-300))[:, None]
    return v


def lloyd(points, r_in, r_out, iterations):
    """Lloyd iterations of get_gmesh.py:15-77 on the disk / annulus (mirror-generator clipping)."""
    from scipy.spatial import Voronoi
    p = np.array(points, np.float64)
    n = len(p)
    for _ in range(iterations):
        P, _ = _with_mirrors(p, r_in, r_out)
        vor = Voronoi(P)
        own, verts = _regions(vor, n)
        v = _clip_radial(vor.vertices[verts], r_in, r_out)
        start = np.r_[0, np.nonzero(np.diff(own))[0] + 1]
        nxt = np.arange(len(own)) + 1
        nxt[np.r_[start[1:] - 1, len(own) - 1]] = start
        cross = v[:, 0] * v[nxt, 1] - v[nxt, 0] * v[:, 1]
        a = np.add.reduceat(cross, start)
        cx = np.add.reduceat((v[:, 0] + v[nxt, 0]) * cross, start)
        cy = np.add.reduceat((v[:, 1] + v[nxt, 1]) * cross, start)
        who = own[start]
        good = np.abs(a) > 1e-300
        p[who[good], 0] = cx[good] / (3.0 * a[good])
        p[who[good], 1] = cy[good] / (3.0 * a[good])
    return p


def voronoi_mesh(n, domain="annulus", seed=0, lloyd_iterations=20, r_in=0.3, r_out=1.0):
    """Polygon mesh dict(xy, cell_ptr, cell_nodes, arc_nodes, arc_data) of n Voronoi cells."""
    from scipy.spatial import Voronoi
    ri = 0.0 if domain == "disk" else float(r_in)
    rng = np.random.default_rng(seed)
    p = lloyd(sample(rng, n, ri, r_out), ri, r_out, lloyd_iterations)
    P, kind = _with_mirrors(p, ri, r_out)
    vor = Voronoi(P)
    own, verts = _regions(vor, n)
    if len(np.unique(own)) != n:
        raise RuntimeError("a real generator has an unbounded Voronoi region")
    vx = vor.vertices.copy()
    # boundary chords: ridges between a real generator and a mirror
    rp = np.asarray(vor.ridge_points)
    rv = np.asarray(vor.ridge_vertices)
    kk = kind[rp]
    bnd = ((kk[:, 0] == 0) & (kk[:, 1] > 0)) | ((kk[:, 1] == 0) & (kk[:, 0] > 0))
    chord = rv[bnd]
    radius = np.where(kk[bnd].max(axis=1) == 1, r_out, ri)
    for j in range(2):
        v = chord[:, j]
        r = np.hypot(vx[v, 0], vx[v, 1])
        vx[v] *= (radius / r)[:, None]
    # Voronoi edges shorter than 1 % of the mean spacing (nearly cocircular generators, mostly
    # where a boundary cell meets its neighbour's mirror) are collapsed: their end points merge
    # into one node everywhere, a merged group on the boundary keeps a boundary position
    h = np.sqrt(np.pi * (r_out ** 2 - ri ** 2) / n)
    start = np.r_[0, np.nonzero(np.diff(own))[0] + 1]
    nxt = np.arange(len(own)) + 1
    nxt[np.r_[start[1:] - 1, len(own) - 1]] = start
    short = np.nonzero(np.hypot(*(vx[verts] - vx[verts[nxt]]).T) < 1e-2 * h)[0]
    vid = np.arange(len(vx))
    if len(short):
        from scipy.sparse import coo_matrix
        from scipy.sparse.csgraph import connected_components
        a, b = verts[short], verts[nxt[short]]
        members = np.unique(np.concatenate([a, b]))
        g = coo_matrix((np.ones(len(a)), (np.searchsorted(members, a), np.searchsorted(members, b))),
                       shape=(len(members), len(members)))
        ncomp, lab = connected_components(g, directed=False)
        root = np.full(ncomp, np.iinfo(np.int64).max)
        np.minimum.at(root, lab, members)
        pos = np.zeros((ncomp, 2))
        cnt = np.zeros(ncomp)
        np.add.at(pos, lab, vx[members])
        np.add.at(cnt, lab, 1.0)
        pos /= cnt[:, None]
        onb = np.zeros(len(vx), bool)
        onb[chord.reshape(-1)] = True
        bsel = np.nonzero(onb[members])[0]
        pos[lab[bsel]] = vx[members[bsel]]
        vx[members] = pos[lab]
        vid[members] = root[lab]
    verts = vid[verts]
    chord = vid[chord]
    keep = verts != verts[nxt]
    own, verts = own[keep], verts[keep]
    chord = chord[chord[:, 0] != chord[:, 1]]
    radius = np.hypot(vx[chord[:, 0], 0], vx[chord[:, 0], 1])
    radius = np.where(np.abs(radius - r_out) < np.abs(radius - ri), r_out, ri)
    if (np.bincount(own, minlength=n) < 3).any():
        raise RuntimeError("degenerate Voronoi cell after merging coincident vertices")
    # nodes numbered by first use over the cells
    uniq, first = np.unique(verts, return_index=True)
    rank = np.empty(len(uniq), np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(uniq))
    remap = np.full(len(vx), -1, np.int64)
    remap[uniq] = rank
    xy = np.zeros((len(uniq), 2))
    xy[remap[uniq]] = vx[uniq]
    counts = np.bincount(own, minlength=n)
    ptr = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=ptr[1:])
    return dict(xy=xy, cell_ptr=ptr.astype(np.int32), cell_nodes=remap[verts].astype(np.int32),
                arc_nodes=remap[chord].astype(np.int32),
                arc_data=np.stack([np.zeros(len(chord)), np.zeros(len(chord)), radius], axis=1))
