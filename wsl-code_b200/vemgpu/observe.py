"""Point observations of the discrete pressure: p_h(x_o) for observation points x_o.

For k = 0 the pressure is one constant per cell, so p_h(x_o) is the pressure unknown of the cell
that contains x_o (cell-major pressure block after the flux unknowns). Points are located on the
host against the straight (chord) polygons of the computational mesh; observation points are meant
to lie in the interior, away from the thin region between a boundary chord and its arc.
"""
import numpy as np


def locate_cells(mesh, points, candidates=12):
    """Index of the polygon containing each point (-1 if none): nearest centroids first, then an
    even-odd crossing test on the polygon."""
    from scipy.spatial import cKDTree
    xy = np.asarray(mesh["xy"], np.float64).reshape(-1, 2)
    ptr = np.asarray(mesh["cell_ptr"], np.int64)
    nodes = np.asarray(mesh["cell_nodes"], np.int64)
    nc = len(ptr) - 1
    cid = np.repeat(np.arange(nc), np.diff(ptr))
    cen = np.zeros((nc, 2))
    np.add.at(cen, cid, xy[nodes])
    cen /= np.diff(ptr)[:, None]
    tree = cKDTree(cen)
    pts = np.asarray(points, np.float64).reshape(-1, 2)
    out = np.full(len(pts), -1, np.int64)
    _, near = tree.query(pts, k=min(candidates, nc))
    near = np.atleast_2d(near)
    for i, p in enumerate(pts):
        for c in near[i]:
            poly = xy[nodes[ptr[c]:ptr[c + 1]]]
            x0, y0 = poly[:, 0], poly[:, 1]
            x1, y1 = np.roll(x0, -1), np.roll(y0, -1)
            cross = ((y0 > p[1]) != (y1 > p[1])) & (p[0] < (x1 - x0) * (p[1] - y0) / (y1 - y0 + 1e-300) + x0)
            if np.count_nonzero(cross) % 2 == 1:
                out[i] = c
                break
    return out


class PointObservation:
    """J(x) = sum_o (p_h(x_o) - d_o)^2 as a torch function of the solution vector (k = 0)."""

    def __init__(self, handle, mesh, points, data=None):
        if handle.k != 0:
            raise NotImplementedError("point observations are implemented for k = 0")
        cells = locate_cells(mesh, points)
        if np.any(cells < 0):
            raise ValueError("observation point outside the mesh")
        import torch
        self.cells = cells
        self.index = torch.as_tensor(handle.nf + cells * handle.q, dtype=torch.long, device="cuda")
        d = np.zeros(len(cells)) if data is None else np.asarray(data, np.float64)
        self.data = torch.as_tensor(d, dtype=torch.float64, device="cuda")

    def pressure(self, x):
        return x[self.index]

    def __call__(self, x):
        r = self.pressure(x) - self.data
        return (r * r).sum()


def seeded_points(n, seed, r_in=0.35, r_out=0.95):
    """n points uniformly distributed in the annulus r_in < r < r_out (interior of the workload's
    0.3 < r < 1 domain)."""
    rng = np.random.default_rng(seed)
    r = np.sqrt(rng.uniform(r_in * r_in, r_out * r_out, n))
    t = rng.uniform(0, 2 * np.pi, n)
    return np.stack([r * np.cos(t), r * np.sin(t)], 1)
