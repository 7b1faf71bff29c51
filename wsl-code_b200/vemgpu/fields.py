"""Seeded Gaussian random fields for the log permeability theta = log K.

Exponential covariance C(r) = sigma^2 exp(-r / corr) sampled by FFT on a periodic grid that
embeds the box [-box, box]^2 twice over (torus of side 4 box, so the covariance of the sampled
window is the free-space one), eigenvalues of the circulant covariance clipped at zero,
evaluated at arbitrary points by bilinear interpolation.
"""
import numpy as np


def gaussian_field(points, sigma=2.0, corr=0.1, seed=0, box=1.25, grid=1024):
    """Values of one field realisation at ``points`` (n, 2)."""
    rng = np.random.default_rng(seed)
    side = 4.0 * box
    m = 2 * grid
    dx = side / m
    i = np.arange(m)
    d = np.minimum(i, m - i) * dx
    r = np.hypot(d[:, None], d[None, :])
    cov = sigma * sigma * np.exp(-r / corr)
    lam = np.maximum(np.fft.fft2(cov).real, 0.0)
    xi = rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))
    f = np.fft.fft2(np.sqrt(lam / (m * m)) * xi).real
    # window [-box, box]^2 -> grid indices [0, grid]
    g = (np.asarray(points, np.float64) + box) / dx
    g = np.clip(g, 0.0, grid - 1.000001)
    i0 = np.floor(g).astype(np.int64)
    t = g - i0
    x0, y0 = i0[:, 0], i0[:, 1]
    v = (f[x0, y0] * (1 - t[:, 0]) * (1 - t[:, 1]) + f[x0 + 1, y0] * t[:, 0] * (1 - t[:, 1]) +
         f[x0, y0 + 1] * (1 - t[:, 0]) * t[:, 1] + f[x0 + 1, y0 + 1] * t[:, 0] * t[:, 1])
    return v


def cell_centroids(mesh):
    """Vertex averages of the cells (the reference's centroid rule for non-quadrilaterals)."""
    xy, ptr, nodes = mesh["xy"], mesh["cell_ptr"], mesh["cell_nodes"]
    cnt = np.diff(ptr)
    s = np.zeros((len(cnt), 2))
    np.add.at(s, np.repeat(np.arange(len(cnt)), cnt), xy[nodes])
    return s / cnt[:, None]
