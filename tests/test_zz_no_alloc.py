"""vg_errors_noalloc (static device scratch, no device allocation) against vg_errors, through the
C ABI. The figures come from the same kernels and the same fixed-order reduction, so they must
agree bit for bit, on repeated calls and across handles that reuse the same static scratch, and
the entry point must keep working when the device has no memory left to allocate (the situation
of a caller whose caching allocator holds all of HBM)."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import vemgpu  # noqa: E402
from vemgpu import _lib as L  # noqa: E402
from vemgpu import meshgen  # noqa: E402


def _figures(g, x, fn):
    out = (ctypes.c_double * 6)()
    L.check(getattr(L.lib(), fn)(g.h, ctypes.c_void_p(x.data_ptr()), out), g.h)
    return np.array(list(out))


def _grid(n):
    """n x n unit squares on [0, 1]^2 as raw polygons."""
    t = np.linspace(0.0, 1.0, n + 1)
    X, Y = np.meshgrid(t, t, indexing="xy")
    xy = np.stack([X.ravel(), Y.ravel()], 1)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    v0 = (j * (n + 1) + i).ravel()
    cells = np.stack([v0, v0 + 1, v0 + n + 2, v0 + n + 1], 1)
    return dict(xy=xy, cell_ptr=np.arange(0, 4 * n * n + 1, 4), cell_nodes=cells.ravel())


@pytest.mark.parametrize("k,geometry,problem,bc", [(0, "arcs", "annulus", "pressure"), (1, "sine", "sincos", "flux")])
def test_noalloc_matches_errors(k, geometry, problem, bc):
    mesh = meshgen.voronoi_mesh(3000, "annulus" if geometry == "arcs" else "disk", seed=11)
    g = vemgpu.DarcyGpu(mesh, k=k, geometry=geometry, eps=0.05 if geometry == "sine" else 0.0,
                        problem=problem, bc=bc)
    x, info = g.solve(g.rhs(), tol=1e-10)
    ref = _figures(g, x, "vg_errors")
    for _ in range(2):  # two calls in a row: the scratch is reused without clearing
        got = _figures(g, x, "vg_errors_noalloc")
        assert np.array_equal(got, ref), (got, ref)
    # a second, smaller handle on the same device reuses the same scratch
    h = vemgpu.DarcyGpu(meshgen.voronoi_mesh(500, "disk", seed=12), k=k, geometry="identity", problem="sincos",
                        bc="flux")
    y, _ = h.solve(h.rhs(), tol=1e-10)
    ref_h = _figures(h, y, "vg_errors")
    for _ in range(2):
        assert np.array_equal(_figures(h, y, "vg_errors_noalloc"), ref_h)
    assert np.array_equal(_figures(g, x, "vg_errors_noalloc"), ref)
    h.close()
    g.close()


def test_noalloc_rejects_meshes_above_limit():
    n = 520  # 270,400 cells > VG_ERRORS_NOALLOC_MAX_CELLS = 262,144
    g = vemgpu.DarcyGpu(_grid(n), k=0, geometry="identity", problem="sincos", bc="flux")
    x = torch.zeros(g.N, dtype=torch.float64, device="cuda")
    with pytest.raises(L.VemGpuError) as e:
        _figures(g, x, "vg_errors_noalloc")
    assert e.value.code == L.VG_EINVAL
    assert "VG_ERRORS_NOALLOC_MAX_CELLS" in str(e.value)
    # the ordinary entry point still works on the same handle
    assert np.all(np.isfinite(_figures(g, x, "vg_errors")))
    g.close()


def test_noalloc_works_with_device_memory_exhausted():
    """With every free byte of the device taken, vg_errors (which allocates its per-cell scratch)
    returns VG_ENOMEM while vg_errors_noalloc still returns the same figures, twice in a row."""
    from cuda.bindings import runtime as rt
    n = 440  # 193,600 cells: vg_errors asks for 6 * 193,600 doubles = 9.3 MB of scratch
    g = vemgpu.DarcyGpu(_grid(n), k=0, geometry="identity", problem="sincos", bc="flux")
    x = torch.randn(g.N, dtype=torch.float64, device="cuda")
    ref = _figures(g, x, "vg_errors")
    assert np.array_equal(_figures(g, x, "vg_errors_noalloc"), ref)  # loads the kernels first
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    held = []
    try:
        # take the device's free memory in decreasing blocks, down to 2 MB
        size = 1 << 30
        while size >= (2 << 20):
            err, ptr = rt.cudaMalloc(size)
            if err == rt.cudaError_t.cudaSuccess:
                held.append(ptr)
            else:
                rt.cudaGetLastError()
                size //= 2
        err, free, _ = rt.cudaMemGetInfo()
        assert err == rt.cudaError_t.cudaSuccess and free < 6 * 8 * g.nc, free
        with pytest.raises(L.VemGpuError) as e:
            _figures(g, x, "vg_errors")
        assert e.value.code == L.VG_ENOMEM
        for _ in range(2):
            assert np.array_equal(_figures(g, x, "vg_errors_noalloc"), ref)
    finally:
        for ptr in held:
            rt.cudaFree(ptr)
    assert np.array_equal(_figures(g, x, "vg_errors"), ref)
    g.close()
