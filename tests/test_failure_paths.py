"""Failure paths: every error the library detects comes back as a status code, and the handle
stays usable afterwards. No test faults, traps or hangs the GPU: the device-side case makes one
bounded wait of the streamed apply run out (a consumer waiting on a barrier that nothing arrives
on) through the test hook vg_debug_stall_apply, and checks that the kernel returns and the call
reports VG_ECUDA.

Reference counterparts: the true-residual failure of Krylov::solve
(vem/CurvedVEM_Darcy_gpu/src/krylov.cu:171-174), the singular-pivot status of the local inverse
(vem/CurvedVEM_Darcy_gpu/include/device.cuh:243-244), the degenerate-element and Jacobian checks
of the mesh packing (vem/CurvedVEM_Darcy_gpu/src/mesh_pack.cpp:77-88).
"""
import ctypes

import numpy as np
import pytest

from vemgpu import _lib as L


def _square(n=2):
    xs = np.linspace(0, 1, n + 1)
    xy = np.array([(x, y) for y in xs for x in xs])
    cells = []
    for j in range(n):
        for i in range(n):
            a = j * (n + 1) + i
            cells.append([a, a + 1, a + n + 2, a + n + 1])
    return dict(xy=xy, cell_ptr=np.arange(0, 4 * len(cells) + 1, 4, dtype=np.int32),
                cell_nodes=np.array(cells, np.int32).reshape(-1))


def _create_code(mesh, k=0):
    """Status of vg_create_polygons for a raw polygon mesh (host checks run before device work)."""
    h = ctypes.c_void_p()
    g = L.VgGeometry()
    xy = np.ascontiguousarray(mesh["xy"], np.float64)
    ptr = np.ascontiguousarray(mesh["cell_ptr"], np.int32)
    nodes = np.ascontiguousarray(mesh["cell_nodes"], np.int32)
    code = L.lib().vg_create_polygons(len(xy), xy.ctypes.data, len(ptr) - 1, ptr.ctypes.data, nodes.ctypes.data,
                                      ctypes.byref(g), k, 9, 9, -1, ctypes.byref(h))
    if h.value:
        L.lib().vg_destroy(h)
    return code, L.lib().vg_last_error(None).decode()


def test_zero_length_edge_rejected():
    m = _square()
    nodes = m["cell_nodes"].copy()
    nodes[1] = nodes[0]  # cell 0 repeats a node: an edge of length zero
    code, msg = _create_code(dict(m, cell_nodes=nodes))
    assert code == L.VG_EMESH and "zero-length edge" in msg
    xy = m["xy"].copy()
    xy[1] = xy[0]  # two distinct nodes at one point
    code, msg = _create_code(dict(m, xy=xy))
    assert code == L.VG_EMESH and "zero-length edge" in msg


def test_zero_area_cell_rejected():
    xy = np.array([[0, 0], [1, 0], [2, 0], [1, 1]], float)
    mesh = dict(xy=xy, cell_ptr=np.array([0, 3], np.int32), cell_nodes=np.array([0, 1, 2], np.int32))
    code, msg = _create_code(mesh)
    assert code == L.VG_EMESH and "zero area" in msg


def test_non_finite_node_rejected():
    m = _square()
    xy = m["xy"].copy()
    xy[4, 0] = np.nan
    code, msg = _create_code(dict(m, xy=xy))
    assert code == L.VG_EMESH and "non-finite" in msg


# ---- on the GPU ---------------------------------------------------------------------------------

def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import vemgpu
    return torch, vemgpu


@pytest.mark.gpu
def test_iteration_cap_reports_no_convergence():
    torch, vemgpu = _gpu()
    from vemgpu import meshgen
    g = vemgpu.DarcyGpu(meshgen.voronoi_mesh(2000, "annulus", seed=71), k=0, geometry="arcs", problem="annulus",
                        bc="pressure")
    for mode in ("fp64", "mixed"):
        with pytest.raises(L.VemGpuError) as e:
            g.solve(mode=mode, tol=1e-10, maxit=1)
        assert e.value.code == L.VG_ENOCONV and "did not converge" in str(e.value)
    x, info = g.solve(tol=1e-10)  # the handle is still usable
    assert info["residual"] <= 1e-10
    g.close()


@pytest.mark.gpu
def test_non_finite_permeability_rejected():
    torch, vemgpu = _gpu()
    from vemgpu import meshgen
    m = meshgen.voronoi_mesh(1500, "annulus", seed=72)
    th = np.random.default_rng(73).normal(0, 1, 1500)
    g = vemgpu.DarcyGpu(m, k=0, geometry="arcs", problem="annulus", bc="pressure", theta=th)
    x0, _ = g.solve(tol=1e-12)
    bad = th.copy()
    bad[17] = np.nan
    with pytest.raises(L.VemGpuError) as e:
        g.set_log_permeability(bad)
    assert e.value.code == L.VG_EINVAL and "cell 17" in str(e.value)
    bad = torch.tensor(th, dtype=torch.float64, device="cuda")
    bad[1234] = float("inf")
    with pytest.raises(L.VemGpuError) as e:
        g.set_log_permeability(bad)
    assert e.value.code == L.VG_EINVAL and "cell 1234" in str(e.value)
    # the field of the handle did not change
    x1, _ = g.solve(tol=1e-12)
    assert torch.equal(x0, x1)
    g.close()


@pytest.mark.gpu
def test_nonpositive_jacobian_reported():
    torch, vemgpu = _gpu()
    # x + eps sin(2 pi y), y + eps sin(2 pi x) folds over for eps > 1 / (2 pi): det J < 0 near (0, 0)
    with pytest.raises(L.VemGpuError) as e:
        vemgpu.DarcyGpu(_square(4), k=0, geometry="sine", eps=0.3, problem="sincos", bc="flux")
    assert e.value.code == L.VG_EGEOMETRY and "nonpositive Jacobian" in str(e.value)


@pytest.mark.gpu
def test_singular_local_matrix_reported():
    torch, vemgpu = _gpu()
    # a square of side 1e-15 (area 1e-30): the pivots of its scaled-monomial mass matrix H are of
    # the size of the area, far below the inverse's absolute singular threshold 1e-28 (the
    # reference's, vem/CurvedVEM_Darcy_gpu/include/device.cuh:243-244)
    s = 1e-15
    xy = np.array([[0, 0], [s, 0], [s, s], [0, s]], float)
    mesh = dict(xy=xy, cell_ptr=np.array([0, 4], np.int32), cell_nodes=np.array([0, 1, 2, 3], np.int32))
    with pytest.raises(L.VemGpuError) as e:
        vemgpu.DarcyGpu(mesh, k=1, geometry="identity", problem="sincos", bc="flux")
    assert e.value.code == L.VG_ESINGULAR and "singular local matrix" in str(e.value)


@pytest.mark.gpu
def test_apply_wait_limit_reports_error_and_recovers():
    """The streamed apply's pipeline: one consumer's one-second wait runs out, the kernel drains
    its copies and returns, vg_apply reports VG_ECUDA on the next call and vg_solve at its end;
    afterwards the handle computes correct results again."""
    torch, vemgpu = _gpu()
    from vemgpu import meshgen
    g = vemgpu.DarcyGpu(meshgen.voronoi_mesh(20000, "annulus", seed=74), k=0, geometry="arcs", problem="annulus",
                        bc="pressure")
    x = torch.randn(g.N, dtype=torch.float64, device="cuda")
    ref = g.apply(x)
    torch.cuda.synchronize()
    L.check(L.lib().vg_debug_stall_apply(g.h), g.h)
    g.apply(x)  # asynchronous: returns before the kernel has given up
    torch.cuda.synchronize()
    with pytest.raises(L.VemGpuError) as e:
        g.apply(x)
    assert e.value.code == L.VG_ECUDA and "pipeline" in str(e.value)
    torch.cuda.synchronize()
    assert torch.equal(g.apply(x), ref)
    torch.cuda.synchronize()
    # the same inside a solve: the solve ends and reports the failure
    L.check(L.lib().vg_debug_stall_apply(g.h), g.h)
    with pytest.raises(L.VemGpuError) as e:
        g.solve(tol=1e-10, maxit=2000)
    assert e.value.code == L.VG_ECUDA and "pipeline" in str(e.value)
    x1, info = g.solve(tol=1e-10)
    assert info["residual"] <= 1e-10
    g.close()
