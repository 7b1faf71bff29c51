"""GPU parity: the CUDA library (through the C ABI) against the CPU FP64 oracle and the
reference's golden results. Tolerances are written in each test:

* FP64 local operators and apply: relative 1e-12 (same FP64 mathematics, different summation
  order and the reference GPU's exact edge moments instead of edge quadrature);
* FP32 operator: relative 2e-6 of the FP64 result;
* solutions: relative 2-norm difference to the oracle's sparse-LU solution at most 1e-10 (the
  discrete-solution target), for solves to the reference's true-residual tolerance 1e-10 on the
  C1 disk and the lognormal annuli, and to 1e-12 where the test says so;
* golden error figures: the oracle's own tolerances (tests/test_oracle_golden.py).
"""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import vemgpu  # noqa: E402
from vemgpu import default_nq  # noqa: E402
from vemgpu import meshgen  # noqa: E402

GEO = {O.GEOM_IDENTITY: "identity", O.GEOM_SINE: "sine", O.GEOM_ARCS: "arcs"}
PROB = {O.PROB_SINCOS: "sincos", O.PROB_SINSIN: "sinsin", O.PROB_ANNULUS: "annulus"}
BCN = {O.BC_FLUX: "flux", O.BC_PRESSURE: "pressure"}


def pair(mesh, k, nq, geom, eps, problem, bc, theta=None, ng=9):
    ng = max(ng, k + 2)
    o = O.Oracle(mesh, k=k, nq=nq, ng=ng, geom=geom, eps=eps, problem=problem, bc=bc, theta=theta)
    g = vemgpu.DarcyGpu(mesh, k=k, nq=nq, ng=ng, geometry=GEO[geom], eps=eps, problem=PROB[problem], bc=BCN[bc],
                        theta=theta)
    assert (g.nc, g.ne, g.nf, g.np, g.N) == (o.nc, o.ne, o.nf, o.np, o.N)
    return o, g


@pytest.fixture(scope="module")
def disk200():
    return meshgen.voronoi_mesh(200, "disk", seed=3)


@pytest.fixture(scope="module")
def annulus300():
    return meshgen.voronoi_mesh(300, "annulus", seed=4)


def _close(a, b, rtol):
    scale = max(np.abs(b).max(), 1e-300)
    assert np.abs(a - b).max() <= rtol * scale, (np.abs(a - b).max() / scale)


LOCAL_CASES = [
    ("square_2x2", 0, 9, O.GEOM_SINE, 0.05, O.BC_FLUX),
    ("square_2x2", 1, 9, O.GEOM_SINE, 0.05, O.BC_FLUX),
    ("square_2x2", 2, 9, O.GEOM_SINE, 0.05, O.BC_FLUX),
    ("square_1x1", 3, 12, O.GEOM_SINE, 0.05, O.BC_FLUX),
    ("square_1x1", 4, 36, O.GEOM_IDENTITY, 0.0, O.BC_FLUX),
]


@pytest.mark.parametrize("name,k,nq,geom,eps,bc", LOCAL_CASES)
def test_local_operators_square(square_meshes, name, k, nq, geom, eps, bc):
    o, g = pair(square_meshes[name], k, nq, geom, eps, O.PROB_SINCOS, bc)
    for c in range(o.nc):
        n = len(o.local(c, "dir"))
        _close(g.local(c, "A"), o.local(c, "A"), 1e-12)
        _close(g.local(c, "P"), o.local(c, "P"), 1e-11)
        _close(g.local(c, "W"), o.local(c, "W") if k else np.ones(n), 1e-13)
        _close(g.local(c, "alpha"), o.local(c, "alpha"), 1e-13)
    # lifted right-hand side of MixedGpu::make_rhs: free rows b - K g, boundary rows g
    K, b = o.system()
    mask, gv = o.boundary()
    ref = b - K @ gv
    ref[mask] = gv[mask]
    _close(g.rhs().cpu().numpy(), ref, 1e-12)


@pytest.mark.parametrize("k", [0, 1])
def test_local_operators_arcs(disk200, k):
    th = np.random.default_rng(5).normal(0, 1, 200)
    o, g = pair(disk200, k, 9, O.GEOM_ARCS, 0.0, O.PROB_SINSIN, O.BC_PRESSURE, theta=th)
    for c in range(0, o.nc, 7):
        _close(g.local(c, "A"), o.local(c, "A"), 1e-12)
        _close(g.local(c, "rhs"), o.local(c, "rhs"), 1e-12)
        _close(g.local(c, "dload"), o.local(c, "dload"), 1e-12)


def _apply_case(o, g, constrained):
    K, _ = o.system()
    rng = np.random.default_rng(11)
    x = rng.standard_normal(o.N)
    y = g.apply(torch.from_numpy(x).cuda(), constrained=constrained).cpu().numpy()
    if constrained and o.bc == O.BC_FLUX:
        mask, _ = o.boundary()
        xq = np.where(mask, 0.0, x)
        ref = K @ xq
        ref[mask] = x[mask]
    else:
        ref = K @ x
    return x, y, ref


@pytest.mark.parametrize("name,k", [("square_4x4", 0), ("square_4x4", 1), ("square_2x2", 2)])
@pytest.mark.parametrize("constrained", [False, True])
def test_apply_matches_oracle_csr(square_meshes, name, k, constrained):
    o, g = pair(square_meshes[name], k, 9, O.GEOM_SINE, 0.05, O.PROB_SINCOS, O.BC_FLUX)
    x, y, ref = _apply_case(o, g, constrained)
    _close(y, ref, 1e-12)
    y32 = g.apply(torch.from_numpy(x).float().cuda(), constrained=constrained).double().cpu().numpy()
    _close(y32, ref, 2e-6)


@pytest.mark.parametrize("k", [0, 1])
def test_apply_arcs_pressure_bc(disk200, k):
    o, g = pair(disk200, k, 9, O.GEOM_ARCS, 0.0, O.PROB_SINSIN, O.BC_PRESSURE)
    x, y, ref = _apply_case(o, g, True)
    _close(y, ref, 1e-12)
    _, b = o.system()
    _close(g.rhs().cpu().numpy(), b, 1e-12)


def _polar_mesh(rings=3, sectors=16, r0=0.2):
    """A 16-gon centre cell inside rings of quadrilaterals: its operator record exceeds a
    shared-memory stage, so the apply reads it from the strided arrays."""
    r = np.linspace(r0, 1.0, rings + 1)
    t = 2 * np.pi * np.arange(sectors) / sectors
    xy = np.concatenate([np.stack([ri * np.cos(t), ri * np.sin(t)], 1) for ri in r])
    cells = [list(range(sectors))]
    for i in range(rings):
        for j in range(sectors):
            a, b = i * sectors + j, i * sectors + (j + 1) % sectors
            cells.append([a, b, b + sectors, a + sectors])
    ptr = np.cumsum([0] + [len(c) for c in cells])
    return dict(xy=xy, cell_ptr=ptr, cell_nodes=np.concatenate(cells))


@pytest.mark.parametrize("k", [0, 1])
@pytest.mark.parametrize("constrained", [False, True])
def test_apply_large_polygon_record(k, constrained):
    o, g = pair(_polar_mesh(), k, 9, O.GEOM_IDENTITY, 0.0, O.PROB_SINCOS, O.BC_FLUX)
    x, y, ref = _apply_case(o, g, constrained)
    _close(y, ref, 1e-12)
    y32 = g.apply(torch.from_numpy(x).float().cuda(), constrained=constrained).double().cpu().numpy()
    _close(y32, ref, 2e-6)


@pytest.mark.parametrize("k", [0, 1])
def test_apply_many_ctas_matches_oracle(k):
    """Enough pieces for every CTA of the streamed apply to own several stages."""
    m = meshgen.voronoi_mesh(20000 if k == 0 else 8000, "annulus", seed=21)
    th = np.random.default_rng(22).normal(0, 1.5, len(m["cell_ptr"]) - 1)
    o, g = pair(m, k, 9, O.GEOM_ARCS, 0.0, O.PROB_ANNULUS, O.BC_PRESSURE, theta=th)
    x, y, ref = _apply_case(o, g, True)
    _close(y, ref, 1e-12)
    y32 = g.apply(torch.from_numpy(x).float().cuda()).double().cpu().numpy()
    _close(y32, ref, 2e-6)


def test_apply_is_deterministic(disk200):
    _, g = pair(disk200, 0, 9, O.GEOM_ARCS, 0.0, O.PROB_SINSIN, O.BC_PRESSURE)
    x = torch.randn(g.N, dtype=torch.float64, device="cuda")
    a = g.apply(x)
    for _ in range(3):
        assert torch.equal(a, g.apply(x))


def test_golden_reports_on_gpu(golden, square_meshes):
    for r in golden["reports"]:
        s = vemgpu.DarcySolver(square_meshes[r["mesh"]], problem=r["example"], gauss_point_num=r["nq"],
                               gauss_point_num_1d=9, k=r["k"])
        assert s.getTotalDofFlux() + s.getTotalDofConc() + 1 == r["dofs"]
        s.solve(tol=1e-12)
        e = s._errors()
        tol = 1e-7 if r["k"] == 4 else 2e-9
        for key in ("scalar_comp", "flux_comp", "scalar_phys", "flux_phys", "div_phys"):
            assert e[key] == pytest.approx(r["values"][key], rel=tol), (r["source"], key)
        assert abs(e["mass"] - r["values"]["mass"]) < 1e-8


@pytest.mark.parametrize("name,k", [("square_8x8", 1), ("square_4x4", 2), ("square_8x8", 0)])
def test_solution_matches_oracle_flux_bc(square_meshes, name, k):
    o, g = pair(square_meshes[name], k, 9, O.GEOM_SINE, 0.05, O.PROB_SINCOS, O.BC_FLUX)
    xo, _, _ = o.solve_direct()
    x, info = g.solve(tol=1e-12)  # essential flux BC with the multiplier: solved to 1e-12
    assert info["residual"] <= 1e-12
    xg = x.cpu().numpy()
    assert np.linalg.norm(xg - xo) <= 1e-10 * np.linalg.norm(xo)
    eo, eg = o.errors(xo), g.errors(x)
    for key in eo:
        assert eg[key] == pytest.approx(eo[key], rel=1e-8, abs=1e-12), key


@pytest.mark.parametrize("k", [0, 1])
@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_solution_matches_oracle_disk(k, mode):
    """Config C1's disk (1000 Voronoi cells, exact arcs, p = sin(pi x) sin(pi y), Dirichlet
    pressure): a solve to the reference's true-residual tolerance 1e-10 is within 1e-10 of the
    oracle's sparse-LU solution, FP64 and FP32-refined."""
    m = meshgen.voronoi_mesh(1000, "disk", seed=2)
    o, g = pair(m, k, 9, O.GEOM_ARCS, 0.0, O.PROB_SINSIN, O.BC_PRESSURE)
    xo, _, _ = o.solve_direct()
    x, info = g.solve(tol=1e-10, mode=mode)
    assert info["residual"] <= 1e-10
    xg = x.cpu().numpy()
    assert np.linalg.norm(xg - xo) <= 1e-10 * np.linalg.norm(xo)
    # the error kernel reproduces the oracle's figures on the same vector
    eo, eg = o.errors(xg), g.errors(x)
    for key in eo:
        assert eg[key] == pytest.approx(eo[key], rel=1e-11, abs=1e-14), key


def test_mixed_precision_refinement(annulus300):
    th = np.random.default_rng(7).normal(0, 2, 300)
    o, g = pair(annulus300, 0, 9, O.GEOM_ARCS, 0.0, O.PROB_ANNULUS, O.BC_PRESSURE, theta=th)
    x64, i64 = g.solve(tol=1e-10, mode="fp64")
    xm, im = g.solve(tol=1e-10, mode="mixed")
    assert i64["residual"] <= 1e-10 and im["residual"] <= 1e-10
    xo, _, _ = o.solve_direct()
    for x in (x64, xm):
        assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-10 * np.linalg.norm(xo)


def test_solve_host_matches_device(annulus300):
    _, g = pair(annulus300, 0, 9, O.GEOM_ARCS, 0.0, O.PROB_ANNULUS, O.BC_PRESSURE)
    b = g.rhs()
    xd, _ = g.solve(b)
    xh, info = g.solve_host(b.cpu().numpy())
    assert info["residual"] <= 1e-10
    assert np.array_equal(xd.cpu().numpy(), xh)


@pytest.mark.parametrize("field", ["lognormal", "iid"])
def test_multigrid_solve_matches_oracle_30k(field):
    """k = 0 with the pressure condition at 30,000 cells of the workload's annulus: a multigrid
    hierarchy of several levels (30k -> ~3.3k -> dense coarsest) preconditions the pressure block.
    The lognormal field is the workload's (Gaussian random field, exponential covariance, sigma 2,
    correlation length 0.1); solves to the true-residual tolerance 1e-10 are within 1e-10 of the
    oracle's sparse-LU solution, FP64 and FP32-refined."""
    from vemgpu import fields
    m = meshgen.voronoi_mesh(30000, "annulus", seed=61)
    if field == "lognormal":
        th = fields.gaussian_field(fields.cell_centroids(m), sigma=2.0, corr=0.1, seed=5)
    else:
        th = np.random.default_rng(62).normal(0, 1.5, 30000)
    o, g = pair(m, 0, 9, O.GEOM_ARCS, 0.0, O.PROB_ANNULUS, O.BC_PRESSURE, theta=th)
    xo, _, _ = o.solve_direct()
    for mode in ("fp64", "mixed"):
        x, info = g.solve(tol=1e-10, mode=mode)
        assert info["residual"] <= 1e-10
        assert info["iterations"] < 200, info
        assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-10 * np.linalg.norm(xo)


def test_multigrid_k1_solve_matches_oracle_20k():
    """k = 1 with the pressure condition at 20,000 cells: the pressure block (three moments per
    cell) is preconditioned by Jacobi smoothing, injection of the cell means and smoothed
    aggregation on the mean block."""
    m = meshgen.voronoi_mesh(20000, "disk", seed=63)
    o, g = pair(m, 1, 9, O.GEOM_ARCS, 0.0, O.PROB_SINSIN, O.BC_PRESSURE)
    xo, _, _ = o.solve_direct()
    for mode in ("fp64", "mixed"):
        x, info = g.solve(tol=1e-12, mode=mode)  # solved to 1e-12
        assert info["residual"] <= 1e-12
        assert info["iterations"] < 700, info
        assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-10 * np.linalg.norm(xo)


def test_vtk_file_handle_matches_dict_handle(tmp_path, disk200):
    """vg_create_vtk (C++ reader of the legacy VTK polygon file) builds the same operator as the
    raw-polygon entry point."""
    from vemgpu import meshio
    p = tmp_path / "disk.vtk"
    meshio.write_vtk(p, disk200)
    a = vemgpu.DarcyGpu(str(p), k=1, geometry="arcs", problem="sinsin", bc="pressure")
    b = vemgpu.DarcyGpu(disk200, k=1, geometry="arcs", problem="sinsin", bc="pressure")
    assert (a.nc, a.ne, a.N) == (b.nc, b.ne, b.N)
    x = torch.randn(a.N, dtype=torch.float64, device="cuda")
    assert torch.equal(a.apply(x), b.apply(x))
    assert torch.equal(a.rhs(), b.rhs())


@pytest.mark.parametrize("name,k,bc", [("square_4x4", 0, O.BC_FLUX), ("square_4x4", 1, O.BC_FLUX),
                                       ("square_2x2", 2, O.BC_FLUX)])
@pytest.mark.parametrize("constrained", [False, True])
def test_assembled_csr_matches_oracle_and_apply(square_meshes, name, k, bc, constrained):
    """vg_assemble_csr (the reference's assembled path) holds the oracle's matrix, and its product
    equals the matrix-free apply."""
    o, g = pair(square_meshes[name], k, 9, O.GEOM_SINE, 0.05, O.PROB_SINCOS, bc)
    C = g.assemble_csr(constrained=constrained)
    K, _ = o.system()
    D = C.to_dense().cpu().numpy()
    if constrained:
        mask, _ = o.boundary()
        ref = K.toarray()
        ref[mask, :] = 0
        ref[:, mask] = 0
        ref[mask, mask] = 1
    else:
        ref = K.toarray()
    _close(D, ref, 1e-12)
    x = torch.randn(g.N, dtype=torch.float64, device="cuda")
    _close((C @ x).cpu().numpy(), g.apply(x, constrained=constrained).cpu().numpy(), 1e-12)


def test_assembled_csr_arcs_pressure_bc(disk200):
    o, g = pair(disk200, 1, 9, O.GEOM_ARCS, 0.0, O.PROB_SINSIN, O.BC_PRESSURE)
    C = g.assemble_csr()
    K, _ = o.system()
    _close(C.to_dense().cpu().numpy(), K.toarray(), 1e-12)


def test_internal_order_apply_and_permute(disk200):
    """vg_permute and vg_apply with VG_ORDER_INTERNAL: the solver's internal numbering gives the
    same operator (bitwise, after the permutations)."""
    _, g = pair(disk200, 1, 9, O.GEOM_ARCS, 0.0, O.PROB_SINSIN, O.BC_PRESSURE)
    x = torch.randn(g.N, dtype=torch.float64, device="cuda")
    xi = g.permute(x)
    assert not torch.equal(xi, x)
    assert torch.equal(g.permute(xi, to_internal=False), x)
    y = g.apply(x)
    yi = g.apply(xi, internal_order=True)
    assert torch.equal(g.permute(yi, to_internal=False), y)


@pytest.mark.parametrize("k", [2, 3])
def test_multigrid_high_order_pressure_bc(k):
    """k >= 2 with the pressure condition: the pressure block's multigrid starts from the
    q-moment Schur block (injection of the cell means)."""
    m = meshgen.voronoi_mesh(1500, "disk", seed=64 + k)
    o, g = pair(m, k, default_nq(k), O.GEOM_ARCS, 0.0, O.PROB_SINSIN, O.BC_PRESSURE)
    xo, _, _ = o.solve_direct()
    x, info = g.solve(tol=1e-12)  # solved to 1e-12
    assert info["residual"] <= 1e-12
    assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-10 * np.linalg.norm(xo)


def test_calls_run_on_the_handles_device():
    """Every call runs on the device the handle was created on and leaves the caller's current
    device as it was (with one GPU both are device 0)."""
    import ctypes
    from vemgpu import _lib as L
    other = 1 if torch.cuda.device_count() > 1 else 0
    torch.cuda.set_device(other)
    try:
        m = meshgen.voronoi_mesh(1000, "disk", seed=2)
        g = vemgpu.DarcyGpu(m, k=0, geometry="arcs", problem="sinsin", bc="pressure", device=0)
        assert torch.cuda.current_device() == other
        b = torch.zeros(g.N, dtype=torch.float64, device="cuda:0")
        x = torch.zeros_like(b)
        L.check(L.lib().vg_rhs(g.h, b.data_ptr()), g.h)
        assert torch.cuda.current_device() == other
        o = g.opts(tol=1e-10)
        info = L.VgSolveInfo()
        L.check(L.lib().vg_solve(g.h, b.data_ptr(), x.data_ptr(), ctypes.byref(o), ctypes.byref(info)), g.h)
        assert torch.cuda.current_device() == other
        assert info.residual <= 1e-10
        g.close()
        assert torch.cuda.current_device() == other
    finally:
        torch.cuda.set_device(0)


@pytest.mark.parametrize("k,order", [(0, 1.0), (1, 2.0)])
def test_disk_convergence_orders(k, order):
    """Manufactured solution p = sin(pi x) sin(pi y) on the curved disk (exact arcs, Dirichlet
    pressure), four Voronoi meshes with h halving: the physical pressure and flux L2 errors fall as
    h^(k+1) (the reference pins its square meshes the same way,
    vem/CurvedVEM_Darcy/results_darcy_convergence_k1.txt:7-13). Slopes within 0.25 of k + 1."""
    hs, ep, eu = [], [], []
    for n in (500, 2000, 8000, 32000):
        m = meshgen.voronoi_mesh(n, "disk", seed=81)
        g = vemgpu.DarcyGpu(m, k=k, geometry="arcs", problem="sinsin", bc="pressure")
        x, info = g.solve(tol=1e-12)
        assert info["residual"] <= 1e-12
        e = g.errors(x)
        hs.append(np.sqrt(np.pi / n))
        ep.append(e["scalar_phys"])
        eu.append(e["flux_phys"])
        g.close()
    lh = np.log(hs)
    for err in (ep, eu):
        slope = np.polyfit(lh, np.log(err), 1)[0]
        assert abs(slope - order) <= 0.25, (slope, err)
