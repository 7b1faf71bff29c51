"""Adjoint gradient dJ/dtheta of point observations of the pressure (log permeability theta per
cell), through the torch.autograd.Function over vg_solve / vg_adjoint_grad.

Checks, with the tolerance of each written in the test:
* against the CPU FP64 adjoint of the oracle (sparse LU on the assembled system, the per-cell
  contraction lambda_E^T A_E u_E with the oracle's own dof map and signs): relative 1e-8;
* against central finite differences (step 1e-6, 20 seeded unit directions) of J computed by the
  GPU solver at tolerance 1e-12: relative 1e-6 of the largest directional derivative;
* against the same central differences with the numerator formed from the solution corrections
  (no cancellation between two values of J): 1e-9 of the largest directional derivative;
* against central finite differences (step 1e-6) of J computed by the oracle's direct solver (no
  Krylov error): 1e-6 of the gradient norm.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import vemgpu  # noqa: E402
from vemgpu import fields, meshgen, observe  # noqa: E402
from vemgpu.autograd import darcy_solve  # noqa: E402

GEO = {O.GEOM_IDENTITY: "identity", O.GEOM_SINE: "sine", O.GEOM_ARCS: "arcs"}


@pytest.fixture(scope="module")
def annulus2k():
    m = meshgen.voronoi_mesh(2000, "annulus", seed=31)
    th = fields.gaussian_field(fields.cell_centroids(m), sigma=1.0, corr=0.2, seed=32)
    pts = observe.seeded_points(16, 33)
    return m, th, pts


def _oracle_J_and_grad(m, th, k, cells, data, problem=O.PROB_ANNULUS, bc=O.BC_PRESSURE, geom=O.GEOM_ARCS,
                       eps=0.0):
    o = O.Oracle(m, k=k, nq=9, ng=9, geom=geom, eps=eps, problem=problem, bc=bc, theta=th)
    K, b = o.system()
    if bc == O.BC_FLUX:
        # essential flux rows: K_c = Q K Q + (I - Q), b_c = Q (b - K g) + g (MixedGpu::make_rhs lift)
        import scipy.sparse as sp
        msk, gv = o.boundary()
        Q = sp.diags((~msk).astype(float))
        K = (Q @ K @ Q + sp.diags(msk.astype(float))).tocsr()
        b = np.where(msk, gv, b - o.system()[0] @ gv)
    lu = spla.splu(K.tocsc())
    x = lu.solve(b)
    q = (k + 1) * (k + 2) // 2
    idx = o.nf + cells * q
    r = x[idx] - data
    J = float(r @ r)
    dJdx = np.zeros(o.N)
    np.add.at(dJdx, idx, 2 * r)
    lam = lu.solve(dJdx, trans="T")
    g = np.zeros(o.nc)
    mask = o.boundary()[0] if bc == O.BC_FLUX else np.zeros(o.N, bool)
    for c in range(o.nc):
        d = o.local(c, "dir")
        n = len(d)
        gd = o.local(c, "gdofs")[:n].astype(np.int64)
        A = o.local(c, "A").reshape(n, n)
        u = d * x[gd]
        w = np.where(mask[gd], 0.0, d * lam[gd])
        g[c] = w @ A @ u
    return J, g, x


def _gpu_J(h, obs, theta, tol):
    x = darcy_solve(h, theta, tol=tol)
    return obs(x)


def test_gradient_matches_cpu_adjoint(annulus2k):
    m, th, pts = annulus2k
    h = vemgpu.DarcyGpu(m, k=0, geometry="arcs", problem="annulus", bc="pressure", theta=th)
    obs = observe.PointObservation(h, m, pts, data=np.linspace(0.2, 0.8, len(pts)))
    theta = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
    J = _gpu_J(h, obs, theta, 1e-12)
    J.backward()
    Jc, gc, _ = _oracle_J_and_grad(m, th, 0, obs.cells, obs.data.cpu().numpy())
    assert float(J.detach()) == pytest.approx(Jc, rel=1e-9)
    g = theta.grad.cpu().numpy()
    assert np.abs(g - gc).max() <= 1e-8 * np.abs(gc).max()
    h.close()


def test_gradient_matches_central_differences(annulus2k):
    m, th, pts = annulus2k
    h = vemgpu.DarcyGpu(m, k=0, geometry="arcs", problem="annulus", bc="pressure", theta=th)
    obs = observe.PointObservation(h, m, pts, data=np.linspace(0.2, 0.8, len(pts)))
    theta = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
    J = _gpu_J(h, obs, theta, 1e-12)
    J.backward()
    g = theta.grad.clone()
    rng = np.random.default_rng(34)
    step = 1e-6
    ad, fd = [], []
    with torch.no_grad():
        for _ in range(20):
            v = rng.standard_normal(len(th))
            v /= np.linalg.norm(v)
            vt = torch.tensor(v, dtype=torch.float64, device="cuda")
            jp = float(_gpu_J(h, obs, theta + step * vt, 1e-12))
            jm = float(_gpu_J(h, obs, theta - step * vt, 1e-12))
            fd.append((jp - jm) / (2 * step))
            ad.append(float(g @ vt))
    ad, fd = np.array(ad), np.array(fd)
    assert np.abs(ad - fd).max() <= 1e-6 * np.abs(ad).max(), (ad, fd)
    h.close()


def test_gradient_matches_cancellation_free_differences(annulus2k):
    """Central differences (step 1e-6) whose numerator J(+) - J(-) = sum_o (p+ - p-)(p+ + p- - 2 d_o)
    is formed from the corrections e = x(theta +- step v) - x0, each solved for directly:
    K(theta') e = (b - K(theta) x0) - (K(theta') - K(theta)) x0, the last term from the per-cell
    scaling of the flux block (an apply of the flux part u0 at theta - log(s + m) less m times its
    apply at theta, s = expm1(-+step v), m a power of two). Free of the rounding of two values of J,
    so the bound is 1e-9 of the largest directional derivative (1e-6 for plain differences)."""
    m, th, pts = annulus2k
    h = vemgpu.DarcyGpu(m, k=0, geometry="arcs", problem="annulus", bc="pressure", theta=th)
    obs = observe.PointObservation(h, m, pts, data=np.linspace(0.2, 0.8, len(pts)))
    x0 = h.zeros()
    try:
        h.solve(x=x0, mode="fp64", tol=1e-13)
    except vemgpu.VemGpuError:
        pass  # the FP64 floor was reached first: x0 is the last iterate (checked below)
    dJdx = torch.autograd.functional.vjp(obs, x0)[1]
    g, _ = h.adjoint_grad(x0, dJdx, mode="fp64", tol=1e-12)
    base = torch.tensor(th, dtype=torch.float64, device="cuda")
    b0 = h.rhs()
    r0 = b0 - h.apply(x0)
    assert float(torch.linalg.norm(r0) / torch.linalg.norm(b0)) <= 1e-12
    u0 = x0.clone()
    u0[h.nf:] = 0
    y0 = h.apply(u0)
    res = obs.pressure(x0) - obs.data

    def correction(v, sigma):
        s = torch.expm1(-sigma * 1e-6 * v)
        mm = 2.0 ** np.ceil(np.log2(2 * float(s.abs().max())))
        h.set_log_permeability(base - torch.log(s + mm))
        ya = h.apply(u0)
        r = r0.clone()
        r[:h.nf] -= ya[:h.nf] - mm * y0[:h.nf]
        h.set_log_permeability(base + sigma * 1e-6 * v)
        e = h.zeros()
        try:
            h.solve(b=r, x=e, mode="fp64", tol=1e-12)
        except vemgpu.VemGpuError:
            pass  # the FP64 floor was reached first: e is the last iterate
        return obs.pressure(e)

    rng = np.random.default_rng(35)
    ad, fd = [], []
    for _ in range(10):
        v = torch.tensor(rng.standard_normal(len(th)), device="cuda")
        v /= torch.linalg.norm(v)
        dp, dm = correction(v, 1.0), correction(v, -1.0)
        fd.append(float(((dp - dm) * (2 * res + dp + dm)).sum()) / 2e-6)
        ad.append(float(g @ v))
    h.set_log_permeability(base)
    ad, fd = np.array(ad), np.array(fd)
    assert np.abs(ad - fd).max() <= 1e-9 * np.abs(ad).max(), (ad, fd)
    h.close()


def test_gradient_matches_oracle_differences_k1():
    m = meshgen.voronoi_mesh(400, "disk", seed=41)
    th = fields.gaussian_field(fields.cell_centroids(m), sigma=1.0, corr=0.3, seed=42)
    pts = observe.seeded_points(8, 43, r_in=0.0, r_out=0.9)
    cells = observe.locate_cells(m, pts)
    data = np.full(len(pts), 0.1)
    h = vemgpu.DarcyGpu(m, k=1, geometry="arcs", problem="sinsin", bc="pressure", theta=th)
    q = 3
    idx = torch.as_tensor(h.nf + cells * q, dtype=torch.long, device="cuda")  # mean-moment unknown
    theta = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
    x = darcy_solve(h, theta, tol=1e-12)
    J = ((x[idx] - torch.as_tensor(data, device="cuda")) ** 2).sum()
    J.backward()
    g = theta.grad.cpu().numpy()
    J0, gc, _ = _oracle_J_and_grad(m, th, 1, cells, data, problem=O.PROB_SINSIN)
    assert float(J.detach()) == pytest.approx(J0, rel=1e-9)
    assert np.abs(g - gc).max() <= 1e-8 * np.abs(gc).max()
    # oracle central differences (step 1e-6) along 3 unit directions (direct solves: no Krylov
    # tolerance in J); with J ~ 10 the rounding of J alone gives ~1e-8 absolute noise in the quotient,
    # so the bound is 1e-6 of the gradient norm (|g.v| <= |g| for a unit v)
    rng = np.random.default_rng(44)
    for _ in range(3):
        v = rng.standard_normal(len(th))
        v /= np.linalg.norm(v)
        jp = _oracle_J_and_grad(m, th + 1e-6 * v, 1, cells, data, problem=O.PROB_SINSIN)[0]
        jm = _oracle_J_and_grad(m, th - 1e-6 * v, 1, cells, data, problem=O.PROB_SINSIN)[0]
        assert abs((jp - jm) / 2e-6 - g @ v) <= 1e-6 * np.linalg.norm(g)
    h.close()


def test_gradient_flux_bc_matches_cpu_adjoint(square_meshes):
    m = square_meshes["square_4x4"]
    nc = len(m["cell_ptr"]) - 1
    th = np.random.default_rng(51).normal(0, 0.5, nc)
    h = vemgpu.DarcyGpu(m, k=1, geometry="sine", eps=0.05, problem="sincos", bc="flux", theta=th)
    cells = np.arange(0, nc, 5)
    data = np.zeros(len(cells))
    idx = torch.as_tensor(h.nf + cells * 3, dtype=torch.long, device="cuda")
    theta = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
    x = darcy_solve(h, theta, tol=1e-12)
    J = (x[idx] ** 2).sum()
    J.backward()
    J0, gc, xo = _oracle_J_and_grad(m, th, 1, cells, data, problem=O.PROB_SINCOS, bc=O.BC_FLUX,
                                    geom=O.GEOM_SINE, eps=0.05)
    assert np.linalg.norm(x.detach().cpu().numpy() - xo) <= 1e-9 * np.linalg.norm(xo)
    g = theta.grad.cpu().numpy()
    assert np.abs(g - gc).max() <= 1e-8 * np.abs(gc).max()
    h.close()


def test_theta_update_after_build_matches_fresh_handle(square_meshes):
    """vg_set_log_permeability after vg_build (operator rescale, preconditioner and the lifted
    essential-BC right-hand side) gives the same solution as a handle built with that theta."""
    m = square_meshes["square_4x4"]
    nc = len(m["cell_ptr"]) - 1
    th = np.random.default_rng(52).normal(0, 0.7, nc)
    a = vemgpu.DarcyGpu(m, k=1, geometry="sine", eps=0.05, problem="sincos", bc="flux")
    a.set_log_permeability(th)
    b = vemgpu.DarcyGpu(m, k=1, geometry="sine", eps=0.05, problem="sincos", bc="flux", theta=th)
    xa, _ = a.solve(tol=1e-12)
    xb, _ = b.solve(tol=1e-12)
    assert torch.allclose(a.rhs(), b.rhs(), rtol=1e-13, atol=1e-14)
    assert torch.linalg.norm(xa - xb) <= 1e-10 * torch.linalg.norm(xb)
    a.close()
    b.close()


def test_theta_update_rebuilds_multigrid(annulus2k):
    """k = 0 with the pressure condition: a permeability update after a graph-captured solve
    rebuilds the multigrid hierarchy (and the captured Krylov loop) before the next solve."""
    m, th, _ = annulus2k
    a = vemgpu.DarcyGpu(m, k=0, geometry="arcs", problem="annulus", bc="pressure")
    a.solve(tol=1e-10)
    for mode in ("fp64", "mixed"):
        a.solve(tol=1e-10, mode=mode)
    a.set_log_permeability(th)
    b = vemgpu.DarcyGpu(m, k=0, geometry="arcs", problem="annulus", bc="pressure", theta=th)
    for mode in ("fp64", "mixed"):
        xa, ia = a.solve(tol=1e-10, mode=mode)
        xb, ib = b.solve(tol=1e-10, mode=mode)
        assert ia["residual"] <= 1e-10 and ib["residual"] <= 1e-10
        assert ia["iterations"] == ib["iterations"]
        assert torch.linalg.norm(xa - xb) <= 1e-9 * torch.linalg.norm(xb)
    a.close()
    b.close()


@pytest.mark.parametrize("k,cells,domain", [(0, 30000, "annulus"), (1, 8000, "disk")])
def test_multigrid_refresh_on_permeability_update(k, cells, domain):
    """A permeability update recomputes the multigrid's values on the device (aggregates and
    patterns kept): the solve matches a handle built from scratch with the new permeability."""
    m = meshgen.voronoi_mesh(cells, domain, seed=81 + k)
    cen = fields.cell_centroids(m)
    th1 = fields.gaussian_field(cen, sigma=1.5, corr=0.1, seed=82)
    th2 = fields.gaussian_field(cen, sigma=1.5, corr=0.1, seed=83)
    geo = dict(geometry="arcs", problem="annulus" if domain == "annulus" else "sinsin", bc="pressure")
    a = vemgpu.DarcyGpu(m, k=k, theta=th1, **geo)
    x1, i1 = a.solve(tol=1e-10)
    a.set_log_permeability(th1)  # same values through the refresh path
    x1b, i1b = a.solve(tol=1e-10)
    assert abs(i1b["iterations"] - i1["iterations"]) <= 2
    assert torch.linalg.norm(x1b - x1) <= 1e-9 * torch.linalg.norm(x1)
    a.set_log_permeability(th2)
    b = vemgpu.DarcyGpu(m, k=k, theta=th2, **geo)
    for mode in ("fp64", "mixed"):
        xa, ia = a.solve(tol=1e-10, mode=mode)
        xb, ib = b.solve(tol=1e-10, mode=mode)
        assert ia["residual"] <= 1e-10
        assert ia["iterations"] <= 1.3 * ib["iterations"] + 5, (ia, ib)
        assert torch.linalg.norm(xa - xb) <= 1e-8 * torch.linalg.norm(xb)
    a.close()
    b.close()
