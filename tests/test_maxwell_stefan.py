"""Ternary Maxwell-Stefan (k = 0, reduced two-species form, backward Euler, no-flux boundary)
through the C ABI, against a CPU FP64 system assembled from the oracle's local operators
(K = I A_E, orientation signs, cell measures) and solved by sparse LU. Tolerances in each test."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from vemgpu import meshgen  # noqa: E402
from vemgpu.maxwell_stefan import MaxwellStefan, initial_fractions  # noqa: E402

D = (1.0, 0.5, 0.2)
DT = 1e-3


def friction(x1, x2):
    i12, i13, i23 = 1 / D[0], 1 / D[1], 1 / D[2]
    x3 = 1 - x1 - x2
    return np.stack([np.stack([x1 * i13 + x2 * i12 + x3 * i13, -x1 * (i12 - i13)], -1),
                     np.stack([-x2 * (i12 - i23), x2 * i23 + x1 * i12 + x3 * i23], -1)], -2)


def cpu_system(o, x1, x2):
    nf, nc = o.nf, o.nc
    N = 2 * nf + 2 * nc
    mask = o.boundary()[0][:nf]
    B = friction(x1, x2)
    R, C, V = [], [], []
    for c in range(nc):
        d = o.local(c, "dir")
        n = len(d)
        gd = o.local(c, "gdofs")[:n].astype(np.int64)
        A = o.local(c, "A").reshape(n, n) * np.outer(d, d)
        area = o.local(c, "L")[0]
        free = ~mask[gd]
        for s in range(2):
            for t in range(2):
                for i in range(n):
                    for j in range(n):
                        if free[i] and free[j]:
                            R.append(s * nf + gd[i]); C.append(t * nf + gd[j]); V.append(B[c, s, t] * A[i, j])
            p = 2 * nf + s * nc + c
            for i in range(n):
                if free[i]:
                    R += [s * nf + gd[i], p]; C += [p, s * nf + gd[i]]; V += [-d[i], d[i]]
            R.append(p); C.append(p); V.append(area / DT)
    for s in range(2):
        for g in np.flatnonzero(mask):
            R.append(s * nf + g); C.append(s * nf + g); V.append(1.0)
    return sp.csr_matrix((V, (R, C)), shape=(N, N))


@pytest.fixture(scope="module")
def case():
    m = meshgen.voronoi_mesh(400, "disk", seed=71)
    o = O.Oracle(m, k=0, nq=9, ng=9, geom=O.GEOM_ARCS, problem=O.PROB_SINCOS, bc=O.BC_FLUX)
    ms = MaxwellStefan(m, D=D, dt=DT)
    x1, x2, x3 = initial_fractions(m, seed=72)
    return m, o, ms, x1, x2


def test_initial_fractions_in_range(case):
    m, _, _, x1, x2 = case
    x3 = 1 - x1 - x2
    for x in (x1, x2, x3):
        assert x.min() >= 0.1 - 1e-12 and x.max() <= 0.8 + 1e-12


def test_operator_matches_cpu_system(case):
    _, o, ms, x1, x2 = case
    K = cpu_system(o, x1, x2)
    s = ms.state(x1, x2)
    x = torch.randn(ms.N, dtype=torch.float64, device="cuda")
    y = ms.apply(s, x).cpu().numpy()
    ref = K @ x.cpu().numpy()
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()
    y32 = ms.apply(s, x.float()).double().cpu().numpy()
    assert np.abs(y32 - ref).max() <= 2e-6 * np.abs(ref).max()


def test_step_matches_direct_solve(case):
    _, o, ms, x1, x2 = case
    s = ms.state(x1, x2)
    K = cpu_system(o, x1, x2)
    areas = np.array([o.local(c, "L")[0] for c in range(o.nc)])
    b = np.zeros(ms.N)
    b[2 * o.nf:] = np.r_[areas * x1, areas * x2] / DT
    ref = spla.spsolve(K.tocsc(), b)
    for mode, rtol in (("fp64", 1e-9), ("mixed", 1e-9)):
        gs0 = ms.gram_schmidt_info()
        new, info = ms.step(s, mode=mode, tol=1e-11)
        assert info["residual"] <= 1e-11
        got = new.cpu().numpy()
        assert np.linalg.norm(got - ref) <= rtol * np.linalg.norm(ref), mode
        # every Arnoldi step is counted; the second Gram-Schmidt pass runs in at most all of them
        gs1 = ms.gram_schmidt_info()
        steps = gs1["arnoldi_steps"] - gs0["arnoldi_steps"]
        reo = gs1["reorthogonalizations"] - gs0["reorthogonalizations"]
        assert steps == info["iterations"] and 0 <= reo <= steps, (mode, steps, reo)


def test_steps_conserve_mass_and_sum(case):
    _, o, ms, x1, x2 = case
    s64 = ms.state(x1, x2)
    s32 = s64.clone()
    m0 = ms.masses(s64)
    for _ in range(5):
        s64, i64 = ms.step(s64, mode="fp64", tol=1e-10)
        s32, i32 = ms.step(s32, mode="mixed", tol=1e-10)
        for s in (s64, s32):
            f = ms.fractions(s)
            assert torch.all(f[0] > 0) and torch.all(f[1] > 0) and torch.all(f[2] > 0)
            assert float(torch.abs(f[0] + f[1] + f[2] - 1).max()) <= 1e-14
            for a, b in zip(ms.masses(s), m0):
                assert abs(a - b) <= 1e-9 * abs(b)
    x64 = torch.cat(ms.fractions(s64)[:2])
    x32 = torch.cat(ms.fractions(s32)[:2])
    assert float(torch.linalg.norm(x64 - x32) / torch.linalg.norm(x64)) <= 1e-9


def test_picard_step_matches_cpu_picard(case):
    """Fully implicit step: Picard iterations on the friction matrix (the reference's time loop,
    vem/CurvedVEM_Darcy_gpu/src/solver_driver.cpp:209-240) against the same iteration on the CPU
    system, each linear system by sparse LU; relative 1e-9 between the two fixed points."""
    m, o, _, x1, x2 = case
    ms = MaxwellStefan(m, D=D, dt=DT, picard=20, picard_tol=1e-11)
    s = ms.state(x1, x2)
    areas = np.array([o.local(c, "L")[0] for c in range(o.nc)])
    b = np.zeros(ms.N)
    b[2 * o.nf:] = np.r_[areas * x1, areas * x2] / DT
    xk = s.cpu().numpy()
    for it in range(20):
        nxt = xk[2 * o.nf:]
        xn = spla.spsolve(cpu_system(o, nxt[:o.nc], nxt[o.nc:]).tocsc(), b)
        change = np.linalg.norm(xn - xk) / max(1.0, np.linalg.norm(xn))
        xk = xn
        if change <= 1e-13:
            break
    for mode in ("fp64", "mixed"):
        new, info = ms.step(s, mode=mode, tol=1e-12)
        assert info["picard"] >= 2 and info["picard_change"] <= 1e-11 and info["nonlinear_residual"] <= 1e-11
        got = new.cpu().numpy()
        assert np.linalg.norm(got - xk) <= 1e-9 * np.linalg.norm(xk), mode
        # the fully implicit step differs from the linearly implicit one
        ms.set_picard(1)
        lin, info1 = ms.step(s, mode=mode, tol=1e-12)
        assert info1["picard"] == 1
        assert np.linalg.norm(lin.cpu().numpy() - xk) > 1e-9 * np.linalg.norm(xk)
        ms.set_picard(20, 1e-11)
    ms.close()
