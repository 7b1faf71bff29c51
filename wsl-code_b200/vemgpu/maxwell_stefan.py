"""Ternary Maxwell-Stefan diffusion on the C ABI (vg_ms_configure / vg_ms_step, k = 0).

State: one device vector [J1, J2, x1, x2] (species fluxes on the flux moments, cell mole fractions),
x3 = 1 - x1 - x2. Each backward-Euler step solves the coupled two-species saddle-point system with
the friction matrix at the previous state (picard=1, linearly implicit) or, with picard > 1, Picard
iterations on the friction matrix until the step is fully implicit to picard_tol. The reference's
counterpart is its MSGpu time loop with Picard iterations
(vem/CurvedVEM_Darcy_gpu/src/solver_driver.cpp:189-245), which keeps all three species.
"""
import ctypes

import numpy as np

from . import _lib as L
from . import fields
from .core import DarcyGpu, _torch


def initial_fractions(mesh, seed, corr=0.2, lo=0.1, hi=0.8):
    """Seeded smooth random mole fractions: x_i = lo + (1 - 3 lo) w_i / sum w, w_i = exp(g_i) for three
    Gaussian fields g_i; each x_i lies in [lo, 1 - 2 lo] and x1 + x2 + x3 = 1 (lo = 0.1: [0.1, 0.8])."""
    if hi < 1 - 2 * lo - 1e-12:
        raise ValueError("with three fractions summing to 1 above lo, the upper bound is 1 - 2 lo")
    cen = fields.cell_centroids(mesh)
    g = np.stack([fields.gaussian_field(cen, sigma=1.0, corr=corr, seed=seed + i) for i in range(3)])
    w = np.exp(g - g.max(axis=0))
    x = lo + (1 - 3 * lo) * w / w.sum(axis=0)
    return x[0], x[1], x[2]


class MaxwellStefan:
    def __init__(self, mesh, D=(1.0, 0.5, 0.2), dt=1e-3, geometry="arcs", eps=0.0, device=-1, picard=1,
                 picard_tol=1e-10):
        self.gpu = DarcyGpu(mesh, k=0, geometry=geometry, eps=eps, problem="sincos", bc="flux", device=device)
        self.D, self.dt = tuple(D), dt
        n = ctypes.c_longlong(0)
        L.check(L.lib().vg_ms_configure(self.gpu.h, D[0], D[1], D[2], dt, ctypes.byref(n)), self.gpu.h)
        self.N = n.value
        self.nf, self.nc = self.gpu.nf, self.gpu.nc
        torch = _torch()
        self.areas = torch.empty(self.nc, dtype=torch.float64, device="cuda")
        L.check(L.lib().vg_cell_areas(self.gpu.h, self.areas.data_ptr()), self.gpu.h)
        self.set_picard(picard, picard_tol)

    def set_picard(self, max_iterations, tol=1e-10):
        L.check(L.lib().vg_ms_set_picard(self.gpu.h, int(max_iterations), float(tol)), self.gpu.h)

    def state(self, x1, x2):
        torch = _torch()
        s = torch.zeros(self.N, dtype=torch.float64, device="cuda")
        s[2 * self.nf:2 * self.nf + self.nc] = torch.as_tensor(np.asarray(x1), dtype=torch.float64)
        s[2 * self.nf + self.nc:] = torch.as_tensor(np.asarray(x2), dtype=torch.float64)
        return s

    def fractions(self, s):
        x1 = s[2 * self.nf:2 * self.nf + self.nc]
        x2 = s[2 * self.nf + self.nc:]
        return x1, x2, 1.0 - x1 - x2

    def masses(self, s):
        return [float((self.areas * x).sum()) for x in self.fractions(s)]

    def apply(self, coeff_state, x):
        torch = _torch()
        y = torch.empty_like(x)
        prec = L.FP64 if x.dtype == torch.float64 else L.FP32
        L.check(L.lib().vg_ms_apply(self.gpu.h, coeff_state.data_ptr(), x.data_ptr(), y.data_ptr(), prec), self.gpu.h)
        return y

    def step(self, s, out=None, **kw):
        torch = _torch()
        out = torch.empty_like(s) if out is None else out
        info = L.VgSolveInfo()
        o = DarcyGpu.opts(**kw)
        L.check(L.lib().vg_ms_step(self.gpu.h, s.data_ptr(), out.data_ptr(), ctypes.byref(o), ctypes.byref(info)),
                self.gpu.h)
        pic, change, nonlin = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        L.check(L.lib().vg_ms_picard_info(self.gpu.h, ctypes.byref(pic), ctypes.byref(change), ctypes.byref(nonlin)),
                self.gpu.h)
        return out, dict(iterations=info.iterations, outer=info.outer, residual=info.residual, seconds=info.seconds,
                         picard=pic.value, picard_change=change.value, nonlinear_residual=nonlin.value)

    def gram_schmidt_info(self):
        """Arnoldi steps of the handle's GMRES solves so far and how many ran the second
        Gram-Schmidt pass (selective reorthogonalisation)."""
        steps, reo = ctypes.c_longlong(), ctypes.c_longlong()
        L.check(L.lib().vg_ms_gs_info(self.gpu.h, ctypes.byref(steps), ctypes.byref(reo)), self.gpu.h)
        return dict(arnoldi_steps=steps.value, reorthogonalizations=reo.value)

    def close(self):
        self.gpu.close()
