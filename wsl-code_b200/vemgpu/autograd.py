"""torch.autograd.Function over the forward solve and the hand-written adjoint.

``darcy_solve(handle, theta, **solve_options) -> x`` solves K(theta) x = b on the device (theta =
log permeability per cell, K_E = exp(theta_E) I); its backward pass solves the adjoint system with
the same Krylov method and contracts the adjoint with the forward solution cell by cell
(vg_adjoint_grad): dJ/dtheta_E = lambda_E^T A_E(theta) x_E. The right-hand side does not depend on
theta (pressure boundary data and sources; for the essential flux condition the lift b - A g is
recomputed by the library and the masked rows carry no sensitivity).
"""
import torch


class _DarcySolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, handle, opts):
        th = theta.detach().contiguous().double()
        handle.set_log_permeability(th)
        handle._theta_version = getattr(handle, "_theta_version", 0) + 1
        x, info = handle.solve(**opts)
        ctx.handle, ctx.opts, ctx.version = handle, opts, handle._theta_version
        ctx.forward_info = info
        ctx.save_for_backward(th, x)
        return x

    @staticmethod
    def backward(ctx, gx):
        th, x = ctx.saved_tensors
        h = ctx.handle
        if getattr(h, "_theta_version", 0) != ctx.version:  # operator changed since the forward solve
            h.set_log_permeability(th)
            h._theta_version += 1
        g, _ = h.adjoint_grad(x, gx.contiguous().double(), **ctx.opts)
        return g, None, None


def darcy_solve(handle, theta, **opts):
    """x(theta) with gradient support; opts are DarcyGpu.solve options (mode, tol, ...)."""
    return _DarcySolve.apply(theta, handle, opts)
