"""vemgpu — B200-native matrix-free curved mixed-VEM Darcy solver (Python side of the C ABI).

* ``DarcyGpu``: one handle of the C ABI (mesh, geometry, degree, problem, boundary condition).
* ``DarcySolver``: the call sequence of the reference CPU class
  (vem/CurvedVEM_Darcy/solver/DarcySolver.h:17-126) on top of ``DarcyGpu``.
* ``meshgen``: seeded Voronoi + Lloyd disk / annulus meshes with exact circular-arc boundaries.
* ``fields``: seeded Gaussian random fields for log permeability.
* ``autograd``: ``torch.autograd.Function`` over the forward solve and the adjoint gradient.
* ``observe``: point observations of the pressure (the adjoint's objective).
"""
from ._lib import VemGpuError, header_functions, lib  # noqa: F401
from .core import DarcyGpu, DarcySolver, default_nq  # noqa: F401
