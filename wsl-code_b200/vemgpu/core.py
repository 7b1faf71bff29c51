"""Python handle over the vemgpu C ABI.

``DarcyGpu`` owns one ``vg_handle``: device setup (vg_build), the matrix-free operator
(vg_apply), right-hand side (vg_rhs), Krylov solve (vg_solve / vg_solve_host), adjoint gradient
(vg_adjoint_grad) and errors (vg_errors). Device vectors are torch CUDA tensors (plumbing only).

``DarcySolver`` mirrors the reference CPU class vem/CurvedVEM_Darcy/solver/DarcySolver.h:17-126:
``DarcySolver(mesh, problem, gauss_point_num=9, gauss_point_num_1d=9, k=1)``, ``solve()``,
``computeL2ErrorPressure()``, ``computeL2ErrorFlux()``, ``getSolution()``,
``getTotalDofFlux()``, ``getTotalDofConc()``.
"""
import ctypes

import numpy as np

from . import _lib as L


def default_nq(k):
    """Triangle rule chosen by the reference for degree k (vem/CurvedVEM_Darcy_gpu/src/solver_options.cpp:123-124)."""
    return 36 if k == 4 else 12 if k == 3 else 9


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("vemgpu needs a CUDA device")
    return torch


class DarcyGpu:
    """One solver handle. mesh: path of a legacy VTK polygon file (vemgpu.meshio), dict with raw
    polygons (xy, cell_ptr, cell_nodes) or the processed
    reader arrays (node_coords, cell_nodes, cell_node_indices, global_edges, edge_endpoints,
    edge_occurrence, cell_centroid_x, cell_centroid_y, cell_diameter); optional arc_nodes /
    arc_data for circular boundary arcs. geometry: 'identity', 'sine' (eps) or 'arcs'."""

    def __init__(self, mesh, k=1, nq=None, ng=9, geometry="identity", eps=0.0, problem="sincos", bc="flux",
                 theta=None, device=-1, build=True):
        self._keep = []
        lib = L.lib()
        vtk_path = None
        if isinstance(mesh, (str, bytes)) or hasattr(mesh, "__fspath__"):
            # legacy VTK polygon file, read by the C ABI (vg_create_vtk); arcs from its FIELD block
            import os
            from . import meshio
            vtk_path = os.fsencode(mesh)
            mesh = meshio.read_vtk_arcs(mesh)
        nq = default_nq(k) if nq is None else nq
        g = L.VgGeometry()
        g.kind = L.GEOM[geometry]
        g.eps = eps
        an, ad = mesh.get("arc_nodes"), mesh.get("arc_data")
        if an is not None and len(an):
            an = np.ascontiguousarray(an, np.int32).reshape(-1)
            ad = np.ascontiguousarray(ad, np.float64).reshape(-1)
            self._keep += [an, ad]
            g.num_arcs = len(an) // 2
            g.arc_nodes = an.ctypes.data
            g.arc_circles = ad.ctypes.data
        h = ctypes.c_void_p()
        if vtk_path is not None:
            code = lib.vg_create_vtk(vtk_path, ctypes.byref(g), k, nq, ng, device, ctypes.byref(h))
        elif "xy" in mesh:
            xy = np.ascontiguousarray(mesh["xy"], np.float64).reshape(-1)
            ptr = np.ascontiguousarray(mesh["cell_ptr"], np.int32)
            nodes = np.ascontiguousarray(mesh["cell_nodes"], np.int32)
            code = lib.vg_create_polygons(len(xy) // 2, xy.ctypes.data, len(ptr) - 1, ptr.ctypes.data,
                                          nodes.ctypes.data, ctypes.byref(g), k, nq, ng, device, ctypes.byref(h))
        else:
            arr = {key: np.ascontiguousarray(mesh[key], np.float64 if key in ("node_coords", "cell_centroid_x",
                                                                              "cell_centroid_y", "cell_diameter")
                                             else np.int32)
                   for key in ("node_coords", "cell_nodes", "cell_node_indices", "global_edges", "edge_endpoints",
                               "edge_occurrence", "cell_centroid_x", "cell_centroid_y", "cell_diameter")}
            self._keep.append(arr)
            m = L.VgMesh()
            m.num_nodes = len(arr["node_coords"]) // 2
            m.num_cells = len(arr["cell_node_indices"]) - 1
            m.num_edges = len(arr["edge_occurrence"])
            for key, a in arr.items():
                setattr(m, key, a.ctypes.data)
            m.nodes_per_cell = None
            m.cell_edge_indices = arr["cell_node_indices"].ctypes.data
            code = lib.vg_create(ctypes.byref(m), ctypes.byref(g), k, nq, ng, device, ctypes.byref(h))
        L.check(code, None)
        self.h = h
        self.k, self.nq, self.ng = k, nq, ng
        L.check(lib.vg_set_problem(self.h, L.PROBLEM[problem], L.BC[bc]), self.h)
        self.problem, self.bc = problem, bc
        if theta is not None:
            self.set_log_permeability(theta, rebuild=False)
        self._sizes()
        if build:
            self.build()

    def _sizes(self):
        s = (ctypes.c_longlong * 9)()
        L.check(L.lib().vg_sizes(self.h, s), self.h)
        (self.nc, self.ne, self.nf, self.np, self.N, self.q, self.p, self.internal, self.maxn) = [int(v) for v in s]

    def close(self):
        if getattr(self, "h", None):
            try:
                L.lib().vg_destroy(self.h)
            except Exception:
                pass
            self.h = None

    def __del__(self):
        self.close()

    def build(self):
        L.check(L.lib().vg_build(self.h), self.h)
        self._sizes()

    def set_log_permeability(self, theta, rebuild=True):
        """theta: numpy array (host) or torch CUDA tensor (device), one value per cell."""
        if hasattr(theta, "data_ptr") and getattr(theta, "is_cuda", False):
            t = theta.contiguous().double()
            L.check(L.lib().vg_set_log_permeability(self.h, t.data_ptr(), 1), self.h)
        else:
            t = np.ascontiguousarray(theta, np.float64)
            L.check(L.lib().vg_set_log_permeability(self.h, t.ctypes.data, 0), self.h)

    # ---- operator / vectors (torch CUDA tensors)
    def zeros(self, dtype=None):
        torch = _torch()
        return torch.zeros(self.N, dtype=dtype or torch.float64, device="cuda")

    def apply(self, x, constrained=True, out=None, internal_order=False):
        """y = K x (reference sign). internal_order: x and y in the solver's internal order (see
        permute), no permutation at the boundary."""
        torch = _torch()
        prec = L.FP64 if x.dtype == torch.float64 else L.FP32
        if internal_order:
            prec |= L.ORDER_INTERNAL
        y = out if out is not None else torch.empty_like(x)
        stream = torch.cuda.current_stream().cuda_stream
        L.check(L.lib().vg_apply(self.h, x.data_ptr(), y.data_ptr(), prec, int(constrained), stream), self.h)
        return y

    def permute(self, x, to_internal=True):
        """Vector in the reference order -> the solver's internal order (to_internal=False: back)."""
        torch = _torch()
        prec = L.FP64 if x.dtype == torch.float64 else L.FP32
        y = torch.empty_like(x)
        stream = torch.cuda.current_stream().cuda_stream
        L.check(L.lib().vg_permute(self.h, int(to_internal), x.data_ptr(), y.data_ptr(), prec, stream), self.h)
        return y

    def rhs(self):
        b = self.zeros()
        L.check(L.lib().vg_rhs(self.h, b.data_ptr()), self.h)
        return b

    @staticmethod
    def opts(mode="fp64", tol=1e-10, maxit=200000, inner_tol=1e-6, max_outer=12, check_every=0, guess=False):
        o = L.VgSolveOpts()
        L.lib().vg_default_solve_opts(ctypes.byref(o))
        o.mode = L.SOLVE_MIXED if mode == "mixed" else L.SOLVE_FP64
        o.tol, o.maxit, o.inner_tol, o.max_outer, o.check_every = tol, maxit, inner_tol, max_outer, check_every
        o.nonzero_guess = int(guess)
        return o

    def solve(self, b=None, x=None, **kw):
        """Solve on the device; returns (x, info dict)."""
        b = self.rhs() if b is None else b
        x = self.zeros() if x is None else x
        info = L.VgSolveInfo()
        o = self.opts(guess=x is not None and kw.pop("guess", False), **kw)
        L.check(L.lib().vg_solve(self.h, b.data_ptr(), x.data_ptr(), ctypes.byref(o), ctypes.byref(info)), self.h)
        return x, dict(iterations=info.iterations, outer=info.outer, residual=info.residual, seconds=info.seconds)

    def solve_host(self, b, out=None, **kw):
        """End-to-end solve from host memory: b (numpy) -> x (numpy; `out` if given, e.g. a view of
        pinned memory)."""
        b = np.ascontiguousarray(b, np.float64)
        if out is not None:
            if out.dtype != np.float64 or out.shape != (self.N,) or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous float64 array of length N")
            x = out
        else:
            x = np.zeros(self.N)
        info = L.VgSolveInfo()
        o = self.opts(**kw)
        L.check(L.lib().vg_solve_host(self.h, b.ctypes.data, x.ctypes.data, ctypes.byref(o), ctypes.byref(info)),
                self.h)
        return x, dict(iterations=info.iterations, outer=info.outer, residual=info.residual, seconds=info.seconds)

    def adjoint_grad(self, x, dJdx, **kw):
        g = _torch().zeros(self.nc, dtype=x.dtype, device="cuda")
        info = L.VgSolveInfo()
        o = self.opts(**kw)
        L.check(L.lib().vg_adjoint_grad(self.h, x.data_ptr(), dJdx.contiguous().data_ptr(), g.data_ptr(),
                                        ctypes.byref(o), ctypes.byref(info)), self.h)
        return g, dict(iterations=info.iterations, outer=info.outer, residual=info.residual, seconds=info.seconds)

    def errors(self, x):
        out = (ctypes.c_double * 6)()
        L.check(L.lib().vg_errors(self.h, x.data_ptr(), out), self.h)
        return dict(zip(("scalar_comp", "flux_comp", "scalar_phys", "flux_phys", "div_phys", "mass"), list(out)))

    def assemble_csr(self, constrained=True):
        """Assembled system as a torch sparse CSR tensor on the device (vg_assemble_csr; reference
        sign). A comparator of the matrix-free apply: its SpMV runs in cuSPARSE."""
        torch = _torch()
        nnz = ctypes.c_longlong(0)
        L.check(L.lib().vg_assemble_csr(self.h, int(constrained), ctypes.byref(nnz), None, None, None), self.h)
        rp = torch.empty(self.N + 1, dtype=torch.int64, device="cuda")
        ci = torch.empty(nnz.value, dtype=torch.int32, device="cuda")
        val = torch.empty(nnz.value, dtype=torch.float64, device="cuda")
        L.check(L.lib().vg_assemble_csr(self.h, int(constrained), ctypes.byref(nnz), rp.data_ptr(), ci.data_ptr(),
                                        val.data_ptr()), self.h)
        return torch.sparse_csr_tensor(rp, ci.long(), val, size=(self.N, self.N))

    def stats(self):
        out = (ctypes.c_longlong * 4)()
        L.check(L.lib().vg_stats(self.h, out), self.h)
        return dict(launches=out[0], applies=out[1], iterations=out[2], solves=out[3])

    def local(self, cell, which):
        names = dict(A=0, W=1, P=2, alpha=3, map=4, rhs=5, dload=6)
        buf = np.zeros(20000)
        cnt = ctypes.c_int()
        L.check(L.lib().vg_local(self.h, cell, names[which], buf.ctypes.data, ctypes.byref(cnt)), self.h)
        return buf[:cnt.value].copy()


class DarcySolver:
    """The reference CPU class's call sequence (vem/CurvedVEM_Darcy/solver/DarcySolver.h:17-126,
    used as in vem/CurvedVEM_Darcy/main/Darcy_curved_main.cpp:54-92) on the GPU. ``problem`` is
    the reference Darcy example index: 1 = sine-perturbed map eps=0.05, 2 = identity map
    (vem/CurvedVEM_Darcy_gpu/examples/darcy_problem.cpp:110-200); essential normal-flux BC with the
    zero-mean pressure multiplier."""

    def __init__(self, mesh_reader, problem=1, gauss_point_num=9, gauss_point_num_1d=9, k=1):
        if problem not in (1, 2):
            raise ValueError("Darcy example must be 1 or 2")
        self.gpu = DarcyGpu(mesh_reader, k=k, nq=gauss_point_num, ng=gauss_point_num_1d, geometry="sine",
                            eps=0.05 if problem == 1 else 0.0, problem="sincos", bc="flux")
        self._x = None
        self._err = None

    def getTotalDofFlux(self):
        return self.gpu.nf

    def getTotalDofConc(self):
        return self.gpu.np

    def solve(self, tol=1e-10):
        self._x, self.info = self.gpu.solve(tol=tol)
        self._err = None
        return True

    def _errors(self):
        if self._x is None:
            raise RuntimeError("error requires a completed numerical solution")
        if self._err is None:
            self._err = self.gpu.errors(self._x)
        return self._err

    def computeL2ErrorPressure(self, gauss_point_num=9):
        return self._errors()["scalar_comp"]

    def computeL2ErrorFlux(self, gauss_point_num=9):
        return self._errors()["flux_comp"]

    def getSolution(self):
        return None if self._x is None else self._x.cpu().numpy()
