"""ORACLE — test infrastructure only (the checker, never the thing measured or shipped).

Python side of the CPU FP64 restatement in ``vem_oracle.cpp``:

* ``Oracle``: element matrices, assembled saddle-point system in the reference sign
  ``[A, -W^T, 0; W, 0, L; 0, L^T, 0]`` (vem/CurvedVEM_Darcy/solver/DarcySolver.cpp:402-500),
  essential normal-flux boundary data (DarcySolver.cpp:502-663), Dirichlet pressure loads,
  the six error figures (DarcySolver.cpp:942-1131, vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:387-462).
* ``solve_direct``: the discrete solution by sparse LU (scipy SuperLU) on the reduced system of
  DarcySolver::solveWithDirichletBC (DarcySolver.cpp:665-788) — the golden discrete solution.
* ``reference_solve``: the reference CPU algorithm restated end to end (assembly + GMRES(100) +
  ILU(0), rtol 1e-10; vem/CurvedVEM_Darcy/core/petsc_utils.cpp:144-211) for the CPU baseline.
* ``read_gmsh41``: the gmsh 4.1 ASCII reader of vem/CurvedVEM_Darcy_gpu/mesh/straight_mesh.cpp:238-431
  (raw node coordinates and polygon node lists, before CCW reordering).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libvemref.so")

GEOM_IDENTITY, GEOM_SINE, GEOM_ARCS = 0, 1, 2
PROB_SINCOS, PROB_SINSIN, PROB_ANNULUS = 1, 2, 3
BC_FLUX, BC_PRESSURE = 0, 1

_lib = None


def build():
    """Compile liboracle.so (and oracle/_ref when the reference checkout is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all", "ref-if-present"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P, I, D, V = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p
        L.orc_create.restype = P
        L.orc_create.argtypes = [I, P, I, P, P, I, I, I, I, D, I, P, P, I, I, P, I]
        L.orc_free.argtypes = [P]
        L.orc_info.argtypes = [P, P]
        L.orc_mesh.argtypes = [P] + [P] * 8
        L.orc_csr.restype = ctypes.c_long
        L.orc_csr.argtypes = [P, P, P, P, P]
        L.orc_boundary.argtypes = [P, P, P]
        L.orc_local.restype = ctypes.c_long
        L.orc_local.argtypes = [P, I, I, P]
        L.orc_samples.restype = ctypes.c_long
        L.orc_samples.argtypes = [P, I, I, P]
        L.orc_errors.argtypes = [P, P, P]
        L.orc_adjoint_contract.argtypes = [P, P, P, P, P]
        L.orc_gmres_ilu.restype = I
        L.orc_gmres_ilu.argtypes = [I, P, P, P, P, P, D, I, I, P]
        L.orc_reference_solve.restype = I
        L.orc_reference_solve.argtypes = [I, P, I, P, P, I, I, I, I, D, I, P, P, I, I, P, I, D, I, P, P, P]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_triangles.restype = ctypes.c_long
        L.orc_triangles.argtypes = [P, I, P]
        L.orc_tri_points.restype = I
        L.orc_tri_points.argtypes = [P, I, P]
        L.orc_line_points.restype = I
        L.orc_line_points.argtypes = [I, D, D, D, D, P]
        L.orc_mono.restype = D
        L.orc_mono.argtypes = [I, D, D, D, D, D]
        L.orc_hdiv.argtypes = [I, I, D, D, D, D, D, P]
        L.orc_edge_coeffs.argtypes = [I, I, D, D, D, D, D, D, D, P]
        L.orc_problem.argtypes = [I, D, D, D, P]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _mesh_args(mesh):
    xy = np.ascontiguousarray(mesh["xy"], dtype=np.float64).reshape(-1)
    ptr = np.ascontiguousarray(mesh["cell_ptr"], dtype=np.int32)
    nodes = np.ascontiguousarray(mesh["cell_nodes"], dtype=np.int32)
    arcs_n = mesh.get("arc_nodes")
    arcs_d = mesh.get("arc_data")
    if arcs_n is not None and len(arcs_n):
        arcs_n = np.ascontiguousarray(arcs_n, dtype=np.int32).reshape(-1)
        arcs_d = np.ascontiguousarray(arcs_d, dtype=np.float64).reshape(-1)
        na = len(arcs_n) // 2
    else:
        arcs_n = arcs_d = None
        na = 0
    return xy, ptr, nodes, arcs_n, arcs_d, na


class Oracle:
    """CPU FP64 restatement of the reference element / assembly path for one mesh and problem."""

    def __init__(self, mesh, k=0, nq=9, ng=9, geom=GEOM_IDENTITY, eps=0.0, problem=PROB_SINCOS,
                 bc=BC_FLUX, theta=None, threads=0):
        L = lib()
        xy, ptr, nodes, an, ad, na = _mesh_args(mesh)
        self._keep = (xy, ptr, nodes, an, ad)
        nc = len(ptr) - 1
        th = None if theta is None else np.ascontiguousarray(theta, dtype=np.float64)
        self.h = L.orc_create(len(xy) // 2, _p(xy), nc, _p(ptr), _p(nodes), k, nq, ng, geom, eps, na,
                              _p(an), _p(ad), problem, bc, _p(th), threads)
        if not self.h:
            raise RuntimeError("oracle: " + L.orc_last_error().decode())
        info = np.zeros(9, dtype=np.int64)
        L.orc_info(self.h, info.ctypes.data)
        (self.nc, self.ne, self.nf, self.np, self.N, self.q, self.p, self.internal, self.nn) = map(int, info)
        self.k, self.bc = k, bc

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    def mesh_arrays(self):
        nodes = np.zeros(len(self._keep[2]), np.int32)
        ge = np.zeros(len(self._keep[2]), np.int32)
        ee = np.zeros(2 * self.ne, np.int32)
        occ = np.zeros(self.ne, np.int32)
        cx, cy, dm, ar = (np.zeros(self.nc) for _ in range(4))
        lib().orc_mesh(self.h, *(a.ctypes.data for a in (nodes, ge, ee, occ, cx, cy, dm, ar)))
        return dict(cell_nodes=nodes, global_edges=ge, edge_endpoints=ee, edge_occurrence=occ,
                    cx=cx, cy=cy, diameter=dm, area=ar)

    def system(self):
        """Full assembled matrix (scipy CSR, reference sign) and right-hand side."""
        import scipy.sparse as sp
        L = lib()
        nnz = L.orc_csr(self.h, None, None, None, None)
        ptr = np.zeros(self.N + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        b = np.zeros(self.N)
        L.orc_csr(self.h, ptr.ctypes.data, col.ctypes.data, val.ctypes.data, b.ctypes.data)
        return sp.csr_matrix((val, col, ptr), shape=(self.N, self.N)), b

    def boundary(self):
        mask = np.zeros(self.N, np.int32)
        g = np.zeros(self.N)
        lib().orc_boundary(self.h, mask.ctypes.data, g.ctypes.data)
        return mask.astype(bool), g

    def local(self, cell, which):
        names = dict(A=0, W=1, P=2, D=3, G=4, B=5, AG=6, M=7, alpha=8, L=9, rhs=10, dir=11, gdofs=12,
                     dload=13, area=14, H=15, Hs=16)
        w = names[which]
        n = lib().orc_local(self.h, cell, w, None)
        out = np.zeros(n)
        lib().orc_local(self.h, cell, w, out.ctypes.data)
        return out

    def triangles(self, cell):
        n = lib().orc_triangles(self.h, cell, None)
        out = np.zeros((n, 6))
        lib().orc_triangles(self.h, cell, out.ctypes.data)
        return out

    def samples(self, cell, edge=False):
        n = lib().orc_samples(self.h, cell, int(edge), None)
        out = np.zeros((n, 10))
        lib().orc_samples(self.h, cell, int(edge), out.ctypes.data)
        return out

    def errors(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(6)
        lib().orc_errors(self.h, x.ctypes.data, out.ctypes.data)
        return dict(scalar_comp=out[0], flux_comp=out[1], scalar_phys=out[2], flux_phys=out[3],
                    div_phys=out[4], mass=out[5])

    def adjoint_contract(self, x, lam, mask=None):
        """Per-cell g_E = (S_E lam_E)^T A_E (S_E x_E), lam zero on masked rows (CPU FP64)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
        g = np.zeros(self.nc)
        lib().orc_adjoint_contract(self.h, x.ctypes.data, lam.ctypes.data, _p(m), g.ctypes.data)
        return g

    def solve_direct(self):
        """Golden discrete solution: sparse LU on the reduced system (free dofs)."""
        import scipy.sparse.linalg as spla
        K, b = self.system()
        mask, g = self.boundary()
        if self.bc == BC_PRESSURE:
            mask[:] = False
            g[:] = 0.0
        free = ~mask
        rhs = b - K @ g
        Kf = K[free][:, free].tocsc()
        x = g.copy()
        x[free] = spla.spsolve(Kf, rhs[free], permc_spec="COLAMD")
        return x, K, b


def gmres_ilu(K, b, rtol=1e-10, restart=100, maxit=1000000):
    """GMRES(restart)+ILU(0) of petsc_utils.cpp:144-211 on a scipy CSR matrix (sorted indices)."""
    K = K.tocsr()
    K.sort_indices()
    ptr = np.ascontiguousarray(K.indptr, np.int32)
    col = np.ascontiguousarray(K.indices, np.int32)
    val = np.ascontiguousarray(K.data, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b)
    rel = np.zeros(1)
    it = lib().orc_gmres_ilu(K.shape[0], ptr.ctypes.data, col.ctypes.data, val.ctypes.data, b.ctypes.data,
                             x.ctypes.data, rtol, restart, maxit, rel.ctypes.data)
    if it < 0:
        raise RuntimeError("oracle gmres: " + lib().orc_last_error().decode())
    return x, it, float(rel[0])


def reference_solve(mesh, k=0, nq=9, ng=9, geom=GEOM_IDENTITY, eps=0.0, problem=PROB_SINCOS, bc=BC_FLUX,
                    theta=None, threads=1, rtol=1e-10, maxit=1000000):
    """The reference CPU solve restated (assembly + GMRES(100)+ILU(0)); returns x, iters, times."""
    L = lib()
    xy, ptr, nodes, an, ad, na = _mesh_args(mesh)
    nc = len(ptr) - 1
    q = (k + 1) * (k + 2) // 2
    # global size from the polygon lists (edges counted once)
    e = set()
    for c in range(nc):
        nd = nodes[ptr[c]:ptr[c + 1]]
        for j in range(len(nd)):
            a, b2 = int(nd[j]), int(nd[(j + 1) % len(nd)])
            e.add((min(a, b2), max(a, b2)))
    internal = (q - 1) + (q - (k + 1))
    N = len(e) * (k + 1) + nc * internal + nc * q + (1 if bc == BC_FLUX else 0)
    th = None if theta is None else np.ascontiguousarray(theta, dtype=np.float64)
    x = np.zeros(N)
    times = np.zeros(2)
    rel = np.zeros(1)
    it = L.orc_reference_solve(len(xy) // 2, _p(xy), nc, _p(ptr), _p(nodes), k, nq, ng, geom, eps, na, _p(an),
                               _p(ad), problem, bc, _p(th), threads, rtol, maxit, x.ctypes.data,
                               times.ctypes.data, rel.ctypes.data)
    if it < 0:
        raise RuntimeError("oracle reference solve: " + L.orc_last_error().decode())
    return x, it, dict(assembly_s=float(times[0]), solve_s=float(times[1]), rel=float(rel[0]))


def read_gmsh41(path):
    """gmsh 4.1 ASCII reader (straight_mesh.cpp:238-431): node coordinates and polygon elements.

    Returns dict(xy (nn,2), cell_ptr, cell_nodes) with 0-based node ids in file order; element
    types 2/3/11/12 (3, 4, 5, 6 nodes) are polygons, lower-dimensional blocks are skipped.
    """
    with open(path) as f:
        lines = f.read().splitlines()
    i = lines.index("$Nodes") + 1
    nblocks, nn = map(int, lines[i].split()[:2])
    i += 1
    xy = np.zeros((nn, 2))
    for _ in range(nblocks):
        _, _, _, cnt = map(int, lines[i].split()[:4])
        i += 1
        tags = []
        while len(tags) < cnt:
            tags += [int(t) for t in lines[i].split()]
            i += 1
        for t in tags:
            vals = lines[i].split()
            xy[t - 1] = float(vals[0]), float(vals[1])
            i += 1
    i = lines.index("$Elements") + 1
    nblocks = int(lines[i].split()[0])
    i += 1
    per_type = {2: 3, 3: 4, 11: 5, 12: 6}
    ptr, nodes = [0], []
    for _ in range(nblocks):
        _, _, etype, cnt = map(int, lines[i].split()[:4])
        i += 1
        npe = per_type.get(etype, -1)
        for _ in range(cnt):
            if npe >= 3:
                vals = [int(v) for v in lines[i].split()]
                nodes += [v - 1 for v in vals[1:1 + npe]]
                ptr.append(len(nodes))
            i += 1
    return dict(xy=xy, cell_ptr=np.array(ptr, np.int32), cell_nodes=np.array(nodes, np.int32))


def tri_points(vertices, nq):
    v = np.ascontiguousarray(vertices, np.float64)
    out = np.zeros((64, 3))
    n = lib().orc_tri_points(v.ctypes.data, nq, out.ctypes.data)
    return out[:n]


def line_points(order, x1, y1, x2, y2):
    out = np.zeros((16, 3))
    n = lib().orc_line_points(order, x1, y1, x2, y2, out.ctypes.data)
    return out[:n]


def mono(idx, frame, x, y):
    return lib().orc_mono(idx, *frame, x, y)


def hdiv(k, idx, frame, x, y):
    out = np.zeros(2)
    lib().orc_hdiv(k, idx, *frame, x, y, out.ctypes.data)
    return out


def edge_coeffs(k, idx, frame, x0, y0, x1, y1):
    out = np.zeros(k + 1)
    lib().orc_edge_coeffs(k, idx, *frame, x0, y0, x1, y1, out.ctypes.data)
    return out


def problem_point(kind, eps, xi, eta):
    out = np.zeros(11)
    lib().orc_problem(kind, eps, xi, eta, out.ctypes.data)
    return out
