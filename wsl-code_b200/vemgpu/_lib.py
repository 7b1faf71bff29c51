"""ctypes binding of libvemgpu.so (include/vemgpu.h). The library is built in-tree by
wsl-code_b200/build.py; there is no fallback: a missing library is an error."""
import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB_PATH = os.path.join(HERE, "libvemgpu.so")
HEADER = os.path.join(ROOT, "include", "vemgpu.h")

ORDER_INTERNAL = 0x100
VG_OK, VG_EINVAL, VG_EMESH, VG_EGEOMETRY, VG_ESINGULAR, VG_ECUDA, VG_ENOCONV, VG_ESTATE, VG_ENOMEM = range(9)
GEOM = {"identity": 0, "sine": 1, "arcs": 2}
PROBLEM = {"sincos": 1, "sinsin": 2, "annulus": 3}
BC = {"flux": 0, "pressure": 1}
FP64, FP32 = 0, 1
SOLVE_FP64, SOLVE_MIXED = 0, 1
CODE_NAMES = {0: "VG_OK", 1: "VG_EINVAL", 2: "VG_EMESH", 3: "VG_EGEOMETRY", 4: "VG_ESINGULAR", 5: "VG_ECUDA",
              6: "VG_ENOCONV", 7: "VG_ESTATE", 8: "VG_ENOMEM"}


class VemGpuError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{CODE_NAMES.get(code, code)}: {message}")
        self.code = code


P, I, D, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong


class VgMesh(ctypes.Structure):
    _fields_ = [("num_nodes", I), ("num_cells", I), ("num_edges", I), ("node_coords", P), ("cell_nodes", P),
                ("cell_node_indices", P), ("nodes_per_cell", P), ("global_edges", P), ("cell_edge_indices", P),
                ("edge_endpoints", P), ("edge_occurrence", P), ("cell_centroid_x", P), ("cell_centroid_y", P),
                ("cell_diameter", P)]


class VgGeometry(ctypes.Structure):
    _fields_ = [("kind", I), ("eps", D), ("num_arcs", I), ("arc_nodes", P), ("arc_circles", P)]


class VgSolveOpts(ctypes.Structure):
    _fields_ = [("mode", I), ("tol", D), ("maxit", I), ("inner_tol", D), ("max_outer", I), ("check_every", I),
                ("nonzero_guess", I)]


class VgSolveInfo(ctypes.Structure):
    _fields_ = [("iterations", I), ("outer", I), ("residual", D), ("seconds", D)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python wsl-code_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        L.vg_create.argtypes = [ctypes.POINTER(VgMesh), ctypes.POINTER(VgGeometry), I, I, I, I, ctypes.POINTER(P)]
        L.vg_create_polygons.argtypes = [I, P, I, P, P, ctypes.POINTER(VgGeometry), I, I, I, I, ctypes.POINTER(P)]
        L.vg_create_vtk.argtypes = [ctypes.c_char_p, ctypes.POINTER(VgGeometry), I, I, I, I, ctypes.POINTER(P)]
        L.vg_destroy.argtypes = [P]
        L.vg_last_error.argtypes = [P]
        L.vg_last_error.restype = ctypes.c_char_p
        L.vg_sizes.argtypes = [P, P]
        L.vg_set_problem.argtypes = [P, I, I]
        L.vg_set_log_permeability.argtypes = [P, P, I]
        L.vg_build.argtypes = [P]
        L.vg_apply.argtypes = [P, P, P, I, I, P]
        L.vg_rhs.argtypes = [P, P]
        L.vg_permute.argtypes = [P, I, P, P, I, P]
        L.vg_default_solve_opts.argtypes = [ctypes.POINTER(VgSolveOpts)]
        L.vg_default_solve_opts.restype = None
        L.vg_solve.argtypes = [P, P, P, ctypes.POINTER(VgSolveOpts), ctypes.POINTER(VgSolveInfo)]
        L.vg_solve_host.argtypes = [P, P, P, ctypes.POINTER(VgSolveOpts), ctypes.POINTER(VgSolveInfo)]
        L.vg_adjoint_grad.argtypes = [P, P, P, P, ctypes.POINTER(VgSolveOpts), ctypes.POINTER(VgSolveInfo)]
        L.vg_errors.argtypes = [P, P, P]
        L.vg_errors_noalloc.argtypes = [P, P, P]
        L.vg_local.argtypes = [P, I, I, P, ctypes.POINTER(I)]
        L.vg_assemble_csr.argtypes = [P, I, ctypes.POINTER(LL), P, P, P]
        L.vg_cell_areas.argtypes = [P, P]
        L.vg_ms_configure.argtypes = [P, D, D, D, D, ctypes.POINTER(LL)]
        L.vg_ms_apply.argtypes = [P, P, P, P, I]
        L.vg_ms_step.argtypes = [P, P, P, ctypes.POINTER(VgSolveOpts), ctypes.POINTER(VgSolveInfo)]
        L.vg_stats.argtypes = [P, P]
        L.vg_debug_stall_apply.argtypes = [P]
        L.vg_ms_set_picard.argtypes = [P, I, D]
        L.vg_ms_picard_info.argtypes = [P, ctypes.POINTER(I), ctypes.POINTER(D), ctypes.POINTER(D)]
        L.vg_ms_gs_info.argtypes = [P, ctypes.POINTER(LL), ctypes.POINTER(LL)]
        _lib = L
    return _lib


def check(code, handle=None):
    if code != VG_OK:
        msg = lib().vg_last_error(handle)
        raise VemGpuError(code, msg.decode() if msg else "")


def header_functions():
    """Names of the functions declared in include/vemgpu.h."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(vg_\w+)\s*\(", text, re.M)))
