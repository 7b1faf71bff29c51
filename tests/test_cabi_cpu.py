"""CPU checks of the C ABI: the library builds for sm_100a, loads, exports every function
declared in include/vemgpu.h, and reports argument / mesh errors with the right status codes
before any device work (no GPU in this process). No compute calls."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    import importlib.util
    spec = importlib.util.spec_from_file_location("vg_build", os.path.join(ROOT, "wsl-code_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build(verbose=False)
    from vemgpu import _lib
    return _lib


def test_exports_every_declared_function(L):
    names = L.header_functions()
    assert len(names) >= 16
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = L.lib()
    for n in names:
        assert hasattr(lib, n)


def test_build_targets_sm100a_only():
    import importlib.util
    spec = importlib.util.spec_from_file_location("vg_build", os.path.join(ROOT, "wsl-code_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    gencodes = [mod.NVCC_FLAGS[i + 1] for i, f in enumerate(mod.NVCC_FLAGS) if f == "-gencode"]
    assert gencodes == ["arch=compute_100a,code=sm_100a"]


def _square(n=2):
    xs = np.linspace(0, 1, n + 1)
    xy = np.array([(x, y) for y in xs for x in xs])
    cells = []
    for j in range(n):
        for i in range(n):
            a = j * (n + 1) + i
            cells.append([a, a + 1, a + n + 2, a + n + 1])
    ptr = np.arange(0, 4 * len(cells) + 1, 4, dtype=np.int32)
    return xy, ptr, np.array(cells, np.int32).reshape(-1)


def _create(L, xy, ptr, nodes, k=0, nq=9, ng=9):
    h = ctypes.c_void_p()
    g = L.VgGeometry()
    code = L.lib().vg_create_polygons(len(xy), np.ascontiguousarray(xy, np.float64).ctypes.data, len(ptr) - 1,
                                      ptr.ctypes.data, nodes.ctypes.data, ctypes.byref(g), k, nq, ng, -1,
                                      ctypes.byref(h))
    return code, h


@pytest.mark.parametrize("k,nq,ng", [(5, 9, 9), (1, 1, 9), (3, 9, 9), (4, 12, 9), (2, 4, 9), (1, 9, 2), (0, 2, 9)])
def test_invalid_options_rejected(L, k, nq, ng):
    xy, ptr, nodes = _square()
    code, h = _create(L, xy, ptr, nodes, k, nq, ng)
    assert code == L.VG_EINVAL
    assert not h.value
    assert L.lib().vg_last_error(None)


def test_bad_meshes_rejected(L):
    xy, ptr, nodes = _square()
    # a 2-vertex cell
    code, _ = _create(L, xy, np.array([0, 2], np.int32), nodes[:2].copy())
    assert code == L.VG_EMESH
    # an edge shared by three cells
    tri = np.array([0, 1, 3, 1, 0, 4, 0, 1, 5], np.int32)
    pts = np.array([[0, 0], [1, 0], [0, 0], [0.5, 1], [0.5, -1], [0.7, 0.5]], float)
    code, _ = _create(L, pts, np.array([0, 3, 6, 9], np.int32), tri)
    assert code == L.VG_EMESH
    # node index out of range
    bad = nodes.copy()
    bad[0] = 99
    code, _ = _create(L, xy, ptr, bad)
    assert code == L.VG_EMESH


def test_no_device_is_reported(L):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    xy, ptr, nodes = _square()
    code, h = _create(L, xy, ptr, nodes)
    assert code == L.VG_ECUDA
    assert not h.value


def test_default_options(L):
    o = L.VgSolveOpts()
    L.lib().vg_default_solve_opts(ctypes.byref(o))
    assert o.mode == L.SOLVE_FP64 and o.tol == 1e-10 and o.check_every == 0 and 0 < o.inner_tol < 1


def test_vtk_reader_errors_before_device_work(L, tmp_path):
    """vg_create_vtk parses and checks the file on the host before any device call."""
    h = ctypes.c_void_p()
    g = L.VgGeometry()
    code = L.lib().vg_create_vtk(str(tmp_path / "missing.vtk").encode(), ctypes.byref(g), 1, 9, 9, -1, ctypes.byref(h))
    assert code == L.VG_EINVAL and b"cannot open" in L.lib().vg_last_error(None)
    p = tmp_path / "bad.vtk"
    p.write_text("# vtk DataFile Version 2.0\nx\nASCII\nDATASET UNSTRUCTURED_GRID\nPOINTS 3 float\n0 0 0 1 0 0 0 1 0\n"
                 "CELLS 1 4\n3 0 1 2\nCELL_TYPES 1\n12\n")
    code = L.lib().vg_create_vtk(str(p).encode(), ctypes.byref(g), 1, 9, 9, -1, ctypes.byref(h))
    assert code == L.VG_EMESH and b"unsupported type" in L.lib().vg_last_error(None)
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        p.write_text(p.read_text().replace("\n12\n", "\n5\n"))
        code = L.lib().vg_create_vtk(str(p).encode(), ctypes.byref(g), 1, 9, 9, -1, ctypes.byref(h))
        assert code == L.VG_ECUDA
