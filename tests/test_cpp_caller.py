"""A compiled C++ caller of libvemgpu.so: tests/cpp/run_case.cpp runs the reference's run_case
sequence (vem/CurvedVEM_Darcy/main/Darcy_curved_main.cpp:54-92) through the header-only facade
include/vemgpu_darcy.hpp. On the CPU: it compiles, links and reports errors through the library's
status (a zero-area cell; no device). On the GPU: the reference's 16-cell mesh (square_2x2,
example 1, k = 1) reproduces the reference's published error report (tolerance 2e-9, as for the
oracle)."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "wsl-code_b200", "vemgpu")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def run_case(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx or not os.path.exists(os.path.join(LIBDIR, "libvemgpu.so")):
        pytest.skip("g++ or libvemgpu.so missing")
    exe = str(tmp_path_factory.mktemp("cpp") / "run_case")
    cmd = [cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "run_case.cpp"), "-o", exe, "-L", LIBDIR, "-lvemgpu",
           f"-Wl,-rpath,{LIBDIR}", "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{CUDA}/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _write_mesh(path, mesh):
    ptr, nodes, xy = mesh["cell_ptr"], mesh["cell_nodes"], mesh["xy"]
    with open(path, "w") as f:
        f.write(f"{len(xy)} {len(ptr) - 1}\n")
        for x, y in xy:
            f.write(f"{float(x)!r} {float(y)!r}\n")
        for c in range(len(ptr) - 1):
            cell = nodes[ptr[c]:ptr[c + 1]]
            f.write(" ".join(str(int(v)) for v in [len(cell), *cell]) + "\n")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_cpp_caller_builds_and_reports_status(run_case, square_meshes, tmp_path):
    p = tmp_path / "m.txt"
    _write_mesh(p, square_meshes["square_2x2"])
    r = subprocess.run([run_case, str(p), "1", "1", "9", "1e-12"], capture_output=True, text=True, timeout=300)
    if not _cuda_available():
        # the library's VG_ECUDA message: no device, or no driver in this process
        assert r.returncode == 1 and ("no CUDA device" in r.stderr or "cudaGetDeviceCount" in r.stderr), r.stderr
    else:
        assert r.returncode == 0, r.stderr
    bad = tmp_path / "bad.txt"
    bad.write_text("3 1\n0 0\n1 0\n2 0\n3 0 1 2\n")  # a cell of zero area
    r = subprocess.run([run_case, str(bad), "1", "1", "9", "1e-12"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "zero area" in r.stderr


@pytest.mark.gpu
def test_cpp_caller_reproduces_reference_report(run_case, square_meshes, golden, tmp_path):
    r0 = next(r for r in golden["reports"] if r["mesh"] == "square_2x2" and r["example"] == 1)
    p = tmp_path / "m.txt"
    _write_mesh(p, square_meshes["square_2x2"])
    r = subprocess.run([run_case, str(p), "1", str(r0["k"]), str(r0["nq"]), "1e-12"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    assert out["dofs"] == r0["dofs"] and out["residual"] <= 1e-12
    for key in ("scalar_comp", "flux_comp", "scalar_phys", "flux_phys", "div_phys"):
        assert out[key] == pytest.approx(r0["values"][key], rel=2e-9), key
    assert abs(out["mass"] - r0["values"]["mass"]) < 1e-8
    assert np.isfinite(out["solution_norm2"]) and out["solution_norm2"] > 0
