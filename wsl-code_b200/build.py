"""Build the vemgpu shared libraries in-tree (sm_100a only).

    python wsl-code_b200/build.py [--force]

* vemgpu/libvemgpu.so — CUDA kernels + C ABI (include/vemgpu.h), nvcc -gencode
  arch=compute_100a,code=sm_100a, static CUDA runtime.
* vemgpu/libvgmesh.so — host-only Lloyd relaxation used by the synthetic mesh generator.

Translation units are compiled in parallel and only when a source is newer than its object.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "vemgpu")
OBJ = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
CUDA_UNITS = ["vg_mesh", "vg_setup", "vg_apply", "vg_krylov", "vg_aux", "vg_amg", "vg_solver", "vg_ms", "vg_capi"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]
LIB = os.path.join(OUT, "libvemgpu.so")
MESHLIB = os.path.join(OUT, "libvgmesh.so")


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    return hs + [os.path.join(INCLUDE, "vemgpu.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(nvcc, unit, force):
    src = os.path.join(CSRC, unit + ".cu")
    obj = os.path.join(OBJ, unit + ".o")
    if force or _stale(obj, [src] + _headers()):
        cmd = [nvcc] + NVCC_FLAGS + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {unit}.cu:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force=False, verbose=True):
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda u: _compile(nvcc, u, force), CUDA_UNITS))
    if force or _stale(LIB, objs):
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    msrc = os.path.join(CSRC, "vg_meshgen.cpp")
    if force or _stale(MESHLIB, [msrc]):
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-shared", "-o", MESHLIB, msrc]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed on vg_meshgen.cpp:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built", LIB, "and", MESHLIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    build(force=ap.parse_args().force)
    sys.exit(0)
