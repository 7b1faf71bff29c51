"""Regenerate the committed golden fixtures from the reference checkout (runs where the checkout
is mounted; the fixtures travel, the checkout does not).

Writes, next to this script:

* ``square_meshes.npz`` — the reference's own square meshes
  (vem/CurvedVEM_Darcy_gpu/mesh/data/square_{1,2,4,8,16,32}x*.msh, read with the gmsh 4.1 reader
  restated in oracle/oracle.py): raw node coordinates and polygon node lists (0-based, file order).
* ``golden.json`` — the reference's published Darcy results for those meshes, parsed from
  the GPU project's report.json files (docs/validation/{final_darcy1,darcy1_4,darcy1_8,darcy_k4,
  main_entries_20260910}) and the CPU project's convergence tables
  (vem/CurvedVEM_Darcy/results_darcy_convergence_k{1,2,3_cpu_vs_gpu}.txt).
* ``ref_blocks.npz`` — outputs of the reference's own PETSc-free modules, compiled from source
  into oracle/_ref (oracle/Makefile target ``ref``): processed mesh topology, ear-clipping
  triangles, quadrature points, basis values, edge restriction coefficients and Darcy example
  data at seeded points. These pin the oracle's restated building blocks.

Usage: python tests/golden/make_golden.py
"""
import ctypes
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

# root of the reference checkout (environment variable REFERENCE, same name as in oracle/Makefile)
REFERENCE = os.environ.get("REFERENCE", "/root/reference")
REF = os.path.join(REFERENCE, "vem")
GPU = REF + "/CurvedVEM_Darcy_gpu"
CPU = REF + "/CurvedVEM_Darcy"
MESHES = ["square_1x1", "square_2x2", "square_4x4", "square_8x8", "square_16x16", "square_32x32"]


def meshes():
    out = {}
    for name in MESHES:
        m = O.read_gmsh41(f"{GPU}/mesh/data/{name}.msh")
        out[name + "/xy"] = m["xy"]
        out[name + "/cell_ptr"] = m["cell_ptr"]
        out[name + "/cell_nodes"] = m["cell_nodes"]
    np.savez_compressed(os.path.join(HERE, "square_meshes.npz"), **out)


def reports():
    rows = []
    cases = [("final_darcy1/report.json", "square_2x2"), ("darcy1_4/report.json", "square_4x4"),
             ("darcy1_8/report.json", "square_8x8"), ("darcy_k4/report.json", "square_1x1"),
             ("main_entries_20260910/darcy1_report.json", "square_2x2"),
             ("main_entries_20260910/darcy2_report.json", "square_2x2")]
    for rel, mesh in cases:
        with open(f"{GPU}/docs/validation/{rel}") as f:
            r = json.load(f)
        k = r["k"]
        rows.append(dict(source="vem/CurvedVEM_Darcy_gpu/docs/validation/" + rel, mesh=mesh, example=r["example"],
                         k=k, nq=36 if k == 4 else 12 if k == 3 else 9, ng=9, cells=r["cells"], dofs=r["dofs"],
                         residual=r["residual"],
                         values={key: r[key][0] for key in
                                 ("scalar_comp", "flux_comp", "scalar_phys", "flux_phys", "div_phys", "mass")}))
    return rows


def table(path, k, nq, cols):
    """Rows 'square_NxN nodes cells dofs ... pressure ... flux ...' of a convergence table."""
    rows = []
    with open(path) as f:
        for lineno, line in enumerate(f, 1):
            t = line.split()
            if not t or not re.fullmatch(r"square_\d+x\d+", t[0]):
                continue
            if t[0] not in MESHES:
                continue
            vals = {name: float(t[i]) for name, i in cols.items()}
            rows.append(dict(mesh=t[0], line=lineno, **vals))
    return dict(source=os.path.relpath(path, REFERENCE), k=k, example=1, nq=nq, ng=9, rows=rows)


def tables():
    k1 = dict(cells=2, dofs=3, pressure=7, flux=9)
    k2 = dict(cells=2, dofs=3, pressure=7, flux=9)
    return [table(f"{CPU}/results_darcy_convergence_k1.txt", 1, 9, k1),
            table(f"{CPU}/results_darcy_convergence_k2.txt", 2, 9, k2)]


def k3_table():
    """k=3 CPU pressure / flux errors (two sub-tables of results_darcy_convergence_k3_cpu_vs_gpu.txt)."""
    path = f"{CPU}/results_darcy_convergence_k3_cpu_vs_gpu.txt"
    rows = {}
    section = None
    with open(path) as f:
        for lineno, line in enumerate(f, 1):
            if "压力 L2" in line:
                section = "pressure"
            elif "通量 L2" in line:
                section = "flux"
            elif "求解速度" in line:
                section = None
            t = line.split()
            if section and t and t[0] in MESHES:
                rows.setdefault(t[0], dict(mesh=t[0], dofs=float(t[1])))[section] = float(t[2])
                rows[t[0]]["line_" + section] = lineno
    return dict(source=os.path.relpath(path, REFERENCE), k=3, example=1, nq=12, ng=9,
                rows=list(rows.values()))


def ref_blocks():
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libvemref.so"))
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.ref_read_mesh.restype = P
    L.ref_read_mesh.argtypes = [ctypes.c_char_p, I]
    L.ref_mesh_sizes.argtypes = [P, P]
    L.ref_mesh_arrays.argtypes = [P] + [P] * 10
    L.ref_triangulate.restype = I
    L.ref_triangulate.argtypes = [P, I, P]
    L.ref_triangle_points.restype = I
    L.ref_triangle_points.argtypes = [P, I, P]
    L.ref_line_points.restype = I
    L.ref_line_points.argtypes = [I, D, D, D, D, P]
    L.ref_mono.restype = D
    L.ref_mono.argtypes = [I, I, D, D, D, D, D]
    L.ref_hdiv.argtypes = [I, I, D, D, D, D, D, P]
    L.ref_edge_coeffs.argtypes = [I, I, D, D, D, D, D, D, D, P]
    L.ref_darcy.argtypes = [I, D, D, P]
    out = {}
    for name in ("square_2x2", "square_8x8"):
        h = L.ref_read_mesh(f"{GPU}/mesh/data/{name}.msh".encode(), 0)
        s = np.zeros(4, np.int32)
        L.ref_mesh_sizes(h, s.ctypes.data)
        nn, nc, ne, tot = map(int, s)
        arr = dict(xy=np.zeros(2 * nn), cell_nodes=np.zeros(tot, np.int32), cell_node_indices=np.zeros(nc + 1, np.int32),
                   global_edges=np.zeros(tot, np.int32), edge_endpoints=np.zeros(2 * ne, np.int32),
                   edge_occurrence=np.zeros(ne, np.int32), cx=np.zeros(nc), cy=np.zeros(nc), area=np.zeros(nc),
                   diameter=np.zeros(nc))
        L.ref_mesh_arrays(h, *(arr[key].ctypes.data for key in ("xy", "cell_nodes", "cell_node_indices",
                                                                 "global_edges", "edge_endpoints", "edge_occurrence",
                                                                 "cx", "cy", "area", "diameter")))
        for key, v in arr.items():
            out[f"{name}/{key}"] = v
        tris = []
        for c in range(nc):
            buf = np.zeros(6 * 16)
            nt = L.ref_triangulate(h, c, buf.ctypes.data)
            tris.append(buf[:6 * nt].reshape(nt, 6))
        out[f"{name}/triangles"] = np.stack(tris)
    rng = np.random.default_rng(20261203)
    tri = np.array([0.1, 0.2, 0.7, 0.25, 0.3, 0.9])
    for nq in (1, 3, 4, 7, 9, 12):
        buf = np.zeros(3 * 64)
        n = L.ref_triangle_points(tri.ctypes.data, nq, buf.ctypes.data)
        out[f"tri/{nq}"] = buf[:3 * n].reshape(n, 3)
    out["tri/vertices"] = tri
    for order in range(1, 11):
        buf = np.zeros(3 * 16)
        n = L.ref_line_points(order, 0.2, 0.1, 0.9, 0.6, buf.ctypes.data)
        out[f"line/{order}"] = buf[:3 * n].reshape(n, 3)
    pts = rng.uniform(0, 1, size=(16, 2))
    frame = np.array([0.45, 0.55, 0.37])
    out["basis/points"] = pts
    out["basis/frame"] = frame
    for k in range(5):
        q = (k + 1) * (k + 2) // 2
        nh = (k + 2) * (k + 3) // 2 - 1 + (k * (k + 1) // 2)
        mono = np.array([[L.ref_mono(k, i, *frame, x, y) for i in range(q)] for x, y in pts])
        hd = np.zeros((len(pts), nh, 2))
        buf = np.zeros(2)
        for a, (x, y) in enumerate(pts):
            for i in range(nh):
                L.ref_hdiv(k, i, *frame, x, y, buf.ctypes.data)
                hd[a, i] = buf
        ec = np.zeros((q, k + 1))
        buf = np.zeros(k + 1)
        for i in range(q):
            L.ref_edge_coeffs(k, i, *frame, 0.3, 0.35, 0.62, 0.71, buf.ctypes.data)
            ec[i] = buf
        out[f"basis/mono{k}"] = mono
        out[f"basis/hdiv{k}"] = hd
        out[f"basis/edge{k}"] = ec
    out["basis/edge_points"] = np.array([0.3, 0.35, 0.62, 0.71])
    dp = np.zeros((2, len(pts), 11))
    buf = np.zeros(11)
    for ex in (1, 2):
        for a, (x, y) in enumerate(pts):
            L.ref_darcy(ex, x, y, buf.ctypes.data)
            dp[ex - 1, a] = buf
    out["darcy/values"] = dp
    np.savez_compressed(os.path.join(HERE, "ref_blocks.npz"), **out)


def main():
    O.build()
    meshes()
    data = dict(reports=reports(), tables=tables() + [k3_table()])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(data, f, indent=1)
    ref_blocks()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
