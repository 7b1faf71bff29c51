"""Legacy ASCII VTK polygon meshes, the format read by the reference's StraightMeshReader::read_mesh_vtk
(vem/CurvedVEM_Darcy_gpu/mesh/straight_mesh.cpp:68-218): POINTS (x y z, z ignored), CELLS (vertex
count then vertices), CELL_TYPES (5 triangle, 7 polygon, 9 quad). Circular boundary arcs, which
that reader does not know, travel in a dataset-level FIELD block (arrays arc_nodes and arc_data) that
its token scanner skips; per-cell values (log permeability, pressure) can be written as CELL_DATA.
``vg_create_vtk`` of the C ABI reads the same files in C++.
"""
import numpy as np


def write_vtk(path, mesh, cell_data=None, title="vemgpu polygon mesh"):
    xy = np.asarray(mesh["xy"], np.float64).reshape(-1, 2)
    ptr = np.asarray(mesh["cell_ptr"], np.int64)
    nodes = np.asarray(mesh["cell_nodes"], np.int64)
    nc = len(ptr) - 1
    cnt = np.diff(ptr)
    with open(path, "w") as f:
        f.write(f"# vtk DataFile Version 3.0\n{title}\nASCII\nDATASET UNSTRUCTURED_GRID\n")
        an, ad = mesh.get("arc_nodes"), mesh.get("arc_data")
        if an is not None and len(an):
            an = np.asarray(an, np.int64).reshape(-1, 2)
            ad = np.asarray(ad, np.float64).reshape(-1, 3)
            f.write("FIELD FieldData 2\n")
            f.write(f"arc_nodes 2 {len(an)} int\n")
            np.savetxt(f, an, fmt="%d")
            f.write(f"arc_data 3 {len(ad)} double\n")
            np.savetxt(f, ad, fmt="%.17g")
        f.write(f"POINTS {len(xy)} double\n")
        np.savetxt(f, np.c_[xy, np.zeros(len(xy))], fmt="%.17g")
        f.write(f"CELLS {nc} {nc + len(nodes)}\n")
        for c in range(nc):
            f.write(" ".join(map(str, [cnt[c]] + nodes[ptr[c]:ptr[c + 1]].tolist())) + "\n")
        f.write(f"CELL_TYPES {nc}\n")
        types = np.where(cnt == 3, 5, np.where(cnt == 4, 9, 7))
        np.savetxt(f, types, fmt="%d")
        if cell_data:
            f.write(f"CELL_DATA {nc}\n")
            for name, v in cell_data.items():
                v = np.asarray(v, np.float64).reshape(-1)
                if len(v) != nc:
                    raise ValueError(f"cell data {name} has {len(v)} values for {nc} cells")
                f.write(f"SCALARS {name} double 1\nLOOKUP_TABLE default\n")
                np.savetxt(f, v, fmt="%.17g")


def read_vtk(path):
    """Raw polygon mesh dict (xy, cell_ptr, cell_nodes[, arc_nodes, arc_data]) with the reference
    reader's checks (at least 3 vertices, node range, cell types 5/7/9, counts)."""
    with open(path) as f:
        tok = f.read().split()
    pos = {}

    def find(key, start=0):
        try:
            return tok.index(key, start)
        except ValueError:
            return -1
    out = {}
    i = find("FIELD")
    p0 = find("POINTS")
    if i >= 0 and (p0 < 0 or i < p0):
        narr, j = int(tok[i + 2]), i + 3
        for _ in range(narr):
            name, ncomp, ntup = tok[j], int(tok[j + 1]), int(tok[j + 2])
            vals = np.array(tok[j + 4:j + 4 + ncomp * ntup], np.float64).reshape(ntup, ncomp)
            j += 4 + ncomp * ntup
            if name == "arc_nodes":
                out["arc_nodes"] = vals.astype(np.int64)
            elif name == "arc_data":
                out["arc_data"] = vals
    if p0 < 0:
        raise ValueError("VTK: POINTS section not found")
    nn = int(tok[p0 + 1])
    pts = np.array(tok[p0 + 3:p0 + 3 + 3 * nn], np.float64).reshape(nn, 3)
    c0 = find("CELLS", p0 + 3 + 3 * nn)
    if c0 < 0:
        raise ValueError("VTK: CELLS section not found")
    nc, total = int(tok[c0 + 1]), int(tok[c0 + 2])
    flat = np.array(tok[c0 + 3:c0 + 3 + total], np.int64)
    ptr, nodes, j = [0], [], 0
    for c in range(nc):
        nv = int(flat[j])
        if nv < 3:
            raise ValueError(f"VTK: cell {c} has fewer than 3 vertices")
        v = flat[j + 1:j + 1 + nv]
        if v.min() < 0 or v.max() >= nn:
            raise ValueError(f"VTK: cell {c} references a node out of range")
        nodes.append(v)
        ptr.append(ptr[-1] + nv)
        j += nv + 1
    t0 = find("CELL_TYPES", c0 + 3 + total)
    if t0 < 0:
        raise ValueError("VTK: CELL_TYPES section not found")
    if int(tok[t0 + 1]) != nc:
        raise ValueError("VTK: CELL_TYPES count does not match CELLS")
    types = np.array(tok[t0 + 2:t0 + 2 + nc], np.int64)
    if not np.isin(types, (5, 7, 9)).all():
        raise ValueError("VTK: unsupported cell type (expected 5, 7 or 9)")
    out.update(xy=pts[:, :2].copy(), cell_ptr=np.asarray(ptr, np.int32),
               cell_nodes=np.concatenate(nodes).astype(np.int32))
    return out


def read_vtk_arcs(path):
    """Only the arc arrays of the dataset-level FIELD block (read up to POINTS)."""
    out, toks = {}, []
    with open(path) as f:
        for line in f:
            t = line.split()
            if t and t[0] == "POINTS":
                break
            toks += t
    if "FIELD" not in toks:
        return out
    i = toks.index("FIELD")
    narr, j = int(toks[i + 2]), i + 3
    for _ in range(narr):
        name, ncomp, ntup = toks[j], int(toks[j + 1]), int(toks[j + 2])
        vals = np.array(toks[j + 4:j + 4 + ncomp * ntup], np.float64).reshape(ntup, ncomp)
        j += 4 + ncomp * ntup
        if name == "arc_nodes":
            out["arc_nodes"] = vals.astype(np.int64)
        elif name == "arc_data":
            out["arc_data"] = vals
    return out
