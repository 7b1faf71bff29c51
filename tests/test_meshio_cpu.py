"""Legacy VTK polygon meshes: the format of the reference reader's VTK path (POINTS / CELLS /
CELL_TYPES 5, 7, 9), with arcs in a FIELD block it skips."""
import numpy as np
import pytest

from vemgpu import meshgen, meshio


def test_round_trip_with_arcs(tmp_path):
    m = meshgen.voronoi_mesh(300, "annulus", seed=7)
    p = tmp_path / "m.vtk"
    meshio.write_vtk(p, m, cell_data={"theta": np.arange(len(m["cell_ptr"]) - 1, dtype=float)})
    r = meshio.read_vtk(p)
    assert np.array_equal(r["xy"], np.asarray(m["xy"]).reshape(-1, 2))
    assert np.array_equal(r["cell_ptr"], m["cell_ptr"]) and np.array_equal(r["cell_nodes"], m["cell_nodes"])
    assert np.array_equal(r["arc_nodes"].reshape(-1), np.asarray(m["arc_nodes"]).reshape(-1))
    assert np.array_equal(r["arc_data"].reshape(-1), np.asarray(m["arc_data"]).reshape(-1))
    a = meshio.read_vtk_arcs(p)
    assert np.array_equal(a["arc_data"], r["arc_data"])


REFERENCE_STYLE = """# vtk DataFile Version 2.0
hanging-node quads
ASCII
DATASET UNSTRUCTURED_GRID
POINTS 6 float
0 0 0  1 0 0  2 0 0
0 1 0  1 1 0  2 1 0
CELLS 2 10
4 0 1 4 3
4 1 2 5 4
CELL_TYPES 2
9
9
"""


def test_reference_style_file(tmp_path):
    p = tmp_path / "q.vtk"
    p.write_text(REFERENCE_STYLE)
    r = meshio.read_vtk(p)
    assert r["xy"].shape == (6, 2) and list(r["cell_ptr"]) == [0, 4, 8]
    assert "arc_nodes" not in meshio.read_vtk_arcs(p)


@pytest.mark.parametrize("bad,msg", [("CELL_TYPES 2\n9\n42\n", "unsupported"), ("CELL_TYPES 3\n9\n9\n9\n", "count")])
def test_rejects_what_the_reference_rejects(tmp_path, bad, msg):
    p = tmp_path / "b.vtk"
    p.write_text(REFERENCE_STYLE.split("CELL_TYPES")[0] + bad)
    with pytest.raises(ValueError, match=msg):
        meshio.read_vtk(p)
    p.write_text(REFERENCE_STYLE.replace("4 1 2 5 4", "4 1 2 5 9"))
    with pytest.raises(ValueError, match="out of range"):
        meshio.read_vtk(p)
