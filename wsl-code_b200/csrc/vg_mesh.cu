// Host mesh processing: the reference reader's post-processing of polygon lists and the per-cell
// triangulation used for volume quadrature.
//
//   process_polygons: vem/CurvedVEM_Darcy_gpu/mesh/straight_mesh.cpp:467-664 (CCW reorder by signed
//     area, centroid = vertex average except the bounding-box centre of 4-gons, area, diameter =
//     largest vertex distance, global edges numbered in (min node, max node) sorted order,
//     occurrence 1 = boundary, 2 = interior).
//   triangulate: ear clipping of vem/CurvedVEM_Darcy_gpu/mesh/polygon_triangulator.cpp:56-150 with
//     its tolerances applied in cell-scaled coordinates ((x - x_D) / h_D), which keeps the reference's
//     choices on its meshes and stays valid on 1e6-cell meshes (the unscaled 1e-6 area tolerance
//     accepts every vertex as "inside" once cell areas fall near 1e-6); cells with an arc edge use
//     the fan of one triangle per edge from the vertex average instead.
#include <algorithm>
#include <cmath>
#include <fstream>
#include <numeric>
#include <string>

#include "vg_solver.hpp"

namespace vg {

// Legacy ASCII VTK polygon mesh, the format of the reference reader's VTK path
// (vem/CurvedVEM_Darcy_gpu/mesh/straight_mesh.cpp:96-218): free-format tokens; POINTS n <type> with
// three coordinates per point (z dropped); CELLS m <total> with a vertex count before each cell's
// vertices; CELL_TYPES m with types 5 (triangle), 7 (polygon) or 9 (quad). Other sections (FIELD,
// CELL_DATA, ...) are skipped. Vertex order is normalised later by process_polygons.
void read_vtk_polygons(const char* path, std::vector<double>& xy, std::vector<int>& ptr, std::vector<int>& nodes) {
    if (!path) throw Error(VG_EINVAL, "null path");
    std::ifstream in(path);
    if (!in) throw Error(VG_EINVAL, std::string("cannot open ") + path);
    auto seek = [&](const char* key) {
        std::string tok;
        while (in >> tok)
            if (tok == key) return true;
        return false;
    };
    if (!seek("POINTS")) throw Error(VG_EMESH, "VTK: POINTS section not found");
    long long nn = 0;
    std::string type;
    if (!(in >> nn >> type) || nn <= 0 || nn > (1LL << 31) - 1) throw Error(VG_EMESH, "VTK: invalid POINTS header");
    xy.assign(2 * size_t(nn), 0.0);
    for (long long i = 0; i < nn; ++i) {
        double x, y, z;
        if (!(in >> x >> y >> z)) throw Error(VG_EMESH, "VTK: failed to read point " + std::to_string(i));
        xy[2 * i] = x;
        xy[2 * i + 1] = y;
    }
    if (!seek("CELLS")) throw Error(VG_EMESH, "VTK: CELLS section not found");
    long long nc = 0, total = 0;
    if (!(in >> nc >> total) || nc <= 0 || nc > (1LL << 31) - 1) throw Error(VG_EMESH, "VTK: invalid CELLS header");
    ptr.assign(1, 0);
    nodes.clear();
    nodes.reserve(size_t(std::max(0LL, total - nc)));
    for (long long e = 0; e < nc; ++e) {
        int nv = 0;
        if (!(in >> nv)) throw Error(VG_EMESH, "VTK: failed to read the vertex count of cell " + std::to_string(e));
        if (nv < 3) throw Error(VG_EMESH, "VTK: cell " + std::to_string(e) + " has fewer than 3 vertices");
        for (int i = 0; i < nv; ++i) {
            long long v = -1;
            if (!(in >> v)) throw Error(VG_EMESH, "VTK: failed to read a vertex of cell " + std::to_string(e));
            if (v < 0 || v >= nn) throw Error(VG_EMESH, "VTK: cell " + std::to_string(e) + " references a node out of range");
            nodes.push_back(int(v));
        }
        ptr.push_back(int(nodes.size()));
    }
    if (!seek("CELL_TYPES")) throw Error(VG_EMESH, "VTK: CELL_TYPES section not found");
    long long nt = 0;
    if (!(in >> nt) || nt != nc) throw Error(VG_EMESH, "VTK: CELL_TYPES count does not match CELLS");
    for (long long e = 0; e < nc; ++e) {
        int t = 0;
        if (!(in >> t)) throw Error(VG_EMESH, "VTK: failed to read cell type " + std::to_string(e));
        if (t != 5 && t != 7 && t != 9)
            throw Error(VG_EMESH, "VTK: cell " + std::to_string(e) + " has unsupported type " + std::to_string(t));
    }
}

void process_polygons(HostMesh& m, int nn, const double* xy, int nc, const int* ptr, const int* nodes) {
    if (nn <= 0 || nc <= 0 || !xy || !ptr || !nodes) throw Error(VG_EINVAL, "empty mesh");
    m.nn = nn;
    m.nc = nc;
    m.xy.assign(xy, xy + 2 * size_t(nn));
    if (ptr[0] != 0) throw Error(VG_EINVAL, "cell_ptr[0] must be 0");
    m.cptr.assign(ptr, ptr + nc + 1);
    m.cnodes.assign(nodes, nodes + ptr[nc]);
    for (int c = 0; c < nc; ++c) {
        int n = ptr[c + 1] - ptr[c];
        if (n < 3) throw Error(VG_EMESH, "cell " + std::to_string(c) + " has fewer than 3 vertices");
        if (n > MAX_NE) throw Error(VG_EMESH, "cell " + std::to_string(c) + " has more than 16 vertices");
        double s = 0;
        for (int i = 0; i < n; ++i) {
            int a = m.cnodes[ptr[c] + i], b = m.cnodes[ptr[c] + (i + 1) % n];
            if (a < 0 || a >= nn || b < 0 || b >= nn) throw Error(VG_EMESH, "node index out of range");
            const double xa = m.xy[2 * a], ya = m.xy[2 * a + 1], xb = m.xy[2 * b], yb = m.xy[2 * b + 1];
            if (!std::isfinite(xa) || !std::isfinite(ya))
                throw Error(VG_EMESH, "cell " + std::to_string(c) + " has a non-finite node coordinate");
            if (a == b || (xa == xb && ya == yb))
                throw Error(VG_EMESH, "cell " + std::to_string(c) + " has a zero-length edge");
            s += xa * yb - xb * ya;
        }
        // the reference rejects cells without positive size (vem/CurvedVEM_Darcy_gpu/src/mesh_pack.cpp:77-78)
        if (!(std::fabs(s) > 0)) throw Error(VG_EMESH, "degenerate element: cell " + std::to_string(c) + " has zero area");
        if (s < 0) std::reverse(m.cnodes.begin() + ptr[c], m.cnodes.begin() + ptr[c + 1]);
    }
    m.cx.assign(nc, 0);
    m.cy.assign(nc, 0);
    m.diam.assign(nc, 0);
    for (int c = 0; c < nc; ++c) {
        int b = m.cptr[c], n = m.cptr[c + 1] - b;
        double x[MAX_NE], y[MAX_NE];
        for (int i = 0; i < n; ++i) {
            x[i] = m.xy[2 * m.cnodes[b + i]];
            y[i] = m.xy[2 * m.cnodes[b + i] + 1];
        }
        if (n == 4) {
            double x0 = *std::min_element(x, x + 4), x1 = *std::max_element(x, x + 4);
            double y0 = *std::min_element(y, y + 4), y1 = *std::max_element(y, y + 4);
            m.cx[c] = (x0 + x1) / 2.0;
            m.cy[c] = (y0 + y1) / 2.0;
        } else {
            double sx = 0, sy = 0;
            for (int i = 0; i < n; ++i) {
                sx += x[i];
                sy += y[i];
            }
            m.cx[c] = sx / n;
            m.cy[c] = sy / n;
        }
        double d = 0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) d = std::max(d, std::sqrt((x[i] - x[j]) * (x[i] - x[j]) + (y[i] - y[j]) * (y[i] - y[j])));
        m.diam[c] = d;
    }
    // global edges: stable sort of (min, max) keys
    size_t tot = m.cnodes.size();
    std::vector<unsigned long long> key(tot);
    std::vector<int> order(tot);
    for (int c = 0; c < nc; ++c) {
        int b = m.cptr[c], n = m.cptr[c + 1] - b;
        for (int j = 0; j < n; ++j) {
            unsigned a = unsigned(m.cnodes[b + j]), e = unsigned(m.cnodes[b + (j + 1) % n]);
            key[b + j] = (static_cast<unsigned long long>(std::min(a, e)) << 32) | std::max(a, e);
        }
    }
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b] || (key[a] == key[b] && a < b); });
    m.gedges.assign(tot, -1);
    m.eend.clear();
    int count = 0;
    for (size_t i = 0; i < tot; ++i) {
        if (i == 0 || key[order[i]] != key[order[i - 1]]) {
            m.eend.push_back(int(key[order[i]] >> 32));
            m.eend.push_back(int(key[order[i]] & 0xffffffffull));
            ++count;
        }
        m.gedges[order[i]] = count - 1;
    }
    m.ne = count;
    m.eocc.assign(count, 0);
    for (int e : m.gedges) m.eocc[e]++;
    for (int e = 0; e < count; ++e)
        if (m.eocc[e] > 2) throw Error(VG_EMESH, "edge shared by more than two cells");
}

void copy_processed(HostMesh& m, const vg_mesh& in) {
    if (in.num_nodes <= 0 || in.num_cells <= 0 || in.num_edges <= 0 || !in.node_coords || !in.cell_nodes ||
        !in.cell_node_indices || !in.global_edges || !in.edge_endpoints || !in.edge_occurrence ||
        !in.cell_centroid_x || !in.cell_centroid_y || !in.cell_diameter)
        throw Error(VG_EINVAL, "incomplete vg_mesh");
    m.nn = in.num_nodes;
    m.nc = in.num_cells;
    m.ne = in.num_edges;
    m.xy.assign(in.node_coords, in.node_coords + 2 * size_t(m.nn));
    m.cptr.assign(in.cell_node_indices, in.cell_node_indices + m.nc + 1);
    m.cnodes.assign(in.cell_nodes, in.cell_nodes + m.cptr[m.nc]);
    if (in.cell_edge_indices)
        for (int c = 0; c <= m.nc; ++c)
            if (in.cell_edge_indices[c] != m.cptr[c]) throw Error(VG_EINVAL, "cell_edge_indices differ from cell_node_indices");
    m.gedges.assign(in.global_edges, in.global_edges + m.cptr[m.nc]);
    m.eend.assign(in.edge_endpoints, in.edge_endpoints + 2 * size_t(m.ne));
    m.eocc.assign(in.edge_occurrence, in.edge_occurrence + m.ne);
    m.cx.assign(in.cell_centroid_x, in.cell_centroid_x + m.nc);
    m.cy.assign(in.cell_centroid_y, in.cell_centroid_y + m.nc);
    m.diam.assign(in.cell_diameter, in.cell_diameter + m.nc);
    for (int c = 0; c < m.nc; ++c) {
        int n = m.cptr[c + 1] - m.cptr[c];
        if (n < 3 || n > MAX_NE) throw Error(VG_EMESH, "cell " + std::to_string(c) + " has an unsupported edge count");
        if (in.nodes_per_cell && in.nodes_per_cell[c] != n) throw Error(VG_EINVAL, "nodes_per_cell inconsistent");
        for (int j = 0; j < n; ++j) {
            int e = m.gedges[m.cptr[c] + j];
            if (e < 0 || e >= m.ne) throw Error(VG_EMESH, "global edge out of range");
            int a = m.cnodes[m.cptr[c] + j], b = m.cnodes[m.cptr[c] + (j + 1) % n];
            if (std::min(a, b) != m.eend[2 * e] || std::max(a, b) != m.eend[2 * e + 1])
                throw Error(VG_EMESH, "edge endpoints do not match the cell's nodes");
        }
    }
    for (int e = 0; e < m.ne; ++e)
        if (m.eocc[e] < 1 || m.eocc[e] > 2) throw Error(VG_EMESH, "edge occurrence must be 1 or 2");
}

namespace {

void ear_clip(const double* x, const double* y, int n, double cx, double cy, double h, std::vector<TriIdx>& out) {
    int idx[MAX_NE];
    double u[MAX_NE], v[MAX_NE];
    for (int i = 0; i < n; ++i) {
        idx[i] = i;
        u[i] = (x[i] - cx) / h;
        v[i] = (y[i] - cy) / h;
    }
    auto inside = [&](int p, int a, int b, int c) {
        double t = 0.5 * std::fabs((u[b] - u[a]) * (v[c] - v[a]) - (u[c] - u[a]) * (v[b] - v[a]));
        double a1 = 0.5 * std::fabs((u[a] - u[p]) * (v[b] - v[p]) - (u[b] - u[p]) * (v[a] - v[p]));
        double a2 = 0.5 * std::fabs((u[b] - u[p]) * (v[c] - v[p]) - (u[c] - u[p]) * (v[b] - v[p]));
        double a3 = 0.5 * std::fabs((u[c] - u[p]) * (v[a] - v[p]) - (u[a] - u[p]) * (v[c] - v[p]));
        return std::fabs((a1 + a2 + a3) - t) < 1e-6;
    };
    int r = n;
    while (r > 3) {
        bool found = false;
        for (int i = 0; i < r && !found; ++i) {
            int pv = idx[(i - 1 + r) % r], cu = idx[i], nx = idx[(i + 1) % r];
            double cross = (u[nx] - u[cu]) * (v[pv] - v[cu]) - (u[pv] - u[cu]) * (v[nx] - v[cu]);
            if (cross <= 1e-8) continue;
            bool ear = true;
            for (int j = 0; j < r && ear; ++j) {
                int q = idx[j];
                if (q != pv && q != cu && q != nx && inside(q, pv, cu, nx)) ear = false;
            }
            if (!ear) continue;
            out.push_back(TriIdx{uint8_t(pv), uint8_t(cu), uint8_t(nx), NO_ARC});
            for (int j = i; j < r - 1; ++j) idx[j] = idx[j + 1];
            --r;
            found = true;
        }
        if (!found) throw Error(VG_EMESH, "no valid ear found for polygon");
    }
    out.push_back(TriIdx{uint8_t(idx[0]), uint8_t(idx[1]), uint8_t(idx[2]), NO_ARC});
}

}  // namespace

void triangulate(const HostMesh& m, const std::vector<char>& cell_curved, const std::vector<int>& edge_arc,
                 std::vector<int>& triptr, std::vector<TriIdx>& tris) {
    triptr.assign(m.nc + 1, 0);
    tris.clear();
    tris.reserve(size_t(m.nc) * 6);
    double x[MAX_NE], y[MAX_NE];
    for (int c = 0; c < m.nc; ++c) {
        int b = m.cptr[c], n = m.cptr[c + 1] - b;
        if (cell_curved[c]) {
            for (int j = 0; j < n; ++j)
                tris.push_back(TriIdx{APEX, uint8_t(j), uint8_t((j + 1) % n),
                                      edge_arc[m.gedges[b + j]] >= 0 ? uint8_t(j) : NO_ARC});
        } else {
            for (int i = 0; i < n; ++i) {
                x[i] = m.xy[2 * m.cnodes[b + i]];
                y[i] = m.xy[2 * m.cnodes[b + i] + 1];
            }
            try {
                ear_clip(x, y, n, m.cx[c], m.cy[c], m.diam[c], tris);
            } catch (const Error& e) {
                throw Error(e.code, std::string(e.what()) + " (cell " + std::to_string(c) + ")");
            }
        }
        triptr[c + 1] = int(tris.size());
    }
}

}  // namespace vg
