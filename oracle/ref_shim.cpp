// ORACLE PIN — test infrastructure only.
//
// A thin extern "C" shim over the reference's own PETSc-free CPU modules, compiled from their
// sources in place (see oracle/Makefile, target ref) into oracle/_ref/libvemref.so. It lets the
// CPU tests check the oracle's restated building blocks against the reference code itself:
//   vem/CurvedVEM_Darcy_gpu/mesh/straight_mesh.cpp      StraightMeshReader::read_mesh / read_mesh_vtk
//   vem/CurvedVEM_Darcy_gpu/mesh/polygon_triangulator.cpp PolygonTriangulator::triangulateElement
//   vem/CurvedVEM_Darcy_gpu/core/gauss_quadrature.cpp   get_triangle_points / get_line_2D_points
//   vem/CurvedVEM_Darcy_gpu/lib/polynomial_basis.cpp    evalMonomial2D / evalHdivBasis / getEdgeBasisCoeffs
//   vem/CurvedVEM_Darcy_gpu/examples/darcy_problem.cpp  DarcyProblem pull-backs (examples 1 and 2)
#include "mesh/straight_mesh.h"
#include "mesh/polygon_triangulator.h"
#include "core/gauss_quadrature.h"
#include "lib/polynomial_basis.h"
#include "examples/darcy_problem.h"

#include <algorithm>
#include <cstring>
#include <memory>

extern "C" {

void* ref_read_mesh(const char* path, int vtk) {
    auto* r = new vem::StraightMeshReader();
    bool ok = vtk ? r->read_mesh_vtk(path) : r->read_mesh(path);
    if (!ok) {
        delete r;
        return nullptr;
    }
    return r;
}

void ref_free_mesh(void* h) { delete static_cast<vem::StraightMeshReader*>(h); }

// nn, nc, ne, total cell nodes
void ref_mesh_sizes(void* h, int* out) {
    const auto& m = static_cast<vem::StraightMeshReader*>(h)->get_mesh_data();
    out[0] = m.num_nodes;
    out[1] = m.num_cells;
    out[2] = m.num_edges;
    out[3] = int(m.cell_nodes.size());
}

void ref_mesh_arrays(void* h, double* xy, int* cell_nodes, int* cell_node_indices, int* global_edges,
                     int* edge_endpoints, int* edge_occurrence, double* cx, double* cy, double* area, double* diam) {
    const auto& m = static_cast<vem::StraightMeshReader*>(h)->get_mesh_data();
    std::copy(m.node_coords.begin(), m.node_coords.end(), xy);
    std::copy(m.cell_nodes.begin(), m.cell_nodes.end(), cell_nodes);
    std::copy(m.cell_node_indices.begin(), m.cell_node_indices.end(), cell_node_indices);
    std::copy(m.global_edges.begin(), m.global_edges.end(), global_edges);
    std::copy(m.edge_endpoints.begin(), m.edge_endpoints.end(), edge_endpoints);
    std::copy(m.edge_occurrence.begin(), m.edge_occurrence.end(), edge_occurrence);
    std::copy(m.cell_centroid_x.begin(), m.cell_centroid_x.end(), cx);
    std::copy(m.cell_centroid_y.begin(), m.cell_centroid_y.end(), cy);
    std::copy(m.cell_area.begin(), m.cell_area.end(), area);
    std::copy(m.cell_diameter.begin(), m.cell_diameter.end(), diam);
}

// triangles of one cell: 6 doubles each; returns the count
int ref_triangulate(void* h, int cell, double* out) {
    const auto& m = static_cast<vem::StraightMeshReader*>(h)->get_mesh_data();
    vem::PolygonTriangulator t;
    auto e = t.triangulateElement(m, cell);
    for (size_t i = 0; i < e.triangles.size(); ++i)
        for (int j = 0; j < 6; ++j) out[6 * i + j] = e.triangles[i].vertices[j];
    return int(e.triangles.size());
}

// quadrature on one triangle: (x, y, w) triples; returns the count
int ref_triangle_points(const double* v, int n, double* out) {
    vem::GaussQuadrature q;
    auto pts = q.get_triangle_points(std::vector<double>(v, v + 6), n);
    for (size_t i = 0; i < pts.size(); ++i) {
        out[3 * i] = pts[i].x[0];
        out[3 * i + 1] = pts[i].x[1];
        out[3 * i + 2] = pts[i].w;
    }
    return int(pts.size());
}

int ref_line_points(int order, double x1, double y1, double x2, double y2, double* out) {
    vem::GaussQuadrature q;
    auto pts = q.get_line_2D_points(vem::QuadratureType::GAUSS_LEGENDRE, order, x1, y1, x2, y2);
    for (size_t i = 0; i < pts.size(); ++i) {
        out[3 * i] = pts[i].x[0];
        out[3 * i + 1] = pts[i].x[1];
        out[3 * i + 2] = pts[i].w;
    }
    return int(pts.size());
}

double ref_mono(int k, int idx, double xd, double yd, double hd, double x, double y) {
    vem::basis::BasisFunctionPloy b(k);
    return b.evalMonomial2D(idx, vem::basis::Point2D(xd, yd), hd, vem::basis::Point2D(x, y));
}

void ref_hdiv(int k, int idx, double xd, double yd, double hd, double x, double y, double* out) {
    vem::basis::BasisFunctionPloy b(k);
    auto v = b.evalHdivBasis(idx, vem::basis::Point2D(xd, yd), hd, vem::basis::Point2D(x, y));
    out[0] = v.x;
    out[1] = v.y;
}

void ref_edge_coeffs(int k, int idx, double xd, double yd, double hd, double x0, double y0, double x1, double y1,
                     double* out) {
    vem::basis::BasisFunctionPloy b(k);
    std::vector<double> c;
    b.getEdgeBasisCoeffs(idx, vem::basis::Point2D(xd, yd), hd, vem::basis::Point2D(x0, y0),
                         vem::basis::Point2D(x1, y1), c);
    std::copy(c.begin(), c.end(), out);
}

// Darcy example data at a computational point: p, u_hat (2), g_hat, X, Y, J (4), det
void ref_darcy(int example, double xi, double eta, double* out) {
    Darcy::DarcyProblem p;
    p.set_problem_index(example);
    p.init_problem();
    auto u = p.computational_solution_u(xi, eta);
    auto X = p.get_mapping().physical_coords(xi, eta);
    auto J = p.get_mapping().jacobian(xi, eta);
    out[0] = p.computational_solution_p(xi, eta);
    out[1] = u.x;
    out[2] = u.y;
    out[3] = p.computational_source_g(xi, eta);
    out[4] = X.x;
    out[5] = X.y;
    out[6] = J.xx;
    out[7] = J.xy;
    out[8] = J.yx;
    out[9] = J.yy;
    out[10] = p.get_mapping().jacobian_det(xi, eta);
}

}  // extern "C"
