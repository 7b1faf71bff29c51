// Declarations shared by the setup, error and adjoint kernels.
#pragma once
#include "vg_common.cuh"

namespace vg {

struct SetupArgs {
    // mesh and geometry
    const double* xy;
    const int* cptr;
    const int* cnodes;
    const int* gedges;
    const int* eocc;
    const double* cx;
    const double* cy;
    const double* diam;
    const int* triptr;
    const TriIdx* tris;
    const double* arc;  // 3 per global edge (cx, cy, r), r = 0 for straight edges; null unless arcs
    const int* slot_cell;
    const int* cell_slot;
    const Piece* pieces;
    const int* map;     // signed flux dof map, piece layout
    const double* theta;
    int k, q, p, ngrad, internal, nqp, ng, geom, problem, bc, nf;
    double eps;
    // outputs
    double *A0, *A64;
    float* A32;
    double* W64;
    float* W32;
    double *P, *HW, *L;
    float* L32;
    double *alpha, *rhs, *bval;
    int* mask;
    unsigned long long* status;
};

struct CellGeo {
    int geom;
    double eps;
    const double* arc;
    const int* gedge_base;  // global edge ids of the cell's local edges
};

struct SmemLayout {
    int vert, vol, edge, G, AG, Gi, H, Hi, Hs, Lm, Rh, Ts, Me, Mi, D, W, HW, B, P, AGP, C, per_warp;
};

void upload_rules(const std::vector<double>& tri, const std::vector<double>& gl);
SmemLayout make_layout(int k, int ne, int nqp, int ng);
void launch_setup(const SetupArgs& a, const CellClass& c, int nqp, cudaStream_t s);
// six error figures per cell into per_cell (6 doubles per cell, cell order), x in reference layout
void launch_errors(const SetupArgs& a, const CellClass& c, int nqp, const double* x, double* per_cell, cudaStream_t s);
// deterministic sum of per-cell figures -> out[6] (square roots of the five error figures)
void launch_error_sum(const double* per_cell, int nc, double* out, cudaStream_t s);

}  // namespace vg
