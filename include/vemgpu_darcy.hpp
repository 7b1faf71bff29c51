/* vemgpu — C++ facade with the call sequence of the reference's CPU class DarcySolver
 * (vem/CurvedVEM_Darcy/solver/DarcySolver.h:17-126, used as in
 * vem/CurvedVEM_Darcy/main/Darcy_curved_main.cpp:54-92):
 *
 *     vemgpu::DarcySolver solver(mesh, problem_index, gauss_point_num, gauss_point_num_1d, k);
 *     solver.solve();
 *     double ep = solver.computeL2ErrorPressure(gauss_point_num);
 *     double eu = solver.computeL2ErrorFlux(gauss_point_num);
 *     std::vector<double> x = solver.getSolution();
 *
 * Header-only, over the C ABI of include/vemgpu.h (link -lvemgpu and the CUDA runtime for the
 * device vectors). The mesh is the raw polygon list of the reference reader's input (node
 * coordinates, cell node lists in any orientation); the library does the reader's
 * post-processing. problem_index is the reference's Darcy example: 1 = sine-perturbed map
 * eps = 0.05, 2 = identity map, both p = sin(pi x) cos(pi y), K = I, essential normal-flux
 * boundary condition with the zero-mean pressure multiplier. Errors are thrown as
 * std::runtime_error with the library's message (the reference throws the same way).
 */
#ifndef VEMGPU_DARCY_HPP
#define VEMGPU_DARCY_HPP

#include <cuda_runtime_api.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "vemgpu.h"

namespace vemgpu {

struct PolygonMesh {
    std::vector<double> xy;        // 2 * num_nodes
    std::vector<int> cell_ptr;     // num_cells + 1
    std::vector<int> cell_nodes;   // cell_ptr[num_cells]
};

class DarcySolver {
public:
    DarcySolver(const PolygonMesh& mesh, int problem_index, int gauss_point_num = 9, int gauss_point_num_1d = 9,
                int k = 1) {
        if (problem_index != 1 && problem_index != 2) throw std::runtime_error("Darcy example must be 1 or 2");
        vg_geometry g{};
        g.kind = problem_index == 1 ? VG_GEOM_SINE : VG_GEOM_IDENTITY;
        g.eps = problem_index == 1 ? 0.05 : 0.0;
        const int nn = int(mesh.xy.size() / 2), nc = int(mesh.cell_ptr.size()) - 1;
        if (vg_create_polygons(nn, mesh.xy.data(), nc, mesh.cell_ptr.data(), mesh.cell_nodes.data(), &g, k,
                               gauss_point_num, gauss_point_num_1d, -1, &h_))
            throw std::runtime_error(vg_last_error(nullptr));
        check(vg_set_problem(h_, VG_PROBLEM_SINCOS, VG_BC_FLUX));
        check(vg_build(h_));
        check(vg_sizes(h_, sizes_));
    }
    ~DarcySolver() {
        if (x_) cudaFree(x_);
        if (b_) cudaFree(b_);
        if (h_) vg_destroy(h_);
    }
    DarcySolver(const DarcySolver&) = delete;
    DarcySolver& operator=(const DarcySolver&) = delete;

    long long getTotalDofFlux() const { return sizes_[2]; }
    long long getTotalDofConc() const { return sizes_[3]; }

    // the reference's solve(): assemble, solve to the true relative residual tol, keep the solution
    bool solve(double tol = 1e-10) {
        const size_t bytes = sizeof(double) * static_cast<size_t>(sizes_[4]);
        if (!b_ && cudaMalloc(reinterpret_cast<void**>(&b_), bytes) != cudaSuccess)
            throw std::runtime_error("cudaMalloc failed");
        if (!x_ && cudaMalloc(reinterpret_cast<void**>(&x_), bytes) != cudaSuccess)
            throw std::runtime_error("cudaMalloc failed");
        check(vg_rhs(h_, b_));
        vg_solve_opts o;
        vg_default_solve_opts(&o);
        o.tol = tol;
        check(vg_solve(h_, b_, x_, &o, &info_));
        check(vg_errors(h_, x_, err_));
        solved_ = true;
        return true;
    }
    double computeL2ErrorPressure(int = 9) const { return figure(0); }
    double computeL2ErrorFlux(int = 9) const { return figure(1); }
    // physical-domain figures of the GPU project's report: 0 scalar, 1 flux, 2 divergence, 3 mass
    double physicalError(int i) const { return figure(2 + i); }
    const vg_solve_info& info() const { return info_; }
    std::vector<double> getSolution() const {
        std::vector<double> x(static_cast<size_t>(sizes_[4]));
        if (solved_ && cudaMemcpy(x.data(), x_, sizeof(double) * x.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("cudaMemcpy failed");
        return x;
    }

private:
    void check(int code) const {
        if (code != VG_OK) throw std::runtime_error(vg_last_error(h_));
    }
    double figure(int i) const {
        if (!solved_) throw std::runtime_error("error requires a completed numerical solution");
        return err_[i];
    }
    vg_handle* h_ = nullptr;
    long long sizes_[9] = {};
    double *b_ = nullptr, *x_ = nullptr;
    double err_[6] = {};
    vg_solve_info info_{};
    bool solved_ = false;
};

}  // namespace vemgpu

#endif /* VEMGPU_DARCY_HPP */
