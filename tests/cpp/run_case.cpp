// A C++ caller of the library: the reference's run_case sequence for one Darcy case
// (vem/CurvedVEM_Darcy/main/Darcy_curved_main.cpp:54-92: read the mesh, DarcySolver(mesh, problem,
// nq, ng, k), solve(), computeL2ErrorPressure/Flux) through the header-only facade
// include/vemgpu_darcy.hpp over libvemgpu.so.
//
//     run_case MESH_FILE PROBLEM K NQ TOL
//
// MESH_FILE: "num_nodes num_cells", num_nodes lines "x y", num_cells lines "n v_1 ... v_n".
// Prints one JSON line with the sizes, the solve and the six error figures; exit code 1 and the
// library's message on stderr on failure.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>

#include "vemgpu_darcy.hpp"

int main(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s MESH_FILE PROBLEM K NQ TOL\n", argv[0]);
        return 2;
    }
    try {
        std::ifstream in(argv[1]);
        int nn = 0, nc = 0;
        if (!(in >> nn >> nc) || nn <= 0 || nc <= 0) throw std::runtime_error("cannot read the mesh header");
        vemgpu::PolygonMesh m;
        m.xy.resize(2 * size_t(nn));
        for (auto& v : m.xy)
            if (!(in >> v)) throw std::runtime_error("cannot read a node");
        m.cell_ptr.push_back(0);
        for (int c = 0; c < nc; ++c) {
            int n = 0;
            if (!(in >> n) || n < 3) throw std::runtime_error("cannot read a cell");
            for (int i = 0; i < n; ++i) {
                int v = 0;
                if (!(in >> v)) throw std::runtime_error("cannot read a cell node");
                m.cell_nodes.push_back(v);
            }
            m.cell_ptr.push_back(int(m.cell_nodes.size()));
        }
        const int problem = std::atoi(argv[2]), k = std::atoi(argv[3]), nq = std::atoi(argv[4]);
        const double tol = std::atof(argv[5]);
        vemgpu::DarcySolver solver(m, problem, nq, 9, k);
        solver.solve(tol);
        const auto x = solver.getSolution();
        double xs = 0;
        for (double v : x) xs += v * v;
        std::printf("{\"cells\": %d, \"dofs\": %lld, \"iterations\": %d, \"residual\": %.17g, "
                    "\"scalar_comp\": %.17g, \"flux_comp\": %.17g, \"scalar_phys\": %.17g, \"flux_phys\": %.17g, "
                    "\"div_phys\": %.17g, \"mass\": %.17g, \"solution_norm2\": %.17g}\n",
                    nc, solver.getTotalDofFlux() + solver.getTotalDofConc() + 1, solver.info().iterations,
                    solver.info().residual, solver.computeL2ErrorPressure(nq), solver.computeL2ErrorFlux(nq),
                    solver.physicalError(0), solver.physicalError(1), solver.physicalError(2),
                    solver.physicalError(3), xs);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "run_case: %s\n", e.what());
        return 1;
    }
}
