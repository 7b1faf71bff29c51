// C ABI of vemgpu (include/vemgpu.h). Every entry point converts exceptions into status codes;
// no C++ exception crosses the boundary (the rule of vem/CurvedVEM_Darcy_gpu/src/krylov.cu:8-36).
#include <cstring>
#include <memory>
#include <string>

#include "vemgpu.h"
#include "vg_solver.hpp"

struct vg_handle {
    std::unique_ptr<vg::Solver> s;
    std::string error;
};

namespace {
thread_local std::string g_create_error;

// Makes a device current for the duration of a call and gives the caller's current device back
// afterwards: a thread may hold handles on several GPUs, and every handle's buffers, streams and
// kernels belong to the device it was created on.
class DeviceScope {
    int prev_ = -1;
    bool switched_ = false, restore_only_ = false;

public:
    // device < 0: only remember the current device (nothing to restore when there is none)
    explicit DeviceScope(int device) {
        if (device < 0) {
            if (cudaGetDevice(&prev_) == cudaSuccess)
                restore_only_ = true;
            else
                cudaGetLastError();
            return;
        }
        VG_CUDA(cudaGetDevice(&prev_));
        if (device != prev_) {
            VG_CUDA(cudaSetDevice(device));
            switched_ = true;
        }
    }
    ~DeviceScope() {
        if (switched_ || restore_only_) {
            int cur = -1;
            if (cudaGetDevice(&cur) == cudaSuccess && cur != prev_) cudaSetDevice(prev_);
        }
    }
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
};

template <class F>
int guarded(vg_handle* h, F f) {
    if (!h || !h->s) return VG_EINVAL;
    try {
        DeviceScope scope(h->s->device());
        f(*h->s);
        h->error.clear();
        return VG_OK;
    } catch (const vg::Error& e) {
        h->error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        h->error = "host allocation failed";
        return VG_ENOMEM;
    } catch (const std::exception& e) {
        h->error = e.what();
        return VG_EINVAL;
    }
}

int create(vg::HostMesh&& m, const vg_geometry* g, int k, int nq, int ng, int device, vg_handle** out) {
    auto h = std::make_unique<vg_handle>();
    DeviceScope scope(-1);  // the constructor selects `device`; the caller's device comes back after it
    h->s = std::make_unique<vg::Solver>(std::move(m), g, k, nq, ng, device);
    *out = h.release();
    return VG_OK;
}
}  // namespace

extern "C" {

int vg_create(const vg_mesh* mesh, const vg_geometry* geometry, int k, int nq, int ng, int device, vg_handle** out) {
    if (!out) return VG_EINVAL;
    *out = nullptr;
    try {
        if (!mesh) throw vg::Error(VG_EINVAL, "null mesh");
        vg::HostMesh m;
        vg::copy_processed(m, *mesh);
        return create(std::move(m), geometry, k, nq, ng, device, out);
    } catch (const vg::Error& e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return VG_EINVAL;
    }
}

int vg_create_polygons(int num_nodes, const double* node_coords, int num_cells, const int* cell_ptr,
                       const int* cell_nodes, const vg_geometry* geometry, int k, int nq, int ng, int device,
                       vg_handle** out) {
    if (!out) return VG_EINVAL;
    *out = nullptr;
    try {
        vg::HostMesh m;
        vg::PhaseTimer pt;
        vg::process_polygons(m, num_nodes, node_coords, num_cells, cell_ptr, cell_nodes);
        pt.mark("reader post-processing");
        return create(std::move(m), geometry, k, nq, ng, device, out);
    } catch (const vg::Error& e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return VG_EINVAL;
    }
}

int vg_create_vtk(const char* path, const vg_geometry* geometry, int k, int nq, int ng, int device, vg_handle** out) {
    if (!out) return VG_EINVAL;
    *out = nullptr;
    try {
        std::vector<double> xy;
        std::vector<int> ptr, nodes;
        vg::read_vtk_polygons(path, xy, ptr, nodes);
        vg::HostMesh m;
        vg::process_polygons(m, int(xy.size() / 2), xy.data(), int(ptr.size()) - 1, ptr.data(), nodes.data());
        return create(std::move(m), geometry, k, nq, ng, device, out);
    } catch (const vg::Error& e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return VG_EINVAL;
    }
}

int vg_destroy(vg_handle* h) {
    if (h && h->s) {
        try {
            DeviceScope scope(h->s->device());  // the buffers are freed on their own device
            h->s.reset();
        } catch (...) {
            h->s.reset();
        }
    }
    delete h;
    return VG_OK;
}

const char* vg_last_error(const vg_handle* h) { return h ? h->error.c_str() : g_create_error.c_str(); }

int vg_sizes(const vg_handle* h, long long out[9]) {
    if (!h || !h->s || !out) return VG_EINVAL;
    const auto& s = *h->s;
    out[0] = s.m.nc;
    out[1] = s.m.ne;
    out[2] = s.nf;
    out[3] = s.np;
    out[4] = s.N;
    out[5] = s.q;
    out[6] = s.p;
    out[7] = s.internal;
    out[8] = s.maxn;
    return VG_OK;
}

int vg_set_problem(vg_handle* h, int problem, int bc) {
    return guarded(h, [&](vg::Solver& s) { s.set_problem(problem, bc); });
}

int vg_set_log_permeability(vg_handle* h, const double* theta, int on_device) {
    return guarded(h, [&](vg::Solver& s) { s.set_theta(theta, on_device != 0); });
}

int vg_build(vg_handle* h) {
    return guarded(h, [&](vg::Solver& s) { s.build(); });
}

int vg_apply(vg_handle* h, const void* x, void* y, int precision, int constrained, void* stream) {
    return guarded(h, [&](vg::Solver& s) {
        if (!s.built) throw vg::Error(VG_ESTATE, "vg_build must run before vg_apply");
        if (!x || !y || x == y) throw vg::Error(VG_EINVAL, "apply requires distinct non-null vectors");
        s.check_apply_probe();
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const bool internal = (precision & VG_ORDER_INTERNAL) != 0;
        precision &= ~VG_ORDER_INTERNAL;
        if (precision == VG_FP64) {
            VG_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * s.N, st));
            if (internal)
                s.apply_int<double>(static_cast<const double*>(x), static_cast<double*>(y), constrained != 0, 1.0, st,
                                    nullptr);
            else
                s.apply64(static_cast<const double*>(x), static_cast<double*>(y), constrained != 0, 1.0, st);
        } else if (precision == VG_FP32) {
            VG_CUDA(cudaMemsetAsync(y, 0, sizeof(float) * s.N, st));
            if (internal)
                s.apply_int<float>(static_cast<const float*>(x), static_cast<float*>(y), constrained != 0, 1.0f, st,
                                   nullptr);
            else
                s.apply32(static_cast<const float*>(x), static_cast<float*>(y), constrained != 0, 1.0f, st);
        } else {
            throw vg::Error(VG_EINVAL, "precision must be VG_FP64 or VG_FP32");
        }
    });
}

int vg_debug_stall_apply(vg_handle* h) {
    return guarded(h, [&](vg::Solver& s) {
        if (!s.built) throw vg::Error(VG_ESTATE, "vg_build must run before vg_debug_stall_apply");
        s.inject_apply_stall();
    });
}

int vg_permute(vg_handle* h, int to_internal, const void* in, void* out, int precision, void* stream) {
    return guarded(h, [&](vg::Solver& s) {
        if (!s.built) throw vg::Error(VG_ESTATE, "vg_build must run before vg_permute");
        if (!in || !out || in == out) throw vg::Error(VG_EINVAL, "permute requires distinct non-null vectors");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (precision == VG_FP64)
            s.permute<double>(static_cast<const double*>(in), static_cast<double*>(out), to_internal != 0, st);
        else if (precision == VG_FP32)
            s.permute<float>(static_cast<const float*>(in), static_cast<float*>(out), to_internal != 0, st);
        else
            throw vg::Error(VG_EINVAL, "precision must be VG_FP64 or VG_FP32");
    });
}

int vg_rhs(vg_handle* h, double* b) {
    return guarded(h, [&](vg::Solver& s) {
        if (!s.built) throw vg::Error(VG_ESTATE, "vg_build must run before vg_rhs");
        if (!b) throw vg::Error(VG_EINVAL, "null vector");
        s.rhs(b, nullptr);
        VG_CUDA(cudaDeviceSynchronize());
    });
}

void vg_default_solve_opts(vg_solve_opts* o) {
    if (!o) return;
    o->mode = VG_SOLVE_FP64;
    o->tol = 1e-10;
    o->maxit = 200000;
    o->inner_tol = 1e-6;
    o->max_outer = 12;
    o->check_every = 0;
    o->nonzero_guess = 0;
}

int vg_solve(vg_handle* h, const double* b, double* x, const vg_solve_opts* opts, vg_solve_info* info) {
    return guarded(h, [&](vg::Solver& s) {
        vg_solve_opts o;
        vg_default_solve_opts(&o);
        if (opts) o = *opts;
        vg_solve_info inf{};
        try {
            s.solve(b, x, o, inf, nullptr);
        } catch (...) {
            if (info) *info = inf;
            throw;
        }
        if (info) *info = inf;
    });
}

int vg_solve_host(vg_handle* h, const double* b_host, double* x_host, const vg_solve_opts* opts, vg_solve_info* info) {
    return guarded(h, [&](vg::Solver& s) {
        if (!b_host || !x_host) throw vg::Error(VG_EINVAL, "null vector");
        vg_solve_opts o;
        vg_default_solve_opts(&o);
        if (opts) o = *opts;
        vg_solve_info inf{};
        s.solve_host(b_host, x_host, o, inf);
        if (info) *info = inf;
    });
}

int vg_adjoint_grad(vg_handle* h, const double* x, const double* dJdx, double* dJdtheta, const vg_solve_opts* opts,
                    vg_solve_info* info) {
    return guarded(h, [&](vg::Solver& s) {
        if (!x || !dJdx || !dJdtheta) throw vg::Error(VG_EINVAL, "null vector");
        vg_solve_opts o;
        vg_default_solve_opts(&o);
        if (opts) o = *opts;
        vg_solve_info inf{};
        s.adjoint(x, dJdx, dJdtheta, o, inf, nullptr);
        if (info) *info = inf;
    });
}

int vg_errors(vg_handle* h, const double* x, double out[6]) {
    return guarded(h, [&](vg::Solver& s) {
        if (!x || !out) throw vg::Error(VG_EINVAL, "null vector");
        s.errors(x, out, nullptr);
    });
}

int vg_errors_noalloc(vg_handle* h, const double* x, double out[6]) {
    return guarded(h, [&](vg::Solver& s) {
        if (!x || !out) throw vg::Error(VG_EINVAL, "null vector");
        s.errors_static(x, out);
    });
}

int vg_assemble_csr(vg_handle* h, int constrained, long long* nnz, long long* row_ptr, int* col_idx, double* values) {
    return guarded(h, [&](vg::Solver& s) {
        if (!nnz) throw vg::Error(VG_EINVAL, "null nnz");
        s.assemble(constrained, nnz, row_ptr, col_idx, values);
    });
}

int vg_cell_areas(vg_handle* h, double* areas) {
    return guarded(h, [&](vg::Solver& s) {
        if (!areas) throw vg::Error(VG_EINVAL, "null vector");
        s.cell_areas(areas);
    });
}

int vg_ms_configure(vg_handle* h, double d12, double d13, double d23, double dt, long long* state_size) {
    return guarded(h, [&](vg::Solver& s) {
        s.ms_configure(d12, d13, d23, dt);
        if (state_size) *state_size = s.ms_size();
    });
}

int vg_ms_apply(vg_handle* h, const double* coeff_state, const void* x, void* y, int precision) {
    return guarded(h, [&](vg::Solver& s) {
        if (!coeff_state || !x || !y || x == y) throw vg::Error(VG_EINVAL, "null or aliased vector");
        VG_CUDA(cudaDeviceSynchronize());  // inputs may come from any stream
        s.ms_coefficients(coeff_state);
        if (precision == VG_FP64)
            s.ms_apply(static_cast<const double*>(x), static_cast<double*>(y));
        else if (precision == VG_FP32)
            s.ms_apply(static_cast<const float*>(x), static_cast<float*>(y));
        else
            throw vg::Error(VG_EINVAL, "precision must be VG_FP64 or VG_FP32");
        VG_CUDA(cudaDeviceSynchronize());
    });
}

int vg_ms_step(vg_handle* h, const double* old_state, double* new_state, const vg_solve_opts* opts,
               vg_solve_info* info) {
    return guarded(h, [&](vg::Solver& s) {
        if (!old_state || !new_state) throw vg::Error(VG_EINVAL, "null state");
        vg_solve_opts o;
        vg_default_solve_opts(&o);
        if (opts) o = *opts;
        vg_solve_info inf{};
        s.ms_step(old_state, new_state, o, inf);
        if (info) *info = inf;
    });
}

int vg_ms_set_picard(vg_handle* h, int max_iterations, double tol) {
    return guarded(h, [&](vg::Solver& s) { s.ms_set_picard(max_iterations, tol); });
}

int vg_ms_picard_info(const vg_handle* h, int* iterations, double* change, double* nonlinear_residual) {
    if (!h || !h->s) return VG_EINVAL;
    if (iterations) *iterations = h->s->ms_last_picard_;
    if (change) *change = h->s->ms_last_change_;
    if (nonlinear_residual) *nonlinear_residual = h->s->ms_last_nonlinear_;
    return VG_OK;
}

int vg_ms_gs_info(const vg_handle* h, long long* arnoldi_steps, long long* reorthogonalizations) {
    if (!h || !h->s) return VG_EINVAL;
    if (arnoldi_steps) *arnoldi_steps = h->s->ms_arnoldi_steps_;
    if (reorthogonalizations) *reorthogonalizations = h->s->ms_reorth_passes_;
    return VG_OK;
}

int vg_local(vg_handle* h, int cell, int which, double* out, int* count) {
    return guarded(h, [&](vg::Solver& s) {
        int c = s.local(cell, which, out);
        if (count) *count = c;
    });
}

int vg_stats(const vg_handle* h, long long out[4]) {
    if (!h || !h->s || !out) return VG_EINVAL;
    out[0] = h->s->n_launch;
    out[1] = h->s->n_apply;
    out[2] = h->s->n_iter;
    out[3] = h->s->n_solve;
    return VG_OK;
}

}  // extern "C"
