// Internal C++ object behind the vemgpu C ABI (one per vg_handle).
//
// Host side: the processed mesh (the reference reader's StraightMeshData), per-cell
// triangulations, the degree-of-freedom map with orientation signs and the edge-count buckets
// (the reference's HostMesh, vem/CurvedVEM_Darcy_gpu/src/mesh_pack.cpp:127-238, without the
// per-point samples: quadrature points are generated on the device).
// Device side: FP64 setup outputs in bucket-slot-major layout (coalesced for one thread per
// cell), FP64 and FP32 copies of the packed local operators, Krylov workspaces.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "vg_common.cuh"
#include "vg_amg.hpp"
#include "vg_apply.cuh"
#include "vg_krylov.cuh"
#include "vg_setup.cuh"

namespace vg {

struct HostMesh {
    int nn = 0, nc = 0, ne = 0;
    std::vector<double> xy;
    std::vector<int> cptr, cnodes, gedges, eend, eocc;
    std::vector<double> cx, cy, diam;
};

// reader post-processing of raw polygons (straight_mesh.cpp:467-664)
void process_polygons(HostMesh& m, int nn, const double* xy, int nc, const int* ptr, const int* nodes);
// legacy ASCII VTK polygon file (POINTS / CELLS / CELL_TYPES) -> raw polygons
void read_vtk_polygons(const char* path, std::vector<double>& xy, std::vector<int>& ptr, std::vector<int>& nodes);
// copy and validate an already processed mesh
void copy_processed(HostMesh& m, const vg_mesh& in);
// triangulation: reference ear clipping (decisions in cell-scaled coordinates) or, for cells with
// an arc edge, the fan from the vertex average
void triangulate(const HostMesh& m, const std::vector<char>& cell_curved, const std::vector<int>& edge_arc,
                 std::vector<int>& triptr, std::vector<TriIdx>& tris);

class Solver {
public:
    Solver(HostMesh&& mesh, const vg_geometry* geo, int k, int nq, int ng, int device);
    ~Solver();

    // configuration
    void set_problem(int problem, int bc);
    void set_theta(const double* theta, bool on_device);
    void build();

    // operator: y = K x (reference sign when psign = +1, symmetric when psign = -1)
    void apply64(const double* x, double* y, bool constrained, double psign, cudaStream_t s, double* quad = nullptr);
    void apply32(const float* x, float* y, bool constrained, float psign, cudaStream_t s, double* quad = nullptr);
    void rhs(double* b, cudaStream_t s);
    void solve(const double* b, double* x, const vg_solve_opts& o, vg_solve_info& info, cudaStream_t s);
    // host buffers in and out (pinned or pageable); device copies kept across calls
    void solve_host(const double* b_host, double* x_host, const vg_solve_opts& o, vg_solve_info& info);
    void adjoint(const double* x, const double* dJdx, double* g, const vg_solve_opts& o, vg_solve_info& info,
                 cudaStream_t s);
    void errors(const double* x, double out[6], cudaStream_t s);
    // same figures with the per-cell scratch in a static device array (no device allocation)
    void errors_static(const double* x, double out[6]);
    int local(int cell, int which, double* out);
    // Maxwell-Stefan (k = 0, no-flux boundary): state [J1 (nf), J2 (nf), x1 (nc), x2 (nc)]
    void ms_configure(double d12, double d13, double d23, double dt);
    void ms_step(const double* old_state, double* new_state, const vg_solve_opts& o, vg_solve_info& info);
    void ms_coefficients(const double* state);
    template <typename T>
    void ms_apply(const T* x, T* y);
    long long ms_size() const { return ms_.N; }
    void ms_set_picard(int max_iterations, double tol);
    int ms_last_picard_ = 0;
    double ms_last_change_ = 0, ms_last_nonlinear_ = 0;
    long long ms_arnoldi_steps_ = 0, ms_reorth_passes_ = 0;  // GMRES Arnoldi steps, second Gram-Schmidt passes
    int device() const { return device_; }  // the CUDA device that holds this handle's data
    // failure-path test hook and the asynchronous error report of vg_apply
    void inject_apply_stall();
    void check_apply_probe();
    void cell_areas(double* out);
    // assembled CSR of the system (comparator of the matrix-free apply); rp == nullptr: size only
    void assemble(int constrained, long long* nnz, long long* rp, int* ci, double* val);

    // sizes
    int k, nq, ng, q, p, ngrad, internal, nf, np, N, maxn;
    int problem = VG_PROBLEM_SINCOS, bc = VG_BC_FLUX;
    bool built = false;
    long long n_launch = 0, n_apply = 0, n_iter = 0, n_solve = 0;
    bool use_amg = false;
    int amg_levels = 0;
    double amg_setup_s = 0;
    std::string error;

    HostMesh m;
    int geom_kind = VG_GEOM_IDENTITY;
    double eps = 0;

private:
    void pack_layout();
    void plan_internal_order();
    std::vector<int> pressure_order() const;
    void internal_copies();  // L, mask (after the setup) in the internal order
public:
    // y = K x with x, y in the internal order (y's flux entries zero on entry)
    template <typename T>
    void apply_int(const T* x, T* y, bool constrained, T psign, cudaStream_t s, double* quad);
private:
    void plan_streams();
    void pack_streams(cudaStream_t s);
    void prepare_reference_order();
    void pack_streams_reference(cudaStream_t s);
    template <typename T>
    void apply_ref(const T* x, T* y, bool constrained, T psign, cudaStream_t s, double* quad);
    DevBuf<int> d_prow_ref_;                // per slot: first pressure row in the reference order
    DevBuf<unsigned char> d_rec64r_, d_rec32r_;  // record streams with the reference-order map
    bool ref_streams_packed_ = false;
    void check_pipeline();
    void make_diagonal(cudaStream_t s);
    void lift_flux_rhs();
    void build_amg();
    void build_amg_high();
    void prepare_amg_refresh();
    void refresh_amg();
    bool amg_refreshable_ = false;
    DevBuf<int> d_inc_ptr_, d_inc_cell_, d_inc_i_, d_rank_cell_, d_cell_rank_;
    DevBuf<signed char> d_inc_s_;
    DevBuf<double> d_schur_vals_;
    template <typename T>
    void ms_precond(const T* r, T* z);
    template <typename T>
    void ms_norm2(const T* x, double* dst);
    template <typename T>
    double ms_norm(const T* x);
    template <typename T>
    void ms_arnoldi_step(cudaGraphConditionalHandle cond);
    template <typename T>
    void ms_build_graph(int p);
    void ms_destroy_graphs();
    template <typename T>
    int ms_gmres(const T* r, T* d, double tol, int maxit, int mres, double* rel);
    struct MsState {
        bool ready = false;
        double i12 = 0, i13 = 0, i23 = 0, dt = 0;
        long long N = 0;
        DevBuf<double> B64, F64, C64, D, m64, V64, b, r, y, d, t64, w64, vn64, partials, kry;
        DevBuf<double> prev;  // Picard: the iterate the friction matrix was taken at
        DevBuf<float> B32, F32, C32, m32, A32, V32, r32, d32, t32, w32, vn32;
        DevBuf<unsigned int> counter;
        long long ld = 0, chunk = 0;  // Krylov basis column stride; rows per dot-product block
        int dblocks = 0;
        cudaGraph_t graph[2] = {nullptr, nullptr};  // captured Arnoldi loops (FP64, FP32)
        cudaGraphExec_t gexec[2] = {nullptr, nullptr};
        // per-species multigrid of the pressure Schur block, built from the first state stepped
        // after vg_ms_configure and kept for the following steps
        Amg amg[2];
        bool amg_ready = false;
    } ms_;
    bool ms_large_ = false;
    int ms_picard_max_ = 1;
    double ms_picard_tol_ = 1e-10;  // pieces of polygons outside 3..9 edges (second apply kernel)
    void ms_build_amg();
    void assembled_pattern();
    std::vector<long long> csr_ptr_;  // assembled pattern (host, built on first request)
    std::vector<int> csr_col_;
    void check_status(const char* where);
    void axpy64(double* x, const double* d, double a, cudaStream_t s);
    void minres(bool fp32, const void* b, void* x, double tol, int maxit, int check_every, int& iters,
                cudaStream_t s);
    template <typename T>
    void minres_t(const T* r, T* x, double tol, int maxit, int check_every, int& iters, cudaStream_t s);
    template <typename T>
    MinresVecs<T> vecs(T* x);
    template <typename T>
    ApplyArgs<T> apply_args(const T* x, T* y, bool constrained, T psign, double* quad, const int* flags);
    template <typename T>
    void iteration(MinresVecs<T>& v, cudaStream_t s);
    template <typename T>
    void build_graph(int p, T* x);
    void destroy_graphs();

    int device_ = 0;
    std::vector<Piece> pieces_;
    std::vector<int> slot_cell_;   // slot -> cell (-1 on padding lanes)
    std::vector<int> cell_slot_;   // cell -> slot
    std::vector<int> map_host_;    // signed flux dof map, piece layout (~g for negative orientation)
    std::vector<CellClass> classes_;
    std::vector<DevBuf<int>> class_cells_;
    std::vector<double> theta_;
    long long a_total_ = 0, w_total_ = 0, map_total_ = 0, p_total_ = 0, hw_total_ = 0;

    // mesh / geometry on the device
    DevBuf<double> d_xy_, d_cx_, d_cy_, d_diam_, d_arc_;
    DevBuf<int> d_cptr_, d_cnodes_, d_gedges_, d_eocc_, d_triptr_, d_slot_cell_, d_cell_slot_;
    DevBuf<Piece> d_pieces_;
    DevBuf<TriIdx> d_tris_;
    // setup outputs
    DevBuf<double> d_A0_, d_A64_, d_W64_, d_P_, d_HW_, d_L_, d_alpha_, d_theta_, d_rhs_, d_bval_;
    DevBuf<float> d_A32_, d_W32_, d_L32_;
    DevBuf<int> d_map_, d_mask_;
    DevBuf<unsigned long long> d_status_;
    // preconditioner (inverse diagonal of the block-diagonal SPD preconditioner)
    DevBuf<double> d_dinv64_;
    DevBuf<float> d_dinv32_;
    // reductions
    DevBuf<double> d_partials_;
    DevBuf<unsigned int> d_counter_;
    DevBuf<double> d_red_;
    // Krylov workspaces
    DevBuf<double> w64_[8];
    DevBuf<float> w32_[8];
    DevBuf<double> d_scal_;
    DevBuf<int> d_flags_;
    SetupArgs setup_args_{};
    Amg amg_;
    // solve workspaces (fixed addresses: the MINRES loop is a CUDA graph)
    DevBuf<double> sv64_[4];
    DevBuf<float> sv32_[2];
    DevBuf<int> d_loop_;
    cudaStream_t stream_ = nullptr;
    cudaStream_t side_ = nullptr;  // second branch of a MINRES iteration (flux rows of the update)
    cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
    cudaEvent_t ev_in_ = nullptr;
    cudaGraph_t graph_[2] = {nullptr, nullptr};
    cudaGraphExec_t gexec_[2] = {nullptr, nullptr};
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    // record streams of the bulk-copy apply (k <= 1), one per precision
    int sm_count_ = 0;
    StreamPlan plan64_, plan32_;
    DevBuf<unsigned char> d_rec64_, d_rec32_;
    DevBuf<long long> d_roff64_, d_roff32_;
    DevBuf<ApplyBatch> d_bat64_, d_bat32_;
    DevBuf<int> d_cta64_, d_cta32_;
    int* h_err_ = nullptr;   // the apply's error word (mapped pinned host memory) ...
    int* d_errp_ = nullptr;  // ... and its device address
    DevBuf<int> d_stall_;    // test hook of the streamed apply (zero in every normal run)
    DevBuf<double> d_hb_, d_hx_;  // device copies of the host-buffer solve
    DevBuf<double> d_rhs0_;       // right-hand side before the essential-BC lift
    DevBuf<double> d_adj_rhs_, d_adj_mu_;  // adjoint right-hand side and solution
    // internal order of the solver's vectors: flux dofs numbered by first touch in piece order (the
    // dofs a cell owns are consecutive across the lanes of its piece), pressure rows in slot order;
    // the public entry points keep the reference's order and permute at the boundary
    std::vector<int> map_int_host_, prow_host_, e2i_host_, i2e_host_;
    DevBuf<int> d_map_int_, d_prow_, d_e2i_, d_i2e_, d_mask_int_;
    DevBuf<double> d_Lint_, d_pdinv64_, d_xi_;
    DevBuf<float> d_Lint32_, d_pdinv32_;
public:
    // x (N) to or from the internal order
    template <typename T>
    void permute(const T* in, T* out, bool to_internal, cudaStream_t s);
private:
};

}  // namespace vg
