/* vemgpu — B200-native matrix-free curved mixed-VEM Darcy solver, C ABI.
 *
 * Drop-in boundary for the reference call sequence of vem/CurvedVEM_Darcy_gpu:
 *   StraightMeshReader -> DarcyGpu(reader, problem, example, k, nq, ng) (HdivGpu + MixedGpu setup)
 *   -> MixedGpu::update / make_rhs -> Krylov::solve -> MixedGpu::errors
 * and of the CPU class vem/CurvedVEM_Darcy/solver/DarcySolver.h:17-126
 * (DarcySolver(mesh, problem, nq, ng, k); solve(); computeL2ErrorPressure/Flux; getSolution()).
 *
 * Conventions (same as the reference GPU project, vem/CurvedVEM_Darcy_gpu/include/equation_gpu.cuh:1-5):
 *   - every vector argument of vg_apply / vg_solve / vg_adjoint_grad / vg_errors / vg_rhs is a
 *     DEVICE pointer, unless the function name ends in _host;
 *   - global vector layout: flux edge moments (degree-major, r * num_edges + edge), flux interior
 *     moments (cell-major), pressure (cell-major, q per cell), then one mean-pressure multiplier
 *     when the boundary condition is VG_BC_FLUX (vem/CurvedVEM_Darcy/solver/DarcySolver.cpp:182-227);
 *   - all functions return 0 on success or a VG_E* code; vg_last_error() describes the failure.
 *     No C++ exception crosses this boundary (vem/CurvedVEM_Darcy_gpu/src/krylov.cu:8-36).
 *   - a handle is not re-entrant: one host thread at a time (vem/CurvedVEM_Darcy_gpu/include/petsc_gpu.h:5).
 */
#ifndef VEMGPU_H
#define VEMGPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vg_handle vg_handle;

enum {
    VG_OK = 0,
    VG_EINVAL = 1,     /* invalid argument (sizes, options, null pointers)          */
    VG_EMESH = 2,      /* degenerate mesh: bad polygon, edge shared by > 2 cells     */
    VG_EGEOMETRY = 3,  /* nonpositive Jacobian of the geometry map                   */
    VG_ESINGULAR = 4,  /* singular local matrix (G, H or edge mass) in some cell     */
    VG_ECUDA = 5,      /* CUDA runtime error or no device                            */
    VG_ENOCONV = 6,    /* Krylov solve did not reach the tolerance within maxit      */
    VG_ESTATE = 7,     /* call out of order (e.g. vg_solve before vg_build)          */
    VG_ENOMEM = 8      /* device allocation failed                                   */
};

enum { VG_GEOM_IDENTITY = 0, VG_GEOM_SINE = 1, VG_GEOM_ARCS = 2 };
/* built-in PDE data: SINCOS = Darcy examples 1/2 of the reference (p = sin(pi x) cos(pi y),
 * vem/CurvedVEM_Darcy_gpu/examples/darcy_problem.cpp:110-200); SINSIN = p = sin(pi x) sin(pi y);
 * ANNULUS = p_D = 1 on r = 0.3, 0 on r = 1, f = 0 (exact p = ln r / ln 0.3 for K = I). */
enum { VG_PROBLEM_SINCOS = 1, VG_PROBLEM_SINSIN = 2, VG_PROBLEM_ANNULUS = 3 };
/* VG_BC_FLUX: essential normal flux on the whole boundary + zero-mean pressure multiplier
 * (the reference's only implemented BC, DarcySolver.cpp:502-663); VG_BC_PRESSURE: Dirichlet
 * pressure on the whole boundary, entering as the load -int p_D v.n ds on boundary edge moments
 * (declared but never defined in the reference, DarcySolver.h:88). */
enum { VG_BC_FLUX = 0, VG_BC_PRESSURE = 1 };
enum { VG_FP64 = 0, VG_FP32 = 1 };
/* solve modes: plain FP64 MINRES, or FP32 inner MINRES under FP64 iterative refinement */
enum { VG_SOLVE_FP64 = 0, VG_SOLVE_MIXED = 1 };

/* The reference reader's StraightMeshData (vem/CurvedVEM_Darcy_gpu/mesh/straight_mesh.h:20-49),
 * host pointers. cell_nodes is counter-clockwise per cell; global_edges has the same layout;
 * edge_endpoints holds (smaller node, larger node); edge_occurrence is 1 (boundary) or 2. */
typedef struct vg_mesh {
    int num_nodes, num_cells, num_edges;
    const double* node_coords;        /* 2 * num_nodes                 */
    const int* cell_nodes;            /* cell_node_indices[num_cells]  */
    const int* cell_node_indices;     /* num_cells + 1                 */
    const int* nodes_per_cell;        /* num_cells                     */
    const int* global_edges;          /* same layout as cell_nodes     */
    const int* cell_edge_indices;     /* num_cells + 1                 */
    const int* edge_endpoints;        /* 2 * num_edges                 */
    const int* edge_occurrence;       /* num_edges                     */
    const double* cell_centroid_x;    /* num_cells                     */
    const double* cell_centroid_y;    /* num_cells                     */
    const double* cell_diameter;      /* num_cells                     */
} vg_mesh;

/* Geometry map from the straight computational mesh to the physical domain. Replaces the
 * reference's CPU std::function callback (vem/CurvedVEM_Darcy_gpu/include/hdiv_gpu.cuh:15),
 * evaluated on the device instead:
 *   VG_GEOM_IDENTITY;
 *   VG_GEOM_SINE: x + eps sin(2 pi y), y + eps sin(2 pi x) (SinPerturbationMapping,
 *                 vem/CurvedVEM_Darcy_gpu/examples/darcy_problem.h:70-121);
 *   VG_GEOM_ARCS: boundary chords (arc_nodes[2a], arc_nodes[2a+1]) are mapped onto circular arcs
 *                 of circle arc_circles[3a..3a+2] = (cx, cy, r); a cell with an arc edge is
 *                 integrated on the fan of triangles from its vertex average, the fan triangle of
 *                 the chord carrying the blending map c + lam (gamma(t) - c). */
typedef struct vg_geometry {
    int kind;
    double eps;
    int num_arcs;
    const int* arc_nodes;       /* 2 * num_arcs node ids (host) */
    const double* arc_circles;  /* 3 * num_arcs (host)          */
} vg_geometry;

typedef struct vg_solve_opts {
    int mode;            /* VG_SOLVE_FP64 or VG_SOLVE_MIXED                                    */
    double tol;          /* relative true residual ||b - A x|| / ||b|| (reference: 1e-10)      */
    int maxit;           /* cap on total inner iterations                                      */
    double inner_tol;    /* MIXED: relative reduction asked of each FP32 inner solve (a later
                            step asks for less, 0.1 tol / current residual, when that suffices) */
    int max_outer;       /* MIXED: cap on refinement steps                                     */
    int check_every;     /* 0: the whole Krylov loop is one CUDA graph (device-side while node,
                            iteration cap on the device); > 0: host-driven batches of this many
                            iterations, every kernel a plain launch (for profilers)            */
    int nonzero_guess;   /* 1: x holds the initial guess on entry                              */
} vg_solve_opts;

typedef struct vg_solve_info {
    int iterations;      /* total Krylov iterations (inner iterations in MIXED mode)            */
    int outer;           /* refinement steps (MIXED) or restarts on the true residual (FP64)   */
    double residual;     /* final ||b - A x|| / ||b||, computed in FP64 on the device          */
    double seconds;      /* device time of the solve (CUDA events)                             */
} vg_solve_info;

/* ---- lifecycle -------------------------------------------------------------------------- */

/* Processed mesh (the reference reader's output). k in 0..4, nq in {1,3,4,7,9,12,36},
 * ng in [k+2, 10], with the reference's consistency rules (vem/CurvedVEM_Darcy_gpu/src/solver_options.cpp:123-136).
 * Replaces HdivGpu::HdivGpu (vem/CurvedVEM_Darcy_gpu/include/hdiv_gpu.cuh:55-56) and
 * HostMesh::HostMesh (vem/CurvedVEM_Darcy_gpu/src/mesh_pack.cpp:127-238). device < 0: current device.
 * The caller's current device is the same on return; every later call on the handle runs on the
 * handle's device and gives the caller's current device back (one thread may hold handles on
 * several GPUs). */
int vg_create(const vg_mesh* mesh, const vg_geometry* geometry, int k, int nq, int ng, int device, vg_handle** out);

/* Raw polygons (any orientation): performs the reader post-processing of
 * vem/CurvedVEM_Darcy_gpu/mesh/straight_mesh.cpp:467-664 (CCW order, centroid with the 4-gon
 * bounding-box rule, diameter, global edges by sorting, occurrence) before vg_create. */
int vg_create_polygons(int num_nodes, const double* node_coords, int num_cells, const int* cell_ptr,
                       const int* cell_nodes, const vg_geometry* geometry, int k, int nq, int ng, int device,
                       vg_handle** out);

/* Legacy ASCII VTK polygon file (POINTS, CELLS with a vertex count per cell, CELL_TYPES 5/7/9; other
 * sections skipped), then the same post-processing as vg_create_polygons. Replaces
 * StraightMeshReader::read_mesh_vtk (vem/CurvedVEM_Darcy_gpu/mesh/straight_mesh.h:101,
 * straight_mesh.cpp:68-218) followed by the handle construction. Arcs, if any, come in geometry. */
int vg_create_vtk(const char* path, const vg_geometry* geometry, int k, int nq, int ng, int device, vg_handle** out);

int vg_destroy(vg_handle* h);
const char* vg_last_error(const vg_handle* h);

/* Sizes: out[0..8] = num_cells, num_edges, nf (flux dofs), np (pressure dofs), N (system size),
 * q, p, internal flux dofs per cell, max local flux dofs. */
int vg_sizes(const vg_handle* h, long long out[9]);

/* Built-in PDE data and boundary condition (MixedGpu example selection, equation_gpu.cu:502-507). */
int vg_set_problem(vg_handle* h, int problem, int bc);

/* Per-cell log permeability theta (K_E = exp(theta_E) I): host (on_device = 0) or device pointer.
 * New in this library; the reference hard-codes K = I (vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:63-68). */
int vg_set_log_permeability(vg_handle* h, const double* theta, int on_device);

/* FP64 setup on the device: geometry, projector and local operators (HdivGpu::build_basis,
 * hdiv_gpu.cu:172-192, + MixedGpu::update, equation_gpu.cu:547-577), right-hand side and boundary
 * data (MixedGpu::make_rhs, equation_gpu.cu:611-625) and the preconditioner. */
int vg_build(vg_handle* h);

/* ---- operator ----------------------------------------------------------------------------- */

/* y = A x, reference sign [A, -W^T, 0; W, 0, L; 0, L^T, 0], device pointers (x != y).
 * precision VG_FP64 (double*) or VG_FP32 (float*). constrained = 1 applies the essential-BC mask
 * as Q A Q + (I - Q) (VG_BC_FLUX only). stream: cudaStream_t or NULL (legacy default stream).
 * Asynchronous: a failure inside the kernel (a copy-pipeline wait that gave up; never in a correct
 * run) sets an error word in mapped host memory and is reported as VG_ECUDA by the next vg_apply
 * on the handle after that kernel has finished, or by the next vg_solve; no call adds a check to
 * the caller's stream.
 * Replaces MixedGpu::apply (vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:580-598). */
int vg_apply(vg_handle* h, const void* x, void* y, int precision, int constrained, void* stream);

/* Failure-path test hook (no counterpart in the reference): in the next matrix-free apply of the
 * handle (k <= 1) one consumer warp waits, at its CTA's last operator batch, on a barrier that
 * nothing arrives on, so that its bounded wait runs out after the one-second limit; the kernel then
 * drains its copies, sets its error word and returns, and the call that launched it reports
 * VG_ECUDA as described for vg_apply and vg_solve. The result of that apply is wrong (the pieces
 * of that batch are missing). For tests of the error path only. */
int vg_debug_stall_apply(vg_handle* h);

/* Internally the solver numbers the flux unknowns by first use in its cell layout and the pressure
 * rows by cell layout, so that the apply's gathers and scatters coalesce; vg_apply and vg_solve
 * permute at the boundary. A caller that runs many applies (its own Krylov loop) can keep vectors
 * in that order: vg_permute(h, 1, x, xi, ...) maps the reference order to the internal one
 * (0: back), and vg_apply with precision | VG_ORDER_INTERNAL takes and returns internal-order
 * vectors (no permutation). No counterpart in the reference. */
#define VG_ORDER_INTERNAL 0x100
int vg_permute(vg_handle* h, int to_internal, const void* in, void* out, int precision, void* stream);

/* Right-hand side of the constrained system (reference sign, device pointer, N doubles):
 * pressure rows int f m det J, Dirichlet loads on flux rows (VG_BC_PRESSURE) or the lifted rows
 * of MixedGpu::make_rhs (VG_BC_FLUX). */
int vg_rhs(vg_handle* h, double* b);

/* ---- solve -------------------------------------------------------------------------------- */

void vg_default_solve_opts(vg_solve_opts* opts);

/* Solve A x = b to ||b - A x|| / ||b|| <= opts->tol (device pointers). Replaces Krylov::solve
 * (vem/CurvedVEM_Darcy_gpu/src/krylov.cu:73-175); PETSc FGMRES is replaced by MINRES on the
 * symmetric form with a block-diagonal preconditioner, the FP64 true-residual acceptance is kept. */
int vg_solve(vg_handle* h, const double* b, double* x, const vg_solve_opts* opts, vg_solve_info* info);

/* Same with host buffers: copies b in and x out inside the call (the end-to-end path). */
int vg_solve_host(vg_handle* h, const double* b_host, double* x_host, const vg_solve_opts* opts,
                  vg_solve_info* info);

/* ---- adjoint ------------------------------------------------------------------------------ */

/* Given the forward solution x and dJ/dx (device, N doubles each), solve the adjoint system and
 * write dJ/dtheta (device, num_cells doubles): dJ/dtheta_E = lambda_E^T A_E u_E with the local
 * gathers of x and lambda. No counterpart in the reference. */
int vg_adjoint_grad(vg_handle* h, const double* x, const double* dJdx, double* dJdtheta,
                    const vg_solve_opts* opts, vg_solve_info* info);

/* Assembled sparse matrix of the same operator (a comparator of the matrix-free apply; the
 * reference's assembled path, MixedGpu::assembled_matrix / coo_matrix / coo_boundary,
 * vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:701-833, which PETSc turns into cuSPARSE CSR).
 * Reference sign [A, -W^T, L; W, 0, 0; L^T, 0, 0]; constrained = 1 (VG_BC_FLUX) zeroes masked rows
 * and columns and puts 1 on their diagonal. First call with row_ptr = NULL: *nnz = number of stored
 * entries (pattern built on the host and kept). Second call: DEVICE arrays row_ptr (N+1, int64,
 * sorted columns per row), col_idx (nnz) and values (nnz doubles) are filled. */
int vg_assemble_csr(vg_handle* h, int constrained, long long* nnz, long long* row_ptr, int* col_idx, double* values);

/* Physical cell measures int_E det J (device, num_cells doubles); the reference keeps them in
 * Cell::area of its device records (vem/CurvedVEM_Darcy_gpu/include/device.cuh:107-134). */
int vg_cell_areas(vg_handle* h, double* areas);

/* ---- ternary Maxwell-Stefan diffusion (k = 0) ------------------------------------------------
 * Replaces the reference's Maxwell-Stefan driver (MSGpu, vem/CurvedVEM_Darcy_gpu/include/equation_gpu.cuh:122-127,
 * run_case time loop src/solver_driver.cpp:189-245), in the reduced two-species form with
 * diffusivities D12, D13, D23: backward Euler, one coupled saddle-point system per step with the
 * friction matrix frozen at x^n, no flux through the boundary (the handle must be built with
 * VG_BC_FLUX; its K = I operator is used whatever the permeability). State vector (device doubles):
 * [J1 (nf), J2 (nf), x1 (num_cells), x2 (num_cells)], x3 = 1 - x1 - x2. */
int vg_ms_configure(vg_handle* h, double d12, double d13, double d23, double dt, long long* state_size);
/* y = K(coeff_state) x for the Maxwell-Stefan system (FP64 or FP32 x, y; device). */
int vg_ms_apply(vg_handle* h, const double* coeff_state, const void* x, void* y, int precision);
/* One backward-Euler step: solve K(old) new = [0; |E|/dt x_old] to ||b - K new|| / ||b|| <= opts->tol
 * by right-preconditioned GMRES(10), FP64 or FP32 inner under FP64 refinement (opts->mode). With
 * Picard iterations enabled (vg_ms_set_picard), the friction matrix is re-evaluated at the latest
 * iterate and the system solved again until the step is fully implicit to the Picard tolerance. */
int vg_ms_step(vg_handle* h, const double* old_state, double* new_state, const vg_solve_opts* opts,
               vg_solve_info* info);
/* Picard iterations of vg_ms_step (the reference's loop, vem/CurvedVEM_Darcy_gpu/src/solver_driver.cpp:209-240):
 * max_iterations = 1 (the default) keeps the friction matrix at x^n (linearly implicit step);
 * > 1 iterates K(x^{n+1,m}) x^{n+1,m+1} = b until ||x^{m+1} - x^m|| / max(1, ||x^{m+1}||) <= tol and
 * the nonlinear residual ||b - K(x) x|| / ||b|| at the accepted x is <= max(tol, 5 opts->tol);
 * VG_ENOCONV otherwise. vg_ms_picard_info reports the last step's iterations, change and residual. */
int vg_ms_set_picard(vg_handle* h, int max_iterations, double tol);
int vg_ms_picard_info(const vg_handle* h, int* iterations, double* change, double* nonlinear_residual);
/* Gram-Schmidt work of the Maxwell-Stefan GMRES since the handle was created: Arnoldi steps and
 * how many of them ran the second classical Gram-Schmidt pass. The second pass runs only when the
 * first removed more than half of |w|^2 (selective reorthogonalisation, Daniel-Gragg-Kaufman-
 * Stewart). No counterpart in the reference (its Krylov solves are PETSc's). */
int vg_ms_gs_info(const vg_handle* h, long long* arnoldi_steps, long long* reorthogonalizations);

/* ---- post-processing ---------------------------------------------------------------------- */

/* Six figures of MixedGpu::errors (equation_gpu.cu:387-479, 627-648): computational scalar and
 * flux L2 errors, physical scalar, flux and divergence L2 errors, physical mean-pressure mass.
 * Runs on the legacy default stream, which does not wait for work queued on non-blocking streams
 * (torch's side streams are non-blocking): synchronize the stream that wrote x before the call. */
int vg_errors(vg_handle* h, const double* x, double out[6]);

/* vg_errors without any device allocation: the per-cell figures and their sums live in a
 * static device array sized for VG_ERRORS_NOALLOC_MAX_CELLS cells (12.6 MB); larger meshes get
 * VG_EINVAL. For callers that must not allocate device memory between solves: a process whose
 * HBM is already reserved by its own caching allocator (cudaMalloc may fail there), or one that
 * monitors the error inside a loop while other streams run (cudaMalloc and cudaFree can
 * synchronize the device). Same results as vg_errors. Every call looks up the array's device
 * address (no allocation); the first call on a device may load the library's device code and must
 * come before any stream capture on that device. The array is shared by every handle of a device,
 * so calls that overlap on the GPU (several host threads) race. Runs on the legacy default stream,
 * like vg_errors (synchronize the stream that wrote x before the call), and returns after the
 * figures are on the host. No counterpart in the reference. */
#define VG_ERRORS_NOALLOC_MAX_CELLS 262144
int vg_errors_noalloc(vg_handle* h, const double* x, double out[6]);

/* Copy one cell's local operator data to the host (verification): which = 0 A_E (n x n, K
 * included), 1 W_E (q x n), 2 P (p x n), 3 alpha (1), 4 global flux dof map with sign (n, as
 * doubles, sign * (index + 1)), 5 rhs (q), 6 Dirichlet load (n). Returns the count in *count. */
int vg_local(vg_handle* h, int cell, int which, double* out, int* count);

/* Diagnostics (no counterpart in the reference): out[0] = kernels launched by this handle,
 * out[1] = operator applies, out[2] = Krylov iterations, out[3] = solves, since creation. */
int vg_stats(const vg_handle* h, long long out[4]);

#ifdef __cplusplus
}
#endif
#endif /* VEMGPU_H */
