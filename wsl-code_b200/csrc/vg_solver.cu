// vemgpu Solver: host orchestration of the device setup, apply, Krylov solve, adjoint and errors.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <unordered_map>

#include "vg_apply.cuh"
#include "vg_krylov.cuh"
#include "vg_setup.cuh"
#include "vg_solver.hpp"

namespace vg {

void diag_flux(const double* A, const int* map, const Piece* pieces, int npieces, double* d, cudaStream_t s);
void diag_finish(const double* W, const int* map, const int* slot_cell, const int* mask, const double* L,
                 const Piece* pieces, int npieces, int k, long long nf, double* d, double* contrib, cudaStream_t s);
void diag_invert(double* d, const int* mask, const double* contrib, int nc, long long nf, long long np, int mult,
                 long long N, cudaStream_t s);
void lift_rhs(const int* mask, const double* g, const double* y, double* b, long long N, cudaStream_t s);
void rescale_ops(const double* theta, const int* slot_cell, const Piece* pieces, int npieces, const double* A0,
                 double* A64, float* A32, cudaStream_t s);
void assemble_values(const double* A, const double* W, const int* map, const int* slot_cell, const int* mask,
                     const double* L, const Piece* pieces, int npieces, int k, long long nf, long long N,
                     int constrained, int mult, const long long* rp, const int* ci, double* val, int* bad,
                     cudaStream_t s);
template <typename T>
void gather_launch(const T* in, const int* idx, long long off, T* out, long long n, cudaStream_t s);
void schur_values(const int* sptr, const int* scol, int nrows, int q, int k, const int* rank_cell, const int* cell_rank,
                  const int* cell_slot, const Piece* pieces, const int* map, const double* W, const double* dinv,
                  const int* inc_ptr, const int* inc_cell, const int* inc_i, const signed char* inc_s, double* sval);
void contract_adjoint(const double* A, const int* map, const int* slot_cell, const int* mask, const Piece* pieces,
                      int npieces, int k, const double* x, const double* mu, int constrained, double* g,
                      cudaStream_t s);
long long first_nonfinite(const double* v, long long n);

namespace {

// Gauss-Legendre rules on [-1, 1] (vem/CurvedVEM_Darcy_gpu/core/gauss_quadrature.cpp:74-167)
std::vector<double> gauss_legendre(int n) {
    struct H {
        double x, w;
    };
    std::vector<H> half;
    bool centre = false;
    double wc = 0;
    switch (n) {
    case 1: return {0.0, 2.0};
    case 2: half = {{0.5773502691896257645091488, 1.0}}; break;
    case 3: half = {{0.7745966692414833770358531, 0.5555555555555556}}; centre = true; wc = 0.8888888888888889; break;
    case 4: half = {{0.8611363115940526, 0.3478548451374539}, {0.3399810435848563, 0.6521451548625461}}; break;
    case 5:
        half = {{0.9061798459386640, 0.2369268850561891}, {0.5384693101056831, 0.4786286704993665}};
        centre = true;
        wc = 0.5688888888888889;
        break;
    case 6:
        half = {{0.9324695142031520, 0.1713244923791703}, {0.6612093864662645, 0.3607615730481386},
                {0.2386191860831969, 0.4679139345726910}};
        break;
    case 7:
        half = {{0.9491079123427585, 0.1294849661688697}, {0.7415311855993944, 0.2797053914892767},
                {0.4058451513773972, 0.3818300505051190}};
        centre = true;
        wc = 0.4179591836734694;
        break;
    case 8:
        half = {{0.9602898564975362, 0.1012285362903763}, {0.7966664774136267, 0.2223810344533745},
                {0.5255324099163290, 0.3137066458778873}, {0.1834346424956498, 0.3626837833783620}};
        break;
    case 9:
        half = {{0.9681602395076261, 0.0812743883615744}, {0.8360311073266358, 0.1806481606948574},
                {0.6133714327005904, 0.2606106964029355}, {0.3242534234038089, 0.3123470770400028}};
        centre = true;
        wc = 0.3302393550012598;
        break;
    case 10:
        half = {{0.9739065285171717, 0.0666713443086881}, {0.8650633666889845, 0.1494513491505806},
                {0.6794095682990244, 0.2190863625159820}, {0.4333953941292472, 0.2692667193099964},
                {0.1488743389816312, 0.2955242247147529}};
        break;
    default: throw Error(VG_EINVAL, "Gauss-Legendre order must be 1..10");
    }
    std::vector<double> out;
    for (auto& h : half) {
        out.push_back(-h.x);
        out.push_back(h.w);
    }
    if (centre) {
        out.push_back(0.0);
        out.push_back(wc);
    }
    for (auto it = half.rbegin(); it != half.rend(); ++it) {
        out.push_back(it->x);
        out.push_back(it->w);
    }
    return out;
}

// triangle rules as (xi, eta, w) on the reference triangle (gauss_quadrature.cpp:258-305) and the
// 36-point Duffy rule of vem/CurvedVEM_Darcy_gpu/src/mesh_pack.cpp:110-124 written the same way
std::vector<double> triangle_rule(int n) {
    std::vector<double> r;
    auto add = [&](double a, double b, double w) {
        r.push_back(a);
        r.push_back(b);
        r.push_back(w);
    };
    switch (n) {
    case 1: add(1.0 / 3.0, 1.0 / 3.0, 0.5); break;
    case 3:
        add(0.5, 0.0, 1.0 / 6.0);
        add(0.5, 0.5, 1.0 / 6.0);
        add(0.0, 0.5, 1.0 / 6.0);
        break;
    case 4: {
        double s = 1.0 / std::sqrt(3.0);
        add((1 + s) / 2, (1 - s) * (1 + s) / 4, (1 - s) / 8.0);
        add((1 + s) / 2, (1 - s) * (1 - s) / 4, (1 - s) / 8.0);
        add((1 - s) / 2, (1 + s) * (1 + s) / 4, (1 + s) / 8.0);
        add((1 - s) / 2, (1 + s) * (1 - s) / 4, (1 + s) / 8.0);
        break;
    }
    case 7: {
        add(1.0 / 3.0, 1.0 / 3.0, 0.1125);
        double a = 0.797426985353087, b = 0.101286507323456, w1 = 0.0629695902724135;
        add(a, b, w1);
        add(b, a, w1);
        add(b, b, w1);
        double c = 0.059715871789770, d = 0.470142064105115, w2 = 0.0661970763907399;
        add(c, d, w2);
        add(d, c, w2);
        add(d, d, w2);
        break;
    }
    case 9: {
        double s = std::sqrt(3.0 / 5.0);
        add(0.5, 0.25, 64.0 / 81.0 * 1.0 / 8.0);
        add((1 + s) / 2, (1 - s) * (1 + s) / 4, 100.0 / 324.0 * (1 - s) / 8.0);
        add((1 + s) / 2, (1 - s) * (1 - s) / 4, 100.0 / 324.0 * (1 - s) / 8.0);
        add((1 - s) / 2, (1 + s) * (1 + s) / 4, 100.0 / 324.0 * (1 + s) / 8.0);
        add((1 - s) / 2, (1 + s) * (1 - s) / 4, 100.0 / 324.0 * (1 + s) / 8.0);
        add(0.5, (1 + s) / 4, 40.0 / 81.0 * 1.0 / 8.0);
        add(0.5, (1 - s) / 4, 40.0 / 81.0 * 1.0 / 8.0);
        add((1 + s) / 2, (1 - s) / 4, 40.0 / 81.0 * (1 - s) / 8.0);
        add((1 - s) / 2, (1 + s) / 4, 40.0 / 81.0 * (1 + s) / 8.0);
        break;
    }
    case 12: {
        const double a = 0.5611400349004341, b = 0.2194299825497830, wa = 0.1713331241529811 * 0.5;
        const double c = 0.0397240717755698, d = 0.4801379641122151, wc = 0.0807310895930309 * 0.5;
        const double e = 0.0193717243612408, f = 0.1416190159239682, g = 0.8390092597147911,
                     we = 0.0406345597936607 * 0.5;
        add(a, b, wa);
        add(b, b, wa);
        add(b, a, wa);
        add(c, d, wc);
        add(d, d, wc);
        add(d, c, wc);
        add(e, f, we);
        add(f, g, we);
        add(g, e, we);
        add(f, e, we);
        add(e, g, we);
        add(g, f, we);
        break;
    }
    case 36: {
        auto g6 = gauss_legendre(6);
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) {
                double u = (g6[2 * i] + 1) / 2, wa = g6[2 * i + 1] / 2, ub = (g6[2 * j] + 1) / 2, wb = g6[2 * j + 1] / 2;
                add(u, (1 - u) * ub, wa * wb * (1 - u));
            }
        break;
    }
    default: throw Error(VG_EINVAL, "triangle quadrature must be 1, 3, 4, 7, 9, 12 or 36");
    }
    return r;
}

}  // namespace

Solver::Solver(HostMesh&& mesh, const vg_geometry* geo, int k_, int nq_, int ng_, int device) : m(std::move(mesh)) {
    // option rules of vem/CurvedVEM_Darcy_gpu/src/solver_options.cpp:123-136
    if (k_ < 0 || k_ > 4) throw Error(VG_EINVAL, "polynomial degree k must be 0..4");
    if (nq_ != 1 && nq_ != 3 && nq_ != 4 && nq_ != 7 && nq_ != 9 && nq_ != 12 && nq_ != 36)
        throw Error(VG_EINVAL, "triangle quadrature must be 1, 3, 4, 7, 9, 12 or 36");
    if ((k_ >= 1 && nq_ == 1) || (k_ >= 2 && (nq_ == 3 || nq_ == 4)))
        throw Error(VG_EINVAL, "triangle quadrature under-integrates this degree");
    if ((k_ == 3 && nq_ < 12) || (k_ == 4 && nq_ != 36))
        throw Error(VG_EINVAL, "insufficient triangle quadrature for this degree");
    if (ng_ < k_ + 2 || ng_ > 10) throw Error(VG_EINVAL, "edge quadrature must be between k+2 and 10");
    k = k_;
    nq = nq_;
    ng = ng_;
    int ndev = 0;
    VG_CUDA(cudaGetDeviceCount(&ndev));
    if (ndev == 0) throw Error(VG_ECUDA, "no CUDA device");
    if (device >= 0) VG_CUDA(cudaSetDevice(device));
    VG_CUDA(cudaGetDevice(&device_));
    VG_CUDA(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device_));
    q = dimP(k);
    p = p_of(k);
    ngrad = ngrad_of(k);
    internal = internal_of(k);
    nf = m.ne * (k + 1) + m.nc * internal;
    np = m.nc * q;
    N = nf + np + 1;  // flux BC (reference default) until set_problem
    // geometry
    std::vector<int> edge_arc(m.ne, -1);
    std::vector<double> arcdata;
    if (geo) {
        geom_kind = geo->kind;
        eps = geo->eps;
        if (geom_kind < VG_GEOM_IDENTITY || geom_kind > VG_GEOM_ARCS) throw Error(VG_EINVAL, "unknown geometry kind");
        if (geom_kind == VG_GEOM_ARCS) {
            if (geo->num_arcs < 0 || (geo->num_arcs > 0 && (!geo->arc_nodes || !geo->arc_circles)))
                throw Error(VG_EINVAL, "arc geometry needs arc_nodes and arc_circles");
            std::unordered_map<unsigned long long, int> look;
            look.reserve(size_t(m.ne) * 2);
            for (int e = 0; e < m.ne; ++e)
                look[(static_cast<unsigned long long>(unsigned(m.eend[2 * e])) << 32) | unsigned(m.eend[2 * e + 1])] = e;
            arcdata.assign(3 * size_t(m.ne), 0.0);
            for (int a = 0; a < geo->num_arcs; ++a) {
                unsigned u = unsigned(geo->arc_nodes[2 * a]), v = unsigned(geo->arc_nodes[2 * a + 1]);
                auto it = look.find((static_cast<unsigned long long>(std::min(u, v)) << 32) | std::max(u, v));
                if (it == look.end()) throw Error(VG_EINVAL, "arc chord is not a mesh edge");
                if (m.eocc[it->second] != 1) throw Error(VG_EINVAL, "arc chord is not a boundary edge");
                if (!(geo->arc_circles[3 * a + 2] > 0)) throw Error(VG_EINVAL, "arc radius must be positive");
                edge_arc[it->second] = a;
                for (int c = 0; c < 3; ++c) arcdata[3 * size_t(it->second) + c] = geo->arc_circles[3 * a + c];
            }
        }
    }
    std::vector<char> curved(m.nc, 0);
    if (geom_kind == VG_GEOM_ARCS)
        for (int c = 0; c < m.nc; ++c)
            for (int j = m.cptr[c]; j < m.cptr[c + 1]; ++j)
                if (edge_arc[m.gedges[j]] >= 0) curved[c] = 1;
    std::vector<int> triptr;
    std::vector<TriIdx> tris;
    PhaseTimer pt;
    triangulate(m, curved, edge_arc, triptr, tris);
    pt.mark("triangulate");
    pack_layout();
    pt.mark("pack layout");
    // uploads
    d_xy_.upload(m.xy);
    d_cptr_.upload(m.cptr);
    d_cnodes_.upload(m.cnodes);
    d_gedges_.upload(m.gedges);
    d_cx_.upload(m.cx);
    d_cy_.upload(m.cy);
    d_diam_.upload(m.diam);
    d_triptr_.upload(triptr);
    d_tris_.upload(tris);
    if (geom_kind == VG_GEOM_ARCS) d_arc_.upload(arcdata);
    d_slot_cell_.upload(slot_cell_);
    d_cell_slot_.upload(cell_slot_);
    d_pieces_.upload(pieces_);
    d_map_.upload(map_host_);
    plan_internal_order();
    pt.mark("uploads");
    plan_streams();
    pt.mark("record-stream plan");
    {
        std::vector<int> occ(m.eocc);
        DevBuf<int> tmp;
        tmp.upload(occ);
        d_eocc_ = std::move(tmp);
    }
    theta_.assign(m.nc, 0.0);
    d_theta_.upload(theta_);
    d_status_.resize(1);
    d_counter_.resize(1);
    d_counter_.zero();
    VG_CUDA(cudaEventCreate(&ev0_));
    VG_CUDA(cudaEventCreate(&ev1_));
    VG_CUDA(cudaEventCreateWithFlags(&ev_in_, cudaEventDisableTiming));
    VG_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    VG_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
    VG_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
    VG_CUDA(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
    d_loop_.resize(2);
}

Solver::~Solver() {
    destroy_graphs();
    ms_destroy_graphs();
    if (h_err_) cudaFreeHost(h_err_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (ev_in_) cudaEventDestroy(ev_in_);
    if (stream_) cudaStreamDestroy(stream_);
    if (side_) cudaStreamDestroy(side_);
    if (ev_fork_) cudaEventDestroy(ev_fork_);
    if (ev_join_) cudaEventDestroy(ev_join_);
}

void Solver::destroy_graphs() {
    for (int p = 0; p < 2; ++p) {
        if (gexec_[p]) cudaGraphExecDestroy(gexec_[p]);
        if (graph_[p]) cudaGraphDestroy(graph_[p]);
        gexec_[p] = nullptr;
        graph_[p] = nullptr;
    }
}

void Solver::plan_internal_order() {
    const long long NN = (long long)nf + np + 1;  // + the multiplier row, which keeps its index
    e2i_host_.assign(NN, -1);
    i2e_host_.assign(NN, -1);
    map_int_host_.assign(map_host_.size(), 0);
    prow_host_.assign(slot_cell_.size(), -1);
    int nextf = 0, nextp = 0;
    for (const auto& P : pieces_) {
        for (int i = 0; i < P.n; ++i)
            for (int j = 0; j < P.count; ++j) {
                const long long o = P.map_off + (long long)i * PIECE + j;
                const int g = map_host_[o], gg = g < 0 ? ~g : g;
                if (e2i_host_[gg] < 0) {
                    e2i_host_[gg] = nextf;
                    i2e_host_[nextf] = gg;
                    ++nextf;
                }
                const int gi = e2i_host_[gg];
                map_int_host_[o] = g < 0 ? ~gi : gi;
            }
        for (int j = 0; j < P.count; ++j) {
            const int c = slot_cell_[P.slot + j];
            prow_host_[P.slot + j] = nf + nextp * q;
            for (int r = 0; r < q; ++r) {
                e2i_host_[nf + (long long)c * q + r] = nf + nextp * q + r;
                i2e_host_[nf + (long long)nextp * q + r] = nf + c * q + r;
            }
            ++nextp;
        }
    }
    e2i_host_[NN - 1] = int(NN - 1);
    i2e_host_[NN - 1] = int(NN - 1);
    if (nextf != nf || nextp != m.nc) throw Error(VG_EMESH, "dof numbering does not cover every unknown");
    d_map_int_.upload(map_int_host_);
    d_prow_.upload(prow_host_);
    d_e2i_.upload(e2i_host_);
    d_i2e_.upload(i2e_host_);
}

void Solver::internal_copies() {
    d_mask_int_.resize(N);
    gather_launch<int>(d_mask_.data(), d_i2e_.data(), 0, d_mask_int_.data(), N, nullptr);
    d_Lint_.resize(size_t(np));
    d_Lint32_.resize(size_t(np));
    gather_launch<double>(d_L_.data(), d_i2e_.data(), nf, d_Lint_.data(), np, nullptr);
    gather_launch<float>(d_L32_.data(), d_i2e_.data(), nf, d_Lint32_.data(), np, nullptr);
    d_xi_.resize(N);
}

template <typename T>
void Solver::permute(const T* in, T* out, bool to_internal, cudaStream_t s) {
    gather_launch<T>(in, to_internal ? d_i2e_.data() : d_e2i_.data(), 0, out, N, s);
}
template void Solver::permute<double>(const double*, double*, bool, cudaStream_t);
template void Solver::permute<float>(const float*, float*, bool, cudaStream_t);

void Solver::pack_layout() {
    // chunks of CHUNK consecutive cells, grouped by edge count inside a chunk, split into pieces
    pieces_.clear();
    slot_cell_.clear();
    cell_slot_.assign(m.nc, -1);
    a_total_ = w_total_ = map_total_ = p_total_ = hw_total_ = 0;
    maxn = 0;
    std::vector<std::vector<int>> byne(MAX_NE + 1), classes(MAX_NE + 1);
    for (int c0 = 0; c0 < m.nc; c0 += CHUNK) {
        int c1 = std::min(m.nc, c0 + CHUNK);
        for (auto& v : byne) v.clear();
        for (int c = c0; c < c1; ++c) byne[m.cptr[c + 1] - m.cptr[c]].push_back(c);
        for (int ne = 3; ne <= MAX_NE; ++ne)
            for (size_t s0 = 0; s0 < byne[ne].size(); s0 += PIECE) {
                Piece P{};
                P.ne = ne;
                P.n = (k + 1) * ne + internal;
                P.count = int(std::min<size_t>(PIECE, byne[ne].size() - s0));
                P.slot = (long long)pieces_.size() * PIECE;
                P.a_off = a_total_;
                P.w_off = w_total_;
                P.map_off = map_total_;
                P.p_off = p_total_;
                P.hw_off = hw_total_;
                a_total_ += (long long)PIECE * (P.n * (P.n + 1) / 2);
                w_total_ += k >= 1 ? (long long)PIECE * q * P.n : 0;
                map_total_ += (long long)PIECE * P.n;
                p_total_ += (long long)PIECE * p * P.n;
                hw_total_ += (long long)PIECE * q * P.n;
                maxn = std::max(maxn, P.n);
                for (int l = 0; l < PIECE; ++l) {
                    int c = l < P.count ? byne[ne][s0 + l] : -1;
                    if (c >= 0) {
                        cell_slot_[c] = int(slot_cell_.size());
                        classes[ne].push_back(c);
                    }
                    slot_cell_.push_back(c);
                }
                pieces_.push_back(P);
            }
    }
    classes_.clear();
    class_cells_.clear();
    for (int ne = 3; ne <= MAX_NE; ++ne)
        if (!classes[ne].empty()) {
            class_cells_.emplace_back();
            class_cells_.back().upload(classes[ne]);
            classes_.push_back(CellClass{ne, (k + 1) * ne + internal, int(classes[ne].size()),
                                         class_cells_.back().data()});
        }
    // signed flux dof map (vem/CurvedVEM_Darcy_gpu/src/mesh_pack.cpp:209-225): edge moments degree-major,
    // sign -1 on even moments of an interior edge traversed against its (min, max) orientation
    map_host_.assign(map_total_, 0);
    for (const auto& P : pieces_) {
        for (int j = 0; j < P.count; ++j) {
            int c = slot_cell_[P.slot + j];
            int base = m.cptr[c];
            for (int r = 0; r <= k; ++r)
                for (int e = 0; e < P.ne; ++e) {
                    int ge = m.gedges[base + e];
                    int g = r * m.ne + ge;
                    bool rev = m.cnodes[base + e] != m.eend[2 * ge];
                    bool neg = m.eocc[ge] == 2 && rev && r % 2 == 0;
                    map_host_[P.map_off + (long long)(r * P.ne + e) * PIECE + j] = neg ? ~g : g;
                }
            for (int i = 0; i < internal; ++i)
                map_host_[P.map_off + (long long)((k + 1) * P.ne + i) * PIECE + j] = m.ne * (k + 1) + c * internal + i;
        }
    }
}

void Solver::set_problem(int problem_, int bc_) {
    if (problem_ < VG_PROBLEM_SINCOS || problem_ > VG_PROBLEM_ANNULUS) throw Error(VG_EINVAL, "unknown problem");
    if (bc_ != VG_BC_FLUX && bc_ != VG_BC_PRESSURE) throw Error(VG_EINVAL, "unknown boundary condition");
    problem = problem_;
    bc = bc_;
    N = nf + np + (bc == VG_BC_FLUX ? 1 : 0);
    built = false;
}

void Solver::set_theta(const double* theta, bool on_device) {
    if (!theta) throw Error(VG_EINVAL, "null theta");
    // a non-finite log permeability would turn the operator and every solve into NaN: rejected
    // before the handle's field changes
    long long bad = -1;
    if (on_device) {
        VG_CUDA(cudaDeviceSynchronize());  // theta may come from any stream
        bad = first_nonfinite(theta, m.nc);
    } else {
        for (int c = 0; c < m.nc && bad < 0; ++c)
            if (!std::isfinite(theta[c])) bad = c;
    }
    if (bad >= 0) throw Error(VG_EINVAL, "non-finite log permeability in cell " + std::to_string(bad));
    if (on_device)
        VG_CUDA(cudaMemcpy(d_theta_.data(), theta, sizeof(double) * m.nc, cudaMemcpyDeviceToDevice));
    else
        VG_CUDA(cudaMemcpy(d_theta_.data(), theta, sizeof(double) * m.nc, cudaMemcpyHostToDevice));
    if (built) {
        PhaseTimer pt;
        rescale_ops(d_theta_.data(), d_slot_cell_.data(), d_pieces_.data(), int(pieces_.size()), d_A0_.data(),
                    d_A64_.data(), d_A32_.data(), nullptr);
        pack_streams(nullptr);
        pt.mark("rescale + record streams");
        make_diagonal(nullptr);
        lift_flux_rhs();
        VG_CUDA(cudaDeviceSynchronize());
    }
}

void Solver::check_status(const char* where) {
    unsigned long long st = 0;
    VG_CUDA(cudaMemcpy(&st, d_status_.data(), sizeof(st), cudaMemcpyDeviceToHost));
    if (!st) return;
    unsigned long long code = st >> 40;
    int cell = int(st & 0xffffffffull);
    if (code == ST_JACOBIAN)
        throw Error(VG_EGEOMETRY, std::string(where) + ": nonpositive Jacobian in cell " + std::to_string(cell));
    throw Error(VG_ESINGULAR, std::string(where) + ": singular local matrix in cell " + std::to_string(cell));
}

void Solver::build() {
    upload_rules(triangle_rule(nq), gauss_legendre(ng));
    const int nqp = nq;
    d_A0_.resize(a_total_);
    d_A64_.resize(a_total_);
    d_A32_.resize(a_total_);
    d_W64_.resize(std::max<long long>(w_total_, 1));
    d_W32_.resize(std::max<long long>(w_total_, 1));
    d_P_.resize(p_total_);
    d_HW_.resize(hw_total_);
    d_L_.resize(size_t(m.nc) * q);
    d_L32_.resize(size_t(m.nc) * q);
    d_alpha_.resize(m.nc);
    d_rhs_.resize(N);
    d_bval_.resize(N);
    d_mask_.resize(N);
    d_rhs_.zero();
    d_bval_.zero();
    d_mask_.zero();
    d_status_.zero();
    SetupArgs a{};
    a.xy = d_xy_.data();
    a.cptr = d_cptr_.data();
    a.cnodes = d_cnodes_.data();
    a.gedges = d_gedges_.data();
    a.eocc = d_eocc_.data();
    a.cx = d_cx_.data();
    a.cy = d_cy_.data();
    a.diam = d_diam_.data();
    a.triptr = d_triptr_.data();
    a.tris = d_tris_.data();
    a.arc = geom_kind == VG_GEOM_ARCS ? d_arc_.data() : nullptr;
    a.slot_cell = d_slot_cell_.data();
    a.cell_slot = d_cell_slot_.data();
    a.pieces = d_pieces_.data();
    a.map = d_map_.data();
    a.theta = d_theta_.data();
    a.k = k;
    a.q = q;
    a.p = p;
    a.ngrad = ngrad;
    a.internal = internal;
    a.nqp = nqp;
    a.ng = ng;
    a.geom = geom_kind;
    a.problem = problem;
    a.bc = bc;
    a.nf = nf;
    a.eps = eps;
    a.A0 = d_A0_.data();
    a.A64 = d_A64_.data();
    a.A32 = d_A32_.data();
    a.W64 = d_W64_.data();
    a.W32 = d_W32_.data();
    a.P = d_P_.data();
    a.HW = d_HW_.data();
    a.L = d_L_.data();
    a.L32 = d_L32_.data();
    a.alpha = d_alpha_.data();
    a.rhs = d_rhs_.data();
    a.bval = d_bval_.data();
    a.mask = d_mask_.data();
    a.status = d_status_.data();
    setup_args_ = a;
    PhaseTimer pt;
    for (const auto& c : classes_) launch_setup(a, c, nqp, nullptr);
    VG_CUDA(cudaDeviceSynchronize());
    check_status("setup");
    internal_copies();
    pt.mark("device setup kernels");
    pack_streams(nullptr);
    pt.mark("pack record streams");
    // workspaces
    d_partials_.resize(2 * size_t(std::max(apply_blocks(int(pieces_.size())), VEC_BLOCKS)) + 16);
    d_red_.resize(8);
    d_scal_.resize(sizeof(Scalars) / sizeof(double) + 1);
    d_flags_.resize(NFLAGS);
    for (int i = 0; i < 8; ++i) {
        w64_[i].resize(N);
        w32_[i].resize(N);
    }
    d_dinv64_.resize(N);
    d_dinv32_.resize(N);
    destroy_graphs();
    for (auto& b : sv64_) b.resize(N);
    for (auto& b : sv32_) b.resize(N);
    amg_refreshable_ = false;  // a build starts the multigrid from scratch (the system may have changed)
    make_diagonal(nullptr);
    pt.mark("preconditioner (incl. multigrid)");
    // BC_FLUX: lifted right-hand side of MixedGpu::make_rhs (equation_gpu.cu:611-625):
    // free rows b - A g (unconstrained apply of the boundary values), boundary rows g
    d_rhs0_.resize(N);
    VG_CUDA(cudaMemcpy(d_rhs0_.data(), d_rhs_.data(), sizeof(double) * N, cudaMemcpyDeviceToDevice));
    lift_flux_rhs();
    VG_CUDA(cudaDeviceSynchronize());
    built = true;
}

// BC_FLUX: the lifted right-hand side depends on the operator (b - A g), so it is recomputed from
// the unlifted one whenever the permeability changes
void Solver::lift_flux_rhs() {
    if (bc != VG_BC_FLUX) return;
    VG_CUDA(cudaMemcpy(d_rhs_.data(), d_rhs0_.data(), sizeof(double) * N, cudaMemcpyDeviceToDevice));
    double* y = w64_[0].data();
    w64_[0].zero();
    apply64(d_bval_.data(), y, false, 1.0, nullptr);
    lift_rhs(d_mask_.data(), d_bval_.data(), y, d_rhs_.data(), N, nullptr);
}

void Solver::make_diagonal(cudaStream_t s) {
    // SPD block-diagonal preconditioner: flux  diag(A) assembled (1 on masked dofs),
    // pressure sum_i W_ri^2 / diag(A)_i, multiplier sum_E sum_r L_r^2 / S_rr
    // (the diagonal of vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:282-315 with |.| of the Schur part)
    DevBuf<double> contrib(m.nc);
    d_dinv64_.zero(s);
    const int np_ = int(pieces_.size());
    diag_flux(d_A64_.data(), d_map_.data(), d_pieces_.data(), np_, d_dinv64_.data(), s);
    diag_finish(d_W64_.data(), d_map_.data(), d_slot_cell_.data(), bc == VG_BC_FLUX ? d_mask_.data() : nullptr,
                d_L_.data(), d_pieces_.data(), np_, k, nf, d_dinv64_.data(), contrib.data(), s);
    diag_invert(d_dinv64_.data(), bc == VG_BC_FLUX ? d_mask_.data() : nullptr, contrib.data(), m.nc, nf, np,
                bc == VG_BC_FLUX, N, s);
    to_float_plain(d_dinv64_.data(), d_dinv32_.data(), N, s);
    d_pdinv64_.resize(N);
    d_pdinv32_.resize(N);
    gather_launch<double>(d_dinv64_.data(), d_i2e_.data(), 0, d_pdinv64_.data(), N, s);
    gather_launch<float>(d_dinv32_.data(), d_i2e_.data(), 0, d_pdinv32_.data(), N, s);
    VG_CUDA(cudaStreamSynchronize(s));
    if (use_amg && amg_refreshable_) {
        // new operator values on the kept structure: device refresh, same device addresses (the
        // captured Krylov loops stay valid)
        PhaseTimer pt;
        pt.mark("diagonal");
        refresh_amg();
        pt.mark("multigrid refresh");
        return;
    }
    // the captured Krylov loops hold the multigrid hierarchy's device addresses, which the rebuild
    // below frees: drop them (they are captured again by the next solve)
    destroy_graphs();
    use_amg = false;
    amg_refreshable_ = false;
    if (bc == VG_BC_PRESSURE) build_amg();
    if (use_amg) prepare_amg_refresh();
}

// device arrays of the Schur values kernel: cells around every flux dof, cell <-> pressure rank
void Solver::prepare_amg_refresh() {
    std::vector<int> cnt(nf + 1, 0);
    for (int c = 0; c < m.nc; ++c) {
        const int slot = cell_slot_[c];
        const Piece& P = pieces_[slot / PIECE];
        for (int i = 0; i < P.n; ++i) {
            int g = map_host_[P.map_off + (long long)i * PIECE + slot % PIECE];
            cnt[(g < 0 ? ~g : g) + 1]++;
        }
    }
    for (int g = 0; g < nf; ++g) cnt[g + 1] += cnt[g];
    std::vector<int> icell(cnt[nf]), ii(cnt[nf]);
    std::vector<signed char> is(cnt[nf]);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int c = 0; c < m.nc; ++c) {
        const int slot = cell_slot_[c];
        const Piece& P = pieces_[slot / PIECE];
        for (int i = 0; i < P.n; ++i) {
            int g = map_host_[P.map_off + (long long)i * PIECE + slot % PIECE], gg = g < 0 ? ~g : g;
            icell[fill[gg]] = c;
            ii[fill[gg]] = i;
            is[fill[gg]++] = g < 0 ? -1 : 1;
        }
    }
    std::vector<int> rank_cell(m.nc), cell_rank(m.nc);
    for (int c = 0; c < m.nc; ++c) {
        const int rank = (e2i_host_[nf + (long long)c * q] - nf) / q;
        cell_rank[c] = rank;
        rank_cell[rank] = c;
    }
    d_inc_ptr_.upload(cnt);
    d_inc_cell_.upload(icell);
    d_inc_i_.upload(ii);
    d_inc_s_.upload(is);
    d_rank_cell_.upload(rank_cell);
    d_cell_rank_.upload(cell_rank);
    d_schur_vals_.resize(size_t(amg_.level0_nnz()));
    amg_refreshable_ = amg_.level0_nnz() > 0;
}

void Solver::refresh_amg() {
    auto t0 = std::chrono::steady_clock::now();
    VG_CUDA(cudaDeviceSynchronize());
    schur_values(amg_.level0_ptr(), amg_.level0_col(), int(np), q, k, d_rank_cell_.data(), d_cell_rank_.data(),
                 d_cell_slot_.data(), d_pieces_.data(), d_map_.data(), d_W64_.data(), d_dinv64_.data(),
                 d_inc_ptr_.data(), d_inc_cell_.data(), d_inc_i_.data(), d_inc_s_.data(), d_schur_vals_.data());
    amg_.refresh(d_schur_vals_.data());
    amg_setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// pressure rows in the solver's internal order (index minus nf)
std::vector<int> Solver::pressure_order() const {
    std::vector<int> o;
    o.resize(static_cast<size_t>(np));
    for (long long i = 0; i < np; ++i) o[i] = e2i_host_[nf + i] - nf;
    return o;
}

// pressure Schur block S = B diag(A)^{-1} B^T for k >= 1 (B[(E,r), g] = W_E[r,i] s_Ei over the local
// flux dofs i of E with global index g and orientation sign s): q x q blocks between cells that share
// an edge. Its multigrid starts with an injection of the cell means (the m_0 moment) onto the cell
// graph, where the mean-mean block is coarsened by smoothed aggregation as for k = 0.
void Solver::build_amg_high() {
    auto t0 = std::chrono::steady_clock::now();
    std::vector<double> dinv(nf);
    VG_CUDA(cudaMemcpy(dinv.data(), d_dinv64_.data(), sizeof(double) * nf, cudaMemcpyDeviceToHost));
    std::vector<double> W = d_W64_.download();
    // incidences of every flux dof: (cell, local dof, sign), at most two per dof
    struct Inc {
        int cell, i;
        double s;
    };
    std::vector<int> cnt(nf + 1, 0);
    for (int c = 0; c < m.nc; ++c) {
        const int slot = cell_slot_[c];
        const Piece& P = pieces_[slot / PIECE];
        const int lane = slot % PIECE;
        for (int i = 0; i < P.n; ++i) {
            int g = map_host_[P.map_off + (long long)i * PIECE + lane];
            cnt[(g < 0 ? ~g : g) + 1]++;
        }
    }
    for (int g = 0; g < nf; ++g) cnt[g + 1] += cnt[g];
    std::vector<Inc> inc(cnt[nf]);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int c = 0; c < m.nc; ++c) {
        const int slot = cell_slot_[c];
        const Piece& P = pieces_[slot / PIECE];
        const int lane = slot % PIECE;
        for (int i = 0; i < P.n; ++i) {
            int g = map_host_[P.map_off + (long long)i * PIECE + lane];
            int gg = g < 0 ? ~g : g;
            inc[fill[gg]++] = Inc{c, i, g < 0 ? -1.0 : 1.0};
        }
    }
    auto wv = [&](int c, int r, int i) {
        const int slot = cell_slot_[c];
        const Piece& P = pieces_[slot / PIECE];
        return W[P.w_off + (long long)(r * P.n + i) * PIECE + slot % PIECE];
    };
    const int np_ = m.nc * q;
    // row by row with one sparse accumulator: row (E, r) couples to (F, r2) through every flux dof
    // shared by E and F
    HostCsr S;
    S.n = S.m = np_;
    S.ptr.assign(np_ + 1, 0);
    std::vector<double> acc(np_, 0.0);
    std::vector<int> mark(np_, -1), cols;
    for (int c = 0; c < m.nc; ++c) {
        const int slot = cell_slot_[c];
        const Piece& P = pieces_[slot / PIECE];
        const int lane = slot % PIECE;
        for (int r = 0; r < q; ++r) {
            const int row = c * q + r;
            cols.clear();
            for (int i = 0; i < P.n; ++i) {
                const int g0 = map_host_[P.map_off + (long long)i * PIECE + lane];
                const int g = g0 < 0 ? ~g0 : g0;
                const double coef = wv(c, r, i) * (g0 < 0 ? -1.0 : 1.0) * dinv[g];
                if (coef == 0.0) continue;
                for (int b = cnt[g]; b < cnt[g + 1]; ++b) {
                    const Inc& B = inc[b];
                    for (int r2 = 0; r2 < q; ++r2) {
                        const int col = B.cell * q + r2;
                        if (mark[col] != row) {
                            mark[col] = row;
                            acc[col] = 0.0;
                            cols.push_back(col);
                        }
                        acc[col] += coef * wv(B.cell, r2, B.i) * B.s;
                    }
                }
            }
            std::sort(cols.begin(), cols.end());
            for (int col : cols) {
                S.col.push_back(col);
                S.val.push_back(acc[col]);
            }
            S.ptr[row + 1] = int(S.col.size());
        }
    }
    // injection of the cell means: pressure row (E, 0) -> coarse E
    HostCsr P0;
    P0.n = np_;
    P0.m = m.nc;
    P0.ptr.assign(np_ + 1, 0);
    for (int c = 0; c < m.nc; ++c)
        for (int r = 0; r < q; ++r) {
            if (r == 0) {
                P0.col.push_back(c);
                P0.val.push_back(1.0);
            }
            P0.ptr[c * q + r + 1] = int(P0.col.size());
        }
    try {
        const std::vector<int> order = pressure_order();
        amg_.setup(S, &P0, &order);
    } catch (const Error&) {
        use_amg = false;
        amg_levels = 0;
        return;
    }
    amg_levels = amg_.levels();
    use_amg = true;
    amg_setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// pressure Schur block S = W diag(A)^{-1} W^T of the k = 0 system (cell graph: S_EE = sum over the
// edges of E of 1/d_e, S_EF = -1/d_e across the shared edge e) and its multigrid hierarchy
void Solver::build_amg() {
    if (k >= 1) {
        build_amg_high();
        return;
    }
    auto t0 = std::chrono::steady_clock::now();
    std::vector<double> dinv(nf);
    VG_CUDA(cudaMemcpy(dinv.data(), d_dinv64_.data(), sizeof(double) * nf, cudaMemcpyDeviceToHost));
    std::vector<int> ec(2 * size_t(m.ne), -1);
    for (int c = 0; c < m.nc; ++c)
        for (int j = m.cptr[c]; j < m.cptr[c + 1]; ++j) {
            int e = m.gedges[j];
            if (ec[2 * e] < 0)
                ec[2 * e] = c;
            else
                ec[2 * e + 1] = c;
        }
    HostCsr S;
    S.n = S.m = m.nc;
    S.ptr.assign(m.nc + 1, 0);
    std::vector<std::pair<int, double>> row;
    for (int c = 0; c < m.nc; ++c) {
        row.clear();
        double diag = 0;
        for (int j = m.cptr[c]; j < m.cptr[c + 1]; ++j) {
            int e = m.gedges[j];
            double d = dinv[e];
            diag += d;
            int o = ec[2 * e] == c ? ec[2 * e + 1] : ec[2 * e];
            if (o >= 0) row.push_back({o, -d});
        }
        row.push_back({c, diag});
        std::sort(row.begin(), row.end());
        for (size_t i = 0; i < row.size(); ++i) {
            if (i > 0 && row[i].first == row[i - 1].first) {
                S.val.back() += row[i].second;
                continue;
            }
            S.col.push_back(row[i].first);
            S.val.push_back(row[i].second);
        }
        S.ptr[c + 1] = int(S.col.size());
    }
    try {
        const std::vector<int> order = pressure_order();
        amg_.setup(S, nullptr, &order);
    } catch (const Error&) {
        use_amg = false;  // diagonal preconditioner on the device
        amg_levels = 0;
        return;
    }
    amg_levels = amg_.levels();
    use_amg = true;
    amg_setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

template <typename T>
void Solver::apply_int(const T* x, T* y, bool constrained, T psign, cudaStream_t s, double* quad) {
    launch_apply(apply_args<T>(x, y, constrained, psign, quad, nullptr), s);
    n_launch += 1;
    ++n_apply;
}
template void Solver::apply_int<double>(const double*, double*, bool, double, cudaStream_t, double*);
template void Solver::apply_int<float>(const float*, float*, bool, float, cudaStream_t, double*);

// Reference order in and out, in one kernel: the same apply with the dof map, the pressure rows,
// the essential-BC mask and the multiplier vector in the reference's numbering, and (k <= 1) record
// streams packed with that map, built on the first call. The gathers and scatters are less
// coalesced than in the internal order, but no permutation pass runs.
void Solver::prepare_reference_order() {
    if (!d_prow_ref_.data()) {
        std::vector<int> prow(slot_cell_.size(), -1);
        for (size_t j = 0; j < slot_cell_.size(); ++j)
            if (slot_cell_[j] >= 0) prow[j] = nf + slot_cell_[j] * q;
        d_prow_ref_.upload(prow);
    }
    if (k <= 1 && !ref_streams_packed_) {
        d_rec64r_.resize(size_t(plan64_.bytes));
        d_rec32r_.resize(size_t(plan32_.bytes));
        pack_streams_reference(nullptr);
    }
}

void Solver::pack_streams_reference(cudaStream_t s) {
    const int np_ = int(pieces_.size());
    pack_stream<double>(d_pieces_.data(), np_, d_roff64_.data(), d_A64_.data(), d_W64_.data(), d_map_.data(),
                        d_prow_ref_.data(), k, d_rec64r_.data(), s);
    pack_stream<float>(d_pieces_.data(), np_, d_roff32_.data(), d_A32_.data(), d_W32_.data(), d_map_.data(),
                       d_prow_ref_.data(), k, d_rec32r_.data(), s);
    VG_CUDA(cudaStreamSynchronize(s));
    ref_streams_packed_ = true;
}

template <typename T>
void Solver::apply_ref(const T* x, T* y, bool constrained, T psign, cudaStream_t s, double* quad) {
    prepare_reference_order();
    ApplyArgs<T> a = apply_args<T>(x, y, constrained, psign, quad, nullptr);
    a.map = d_map_.data();
    a.prow = d_prow_ref_.data();
    a.mask = d_mask_.data();
    if constexpr (sizeof(T) == 8) {
        a.L = d_L_.data();
        if (a.rec) a.rec = d_rec64r_.data();
    } else {
        a.L = d_L32_.data();
        if (a.rec) a.rec = d_rec32r_.data();
    }
    launch_apply(a, s);
    n_launch += 1;
    ++n_apply;
}

void Solver::apply64(const double* x, double* y, bool constrained, double psign, cudaStream_t s, double* quad) {
    apply_ref<double>(x, y, constrained, psign, s, quad);
}

void Solver::apply32(const float* x, float* y, bool constrained, float psign, cudaStream_t s, double* quad) {
    apply_ref<float>(x, y, constrained, psign, s, quad);
}

void Solver::plan_streams() {
    if (k > 1) return;
    plan64_ = plan_stream(pieces_, k, 8, sm_count_);
    plan32_ = plan_stream(pieces_, k, 4, sm_count_);
    d_rec64_.resize(size_t(plan64_.bytes));
    d_rec32_.resize(size_t(plan32_.bytes));
    d_roff64_.upload(plan64_.rec_off);
    d_roff32_.upload(plan32_.rec_off);
    d_bat64_.upload(plan64_.batches);
    d_bat32_.upload(plan32_.batches);
    d_cta64_.upload(plan64_.cta_batch);
    d_cta32_.upload(plan32_.cta_batch);
    // the apply's error word: mapped pinned host memory, written by a kernel only when a pipeline
    // wait gave up (a plain store) and read by the host with a plain load, no copy in any call
    if (!h_err_) {
        VG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&h_err_), sizeof(int), cudaHostAllocMapped));
        *h_err_ = 0;
        VG_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&d_errp_), h_err_, 0));
    }
    d_stall_.resize(1);
    d_stall_.zero();
    VG_CUDA(cudaDeviceSynchronize());
    prepare_stream_kernels();
}

void Solver::pack_streams(cudaStream_t s) {
    if (k > 1) return;
    const int np_ = int(pieces_.size());
    pack_stream<double>(d_pieces_.data(), np_, d_roff64_.data(), d_A64_.data(), d_W64_.data(), d_map_int_.data(),
                        d_prow_.data(), k, d_rec64_.data(), s);
    pack_stream<float>(d_pieces_.data(), np_, d_roff32_.data(), d_A32_.data(), d_W32_.data(), d_map_int_.data(),
                       d_prow_.data(), k, d_rec32_.data(), s);
    VG_CUDA(cudaStreamSynchronize(s));
    if (ref_streams_packed_) pack_streams_reference(s);  // new operator values (permeability update)
}

// Test hook of the failure path: in the next streamed apply one consumer's bounded wait runs out
// (a barrier nothing arrives on) and the apply reports its error word.
void Solver::inject_apply_stall() {
    if (k > 1 || !d_stall_.data()) throw Error(VG_ESTATE, "no streamed apply on this handle (k > 1)");
    const int one = 1;
    VG_CUDA(cudaMemcpy(d_stall_.data(), &one, sizeof(one), cudaMemcpyHostToDevice));
}

// vg_apply is asynchronous: a failed apply sets the mapped error word when its kernel gives up,
// and the next call on the handle that finds it set reports VG_ECUDA (the caller's stream never
// waits for a check)
void Solver::check_apply_probe() {
    if (h_err_ && *reinterpret_cast<volatile int*>(h_err_)) {
        VG_CUDA(cudaDeviceSynchronize());
        *reinterpret_cast<volatile int*>(h_err_) = 0;
        throw Error(VG_ECUDA, "an earlier vg_apply failed: apply pipeline wait timed out");
    }
}

// the bulk-copy apply sets the error word when a pipeline wait gave up (never in a correct run)
void Solver::check_pipeline() {
    if (amg_.ready() && amg_.failed()) throw Error(VG_ECUDA, "multigrid copy wait timed out");
    if (k > 1) return;
    if (h_err_ && *reinterpret_cast<volatile int*>(h_err_)) {
        VG_CUDA(cudaDeviceSynchronize());
        *reinterpret_cast<volatile int*>(h_err_) = 0;
        throw Error(VG_ECUDA, "apply pipeline wait timed out");
    }
}

void Solver::rhs(double* b, cudaStream_t s) {
    VG_CUDA(cudaMemcpyAsync(b, d_rhs_.data(), sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
}

template <>
MinresVecs<float> Solver::vecs<float>(float* x) {
    return MinresVecs<float>{w32_[0].data(), w32_[1].data(), w32_[2].data(), w32_[3].data(), w32_[4].data(),
                             w32_[5].data(), w32_[6].data(), x, d_pdinv32_.data()};
}

template <>
MinresVecs<double> Solver::vecs<double>(double* x) {
    return MinresVecs<double>{w64_[0].data(), w64_[1].data(), w64_[2].data(), w64_[3].data(), w64_[4].data(),
                              w64_[5].data(), w64_[6].data(), x, d_pdinv64_.data()};
}

template <typename T>
ApplyArgs<T> Solver::apply_args(const T* x, T* y, bool constrained, T psign, double* quad, const int* flags) {
    ApplyArgs<T> a{};
    a.x = x;
    a.y = y;
    if constexpr (sizeof(T) == 8) {
        a.A = d_A64_.data();
        a.W = d_W64_.data();
        a.L = d_Lint_.data();
    } else {
        a.A = d_A32_.data();
        a.W = d_W32_.data();
        a.L = d_Lint32_.data();
    }
    a.map = d_map_int_.data();
    a.prow = d_prow_.data();
    a.pieces = d_pieces_.data();
    a.npieces = int(pieces_.size());
    a.k = k;
    a.mask = d_mask_int_.data();
    a.flags = flags;
    a.nf = nf;
    a.N = N;
    a.psign = psign;
    a.constrained = (constrained && bc == VG_BC_FLUX) ? 1 : 0;
    a.mult = bc == VG_BC_FLUX ? 1 : 0;
    a.partials = d_partials_.data();
    a.counter = d_counter_.data();
    a.red = quad;
    if (k <= 1 && d_errp_) {
        const StreamPlan& pl = sizeof(T) == 8 ? plan64_ : plan32_;
        a.rec = sizeof(T) == 8 ? d_rec64_.data() : d_rec32_.data();
        a.batches = sizeof(T) == 8 ? d_bat64_.data() : d_bat32_.data();
        a.cta_batch = sizeof(T) == 8 ? d_cta64_.data() : d_cta32_.data();
        a.ncta = pl.ncta;
        a.stages = pl.stages;
        a.stage_bytes = pl.stage_bytes;
        a.err = d_errp_;
        a.stall = d_stall_.data();
    }
    return a;
}

// one MINRES iteration: apply (with delta), update + preconditioner + gamma, step
template <typename T>
void Solver::iteration(MinresVecs<T>& v, cudaStream_t s) {
    Scalars* sc = reinterpret_cast<Scalars*>(d_scal_.data());
    int* flags = d_flags_.data();
    const long long plo = use_amg ? nf : 0, phi = use_amg ? nf + np : 0;
    launch_apply(apply_args<T>(v.z_cur, v.y, true, T(-1), &sc->delta, flags), s);
    if (use_amg && phi == N) {
        // the flux rows of the update (bandwidth-bound) run on a second stream beside the pressure
        // rows and the V-cycle (latency-bound); both join before the scalar update
        VG_CUDA(cudaEventRecord(ev_fork_, s));
        VG_CUDA(cudaStreamWaitEvent(side_, ev_fork_, 0));
        minres_update_rows<T>(v, 0, plo, 1, sc, flags, d_partials_.data(), d_counter_.data(), side_, plo, phi);
        VG_CUDA(cudaEventRecord(ev_join_, side_));
        minres_update_rows<T>(v, plo, phi, 0, sc, flags, d_partials_.data(), d_counter_.data(), s, plo, phi);
        amg_.vcycle(v.v_old + nf, v.z_new + nf, s);
        VG_CUDA(cudaStreamWaitEvent(s, ev_join_, 0));
        minres_finish<T>(v.z_new, v.v_old, plo, phi, sc, flags, d_partials_.data(), d_counter_.data(), 0, 0.0, s);
    } else {
        minres_update<T>(v, N, sc, flags, d_partials_.data(), d_counter_.data(), s, plo, phi);
    }
    if (use_amg && phi != N) {
        amg_.vcycle(v.v_old + nf, v.z_new + nf, s);
        minres_finish<T>(v.z_new, v.v_old, plo, phi, sc, flags, d_partials_.data(), d_counter_.data(), 0, 0.0, s);
    }
    minres_step<T>(v, N, sc, flags, s);
    std::swap(v.v_cur, v.v_old);
    std::swap(v.z_cur, v.z_new);
    std::swap(v.w_cur, v.w_old);
}

// the MINRES loop as a CUDA graph: a conditional while node whose body is two iterations (the
// vector roles repeat with period two) followed by the condition kernel; the body count is capped
// on the device, so the loop ends even if the convergence flag is never raised
template <typename T>
void Solver::build_graph(int p, T* x) {
    VG_CUDA(cudaGraphCreate(&graph_[p], 0));
    cudaGraphConditionalHandle h;
    VG_CUDA(cudaGraphConditionalHandleCreate(&h, graph_[p], 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    VG_CUDA(cudaGraphAddNode(&node, graph_[p], nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    VG_CUDA(cudaStreamBeginCaptureToGraph(stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    MinresVecs<T> v = vecs<T>(x);
    const long long saved = amg_.launches;
    try {
        iteration<T>(v, stream_);
        iteration<T>(v, stream_);
        loop_check(h, d_flags_.data(), d_loop_.data(), stream_);
    } catch (...) {
        cudaGraph_t dummy;
        cudaStreamEndCapture(stream_, &dummy);
        throw;
    }
    amg_.launches = saved;
    VG_CUDA(cudaStreamEndCapture(stream_, &body));
    VG_CUDA(cudaGraphInstantiate(&gexec_[p], graph_[p], 0));
}

// MINRES on the symmetric constrained system K_sym x = r (x starts at zero)
template <typename T>
void Solver::minres_t(const T* r, T* x, double tol, int maxit, int check_every, int& iters, cudaStream_t s) {
    Scalars* sc = reinterpret_cast<Scalars*>(d_scal_.data());
    int* flags = d_flags_.data();
    const int p = sizeof(T) == 4 ? 1 : 0;
    const long long plo = use_amg ? nf : 0, phi = use_amg ? nf + np : 0;
    const bool graph = check_every <= 0;
    if (graph && !gexec_[p]) build_graph<T>(p, x);
    MinresVecs<T> v = vecs<T>(x);
    VG_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * N, s));
    minres_init<T>(r, v, N, sc, flags, tol, d_partials_.data(), d_counter_.data(), s, plo, phi);
    if (use_amg) {
        amg_.vcycle(v.v_cur + nf, v.z_cur + nf, s);
        minres_finish<T>(v.z_cur, v.v_cur, plo, phi, sc, flags, d_partials_.data(), d_counter_.data(), 1, tol, s);
    }
    int h_flags[NFLAGS] = {0, 0, 0, 0};
    if (graph) {
        int loop[2] = {0, (maxit + 1) / 2};
        VG_CUDA(cudaMemcpyAsync(d_loop_.data(), loop, sizeof(loop), cudaMemcpyHostToDevice, s));
        VG_CUDA(cudaGraphLaunch(gexec_[p], s));
        VG_CUDA(cudaMemcpyAsync(h_flags, flags, sizeof(h_flags), cudaMemcpyDeviceToHost, s));
        VG_CUDA(cudaStreamSynchronize(s));
    } else {
        // host-driven batches of check_every iterations (every kernel is a plain launch)
        for (int done = 0; done < maxit;) {
            int batch = std::min(check_every, maxit - done);
            for (int it = 0; it < batch; ++it) iteration<T>(v, s);
            done += batch;
            VG_CUDA(cudaMemcpyAsync(h_flags, flags, sizeof(h_flags), cudaMemcpyDeviceToHost, s));
            VG_CUDA(cudaStreamSynchronize(s));
            if (h_flags[0]) break;
        }
    }
    iters = h_flags[2];
    // kernels per iteration: apply, update (flux and pressure rows apart with multigrid), step, and
    // with multigrid the composite V-cycle (residual, restriction and prolongation per level, the
    // dense coarsest product) and the finish
    const long long plo_hi = use_amg ? nf + np : 0;
    const long long vc = use_amg ? 3LL * (amg_levels - 1) + 1 : 0;
    const long long upd = (use_amg && plo_hi == N) ? 2 : 1;
    const long long per = 2 + upd + (use_amg ? vc + 1 : 0);
    n_launch += 2 + (use_amg ? vc + 1 : 0) + per * iters + (iters + 2) / 2;
    n_apply += iters;
    n_iter += iters;
}

void Solver::minres(bool fp32, const void* r, void* x, double tol, int maxit, int check_every, int& iters,
                    cudaStream_t s) {
    if (fp32)
        minres_t<float>(static_cast<const float*>(r), static_cast<float*>(x), tol, maxit, check_every, iters, s);
    else
        minres_t<double>(static_cast<const double*>(r), static_cast<double*>(x), tol, maxit, check_every, iters, s);
}

void Solver::solve(const double* b, double* x, const vg_solve_opts& o, vg_solve_info& info, cudaStream_t s) {
    if (!built) throw Error(VG_ESTATE, "vg_build must run before vg_solve");
    if (!b || !x) throw Error(VG_EINVAL, "null vector");
    if (!(o.tol > 0) || o.maxit < 1 || o.check_every < 0 || (o.mode == VG_SOLVE_MIXED && !(o.inner_tol > 0 && o.inner_tol < 1)))
        throw Error(VG_EINVAL, "invalid solve options");
    info = vg_solve_info{};
    (void)s;
    s = stream_;
    // order after the caller's work on the legacy default stream
    VG_CUDA(cudaEventRecord(ev_in_, nullptr));
    VG_CUDA(cudaStreamWaitEvent(s, ev_in_, 0));
    VG_CUDA(cudaEventRecord(ev0_, s));
    const bool cons = bc == VG_BC_FLUX;
    // symmetric form: pressure / multiplier rows negated
    DevBuf<double>&bs = sv64_[0], &r = sv64_[1], &y = sv64_[2], &d = sv64_[3];
    // the Krylov solve runs in the internal order: b and the initial x are permuted in, x out
    double* const x_ext = x;
    x = d_xi_.data();
    permute<double>(b, bs.data(), true, s);
    flip_pressure(bs.data(), bs.data(), nf, N, s);
    n_launch += 2;
    ++n_solve;
    if (o.nonzero_guess)
        permute<double>(x_ext, x, true, s);
    else
        VG_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * N, s));
    double h_red[2] = {0, 0};
    // zero_x: x is the zero initial guess, K x = 0 and r = b without an apply
    auto true_residual = [&](bool zero_x = false) {
        y.zero(s);
        if (!zero_x) apply_int<double>(x, y.data(), cons, -1.0, s, nullptr);
        residual64(bs.data(), y.data(), r.data(), N, d_red_.data(), d_partials_.data(), d_counter_.data(), s);
        n_launch += 1;
        VG_CUDA(cudaMemcpyAsync(h_red, d_red_.data(), sizeof(h_red), cudaMemcpyDeviceToHost, s));
        VG_CUDA(cudaStreamSynchronize(s));
        double nb = std::sqrt(h_red[1]);
        return std::sqrt(h_red[0]) / (nb > 0 ? nb : 1.0);
    };
    double rel = true_residual(!o.nonzero_guess);
    int total = 0, outer = 0;
    const double nb = std::sqrt(h_red[1]) > 0 ? std::sqrt(h_red[1]) : 1.0;
    if (o.mode == VG_SOLVE_FP64) {
        // MINRES in FP64 to 0.1 tol (the reference's KSP tolerance factor, krylov.cu:142), then the
        // true FP64 residual decides; at most two restarts from the current iterate (krylov.cu:136-170)
        for (outer = 0; outer < 3 && rel > o.tol && total < o.maxit; ++outer) {
            int it = 0;
            double rn = rel * nb;
            minres(false, r.data(), d.data(), std::min(0.5, 0.1 * o.tol * nb / rn), o.maxit - total, o.check_every, it, s);
            total += it;
            axpy64(x, d.data(), 1.0, s);
            n_launch += 1;
            rel = true_residual();
        }
    } else {
        DevBuf<float>&r32 = sv32_[0], &d32 = sv32_[1];
        for (outer = 0; outer < o.max_outer && rel > o.tol && total < o.maxit; ++outer) {
            double rn = rel * nb;
            to_float(r.data(), r32.data(), 1.0 / rn, N, s);
            n_launch += 2;
            int it = 0;
            // reduction asked of this FP32 solve: inner_tol, or less when less reaches tol (with the
            // same 0.1 margin as the FP64 path)
            const double itol = std::min(0.5, std::max(o.inner_tol, 0.1 * o.tol / rel));
            minres(true, r32.data(), d32.data(), itol, o.maxit - total, o.check_every, it, s);
            total += it;
            axpy_from_float(x, d32.data(), rn, N, s);
            rel = true_residual();
        }
    }
    permute<double>(x, x_ext, false, s);
    VG_CUDA(cudaEventRecord(ev1_, s));
    VG_CUDA(cudaEventSynchronize(ev1_));
    check_pipeline();
    float ms = 0;
    VG_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    info.iterations = total;
    info.outer = outer;
    info.residual = rel;
    info.seconds = ms * 1e-3;
    if (!(rel <= o.tol))
        throw Error(VG_ENOCONV, "Krylov solve did not converge: iterations=" + std::to_string(total) +
                                    " true_relative_residual=" + std::to_string(rel));
}

void Solver::solve_host(const double* b_host, double* x_host, const vg_solve_opts& o, vg_solve_info& info) {
    if (!built) throw Error(VG_ESTATE, "vg_build must run before vg_solve_host");
    d_hb_.resize(N);
    d_hx_.resize(N);
    // copies on the solver stream: solve() orders its own work after the legacy stream, so the
    // inputs are enqueued there first
    VG_CUDA(cudaMemcpyAsync(d_hb_.data(), b_host, sizeof(double) * N, cudaMemcpyHostToDevice, nullptr));
    if (o.nonzero_guess)
        VG_CUDA(cudaMemcpyAsync(d_hx_.data(), x_host, sizeof(double) * N, cudaMemcpyHostToDevice, nullptr));
    solve(d_hb_.data(), d_hx_.data(), o, info, nullptr);
    VG_CUDA(cudaMemcpyAsync(x_host, d_hx_.data(), sizeof(double) * N, cudaMemcpyDeviceToHost, stream_));
    VG_CUDA(cudaStreamSynchronize(stream_));
}

// sparsity pattern of the assembled system (host, cached): row g of a flux dof holds the dofs of
// the cells around g, a pressure row the dofs of its cell, the multiplier row every pressure dof;
// every row holds its diagonal (the unit diagonal of masked rows)
void Solver::assembled_pattern() {
    if (!csr_ptr_.empty()) return;
    const bool mult = bc == VG_BC_FLUX;
    auto dofs_of = [&](int c, std::vector<int>& out) {
        const int slot = cell_slot_[c];
        const Piece& P = pieces_[slot / PIECE];
        const int lane = slot % PIECE;
        for (int i = 0; i < P.n; ++i) {
            int g = map_host_[P.map_off + (long long)i * PIECE + lane];
            out.push_back(g < 0 ? ~g : g);
        }
        for (int r = 0; r < q; ++r) out.push_back(nf + c * q + r);
        if (mult) out.push_back(N - 1);
    };
    // cells around every flux dof
    std::vector<int> cnt(nf + 1, 0), cells;
    std::vector<int> tmp;
    for (int c = 0; c < m.nc; ++c) {
        tmp.clear();
        dofs_of(c, tmp);
        for (int g : tmp)
            if (g < nf) cnt[g + 1]++;
    }
    for (int g = 0; g < nf; ++g) cnt[g + 1] += cnt[g];
    cells.assign(cnt[nf], 0);
    {
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        for (int c = 0; c < m.nc; ++c) {
            tmp.clear();
            dofs_of(c, tmp);
            for (int g : tmp)
                if (g < nf) cells[fill[g]++] = c;
        }
    }
    csr_ptr_.assign(size_t(N) + 1, 0);
    csr_col_.clear();
    std::vector<int> row;
    auto emit = [&](long long r) {
        row.push_back(int(r));
        std::sort(row.begin(), row.end());
        row.erase(std::unique(row.begin(), row.end()), row.end());
        csr_col_.insert(csr_col_.end(), row.begin(), row.end());
        csr_ptr_[r + 1] = (long long)csr_col_.size();
    };
    for (int g = 0; g < nf; ++g) {
        row.clear();
        for (int t = cnt[g]; t < cnt[g + 1]; ++t) dofs_of(cells[t], row);
        emit(g);
    }
    for (int c = 0; c < m.nc; ++c)
        for (int r = 0; r < q; ++r) {
            row.clear();
            dofs_of(c, row);
            emit(nf + (long long)c * q + r);
        }
    if (mult) {
        row.clear();
        for (long long i = nf; i < nf + np; ++i) row.push_back(int(i));
        emit(N - 1);
    }
}

void Solver::assemble(int constrained, long long* nnz, long long* rp, int* ci, double* val) {
    if (!built) throw Error(VG_ESTATE, "vg_build must run before vg_assemble_csr");
    assembled_pattern();
    *nnz = (long long)csr_col_.size();
    if (!rp) return;
    if (!ci || !val) throw Error(VG_EINVAL, "vg_assemble_csr needs row_ptr, col_idx and values");
    VG_CUDA(cudaMemcpy(rp, csr_ptr_.data(), sizeof(long long) * csr_ptr_.size(), cudaMemcpyHostToDevice));
    VG_CUDA(cudaMemcpy(ci, csr_col_.data(), sizeof(int) * csr_col_.size(), cudaMemcpyHostToDevice));
    VG_CUDA(cudaMemset(val, 0, sizeof(double) * csr_col_.size()));
    DevBuf<int> bad(1);
    bad.zero();
    assemble_values(d_A64_.data(), d_W64_.data(), d_map_.data(), d_slot_cell_.data(), d_mask_.data(), d_L_.data(),
                    d_pieces_.data(), int(pieces_.size()), k, nf, N, (constrained && bc == VG_BC_FLUX) ? 1 : 0,
                    bc == VG_BC_FLUX ? 1 : 0, rp, ci, val, bad.data(), nullptr);
    int b = 0;
    VG_CUDA(cudaMemcpy(&b, bad.data(), sizeof(int), cudaMemcpyDeviceToHost));
    if (b) throw Error(VG_ESTATE, "assembled pattern does not hold an entry of a local block");
}

void Solver::axpy64(double* x, const double* d, double a, cudaStream_t s) {
    axpy64_kernel_launch(x, d, a, N, s);
}

void Solver::adjoint(const double* x, const double* dJdx, double* g, const vg_solve_opts& o, vg_solve_info& info,
                     cudaStream_t s) {
    if (!built) throw Error(VG_ESTATE, "vg_build must run before vg_adjoint_grad");
    // K_ref^T lambda = dJ/dx  <=>  K_sym mu = dJ/dx with mu = S lambda (S = diag(I, -I));
    // solve() takes a reference-sign right-hand side b and solves K_sym x = S b, so pass S dJ/dx
    d_adj_rhs_.resize(N);
    d_adj_mu_.resize(N);
    DevBuf<double>&rhs = d_adj_rhs_, &mu = d_adj_mu_;
    flip_pressure(dJdx, rhs.data(), nf, N, nullptr);  // legacy stream: solve() orders after it
    vg_solve_opts oo = o;
    oo.nonzero_guess = 0;
    solve(rhs.data(), mu.data(), oo, info, s);
    s = stream_;
    // dJ/dtheta_E = -lambda^T (dK/dtheta_E) x = mu_u,E^T A_E(theta) x_u,E  (dA_E/dtheta_E = -A_E)
    contract_adjoint(d_A64_.data(), d_map_.data(), d_slot_cell_.data(), d_mask_.data(), d_pieces_.data(),
                     int(pieces_.size()), k, x, mu.data(), bc == VG_BC_FLUX, g, s);
    VG_CUDA(cudaStreamSynchronize(s));
}

void Solver::errors(const double* x, double out[6], cudaStream_t s) {
    if (!built) throw Error(VG_ESTATE, "vg_build must run before vg_errors");
    DevBuf<double> per(6 * size_t(m.nc)), sum(6);
    for (const auto& c : classes_) launch_errors(setup_args_, c, nq, x, per.data(), s);
    launch_error_sum(per.data(), m.nc, sum.data(), s);
    VG_CUDA(cudaMemcpyAsync(out, sum.data(), 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
    VG_CUDA(cudaStreamSynchronize(s));
}

namespace {
// Per-cell error figures (6 doubles a cell) and their sums for Solver::errors_static. Every word
// of the used part is overwritten by each call (error_kernel writes all six figures of every
// cell, error_sum_kernel all six sums), so nothing has to be cleared between calls. Shared by all
// handles of a device: calls that overlap on the GPU race on it.
constexpr long long kErrScratch = 6LL * VG_ERRORS_NOALLOC_MAX_CELLS + 8;
static __device__ __align__(256) double g_err_scratch[kErrScratch];

// device address of g_err_scratch on the current device. Looked up on every call (the lookup
// allocates nothing and is cheap): an address kept across calls would go stale when the device's
// primary context is reset and created again in the same process.
double* err_scratch() {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_err_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        throw Error(VG_ECUDA, std::string("cudaGetSymbolAddress(error scratch): ") + cudaGetErrorString(e));
    }
    return static_cast<double*>(p);
}
}  // namespace

// The C ABI makes the handle's device current before this runs (DeviceScope in vg_capi.cu).
void Solver::errors_static(const double* x, double out[6]) {
    if (!built) throw Error(VG_ESTATE, "vg_build must run before vg_errors_noalloc");
    if (m.nc > VG_ERRORS_NOALLOC_MAX_CELLS)
        throw Error(VG_EINVAL, "vg_errors_noalloc: " + std::to_string(m.nc) +
                                   " cells exceed the static scratch limit VG_ERRORS_NOALLOC_MAX_CELLS = " +
                                   std::to_string(VG_ERRORS_NOALLOC_MAX_CELLS));
    double* per = err_scratch();
    double* sum = per + 6LL * VG_ERRORS_NOALLOC_MAX_CELLS;
    for (const auto& c : classes_) launch_errors(setup_args_, c, nq, x, per, nullptr);
    launch_error_sum(per, m.nc, sum, nullptr);
    VG_CUDA(cudaMemcpyAsync(out, sum, 6 * sizeof(double), cudaMemcpyDeviceToHost, nullptr));
    VG_CUDA(cudaStreamSynchronize(nullptr));
}

int Solver::local(int cell, int which, double* out) {
    if (!built) throw Error(VG_ESTATE, "vg_build must run before vg_local");
    if (cell < 0 || cell >= m.nc) throw Error(VG_EINVAL, "cell out of range");
    int slot = cell_slot_[cell];
    const Piece& b = pieces_[slot / PIECE];
    long long j = slot % PIECE, mcount = PIECE;
    int n = b.n;
    auto strided = [&](const double* base, long long off, int cnt, std::vector<double>& v) {
        v.resize(cnt);
        for (int e = 0; e < cnt; ++e)
            VG_CUDA(cudaMemcpy(&v[e], base + off + e * mcount + j, sizeof(double), cudaMemcpyDeviceToHost));
    };
    std::vector<double> v;
    switch (which) {
    case 0: {
        std::vector<double> pk;
        strided(d_A64_.data(), b.a_off, n * (n + 1) / 2, pk);
        v.assign(size_t(n) * n, 0.0);
        int e = 0;
        for (int i = 0; i < n; ++i)
            for (int c = i; c < n; ++c) {
                v[size_t(i) * n + c] = pk[e];
                v[size_t(c) * n + i] = pk[e];
                ++e;
            }
        break;
    }
    case 1:
        if (k == 0)
            v.assign(n, 1.0);
        else
            strided(d_W64_.data(), b.w_off, q * n, v);
        break;
    case 2: strided(d_P_.data(), b.p_off, p * n, v); break;
    case 3: {
        double a = 0;
        VG_CUDA(cudaMemcpy(&a, d_alpha_.data() + cell, sizeof(double), cudaMemcpyDeviceToHost));
        v.assign(1, a);
        break;
    }
    case 4: {
        v.resize(n);
        for (int i = 0; i < n; ++i) {
            int g = map_host_[b.map_off + i * mcount + j];
            v[i] = g < 0 ? -double(~g + 1) : double(g + 1);
        }
        break;
    }
    case 5: {
        v.resize(q);
        VG_CUDA(cudaMemcpy(v.data(), d_rhs_.data() + nf + (long long)cell * q, q * sizeof(double), cudaMemcpyDeviceToHost));
        break;
    }
    case 6: {
        v.assign(n, 0.0);
        if (bc == VG_BC_PRESSURE)
            for (int i = 0; i < (k + 1) * b.ne; ++i) {
                int g = map_host_[b.map_off + i * mcount + j];
                int e = m.gedges[m.cptr[cell] + i % b.ne];
                if (m.eocc[e] == 1)
                    VG_CUDA(cudaMemcpy(&v[i], d_rhs_.data() + g, sizeof(double), cudaMemcpyDeviceToHost));
            }
        break;
    }
    default: throw Error(VG_EINVAL, "unknown local quantity");
    }
    if (out) std::copy(v.begin(), v.end(), out);
    return int(v.size());
}

}  // namespace vg
