// Isothermal ternary Maxwell-Stefan diffusion, mixed VEM (k = 0), backward Euler: one coupled
// two-species saddle-point system per step,
//     [B(x^n)_E (x) A_E, -W^T; W, (|E|/dt) I] [J; x^{n+1}] = [0; (|E|/dt) x^n],
// with x = (x1, x2) the cell mole fractions (x3 = 1 - x1 - x2), J = (J1, J2) the species fluxes,
// no flux through the boundary (essential J.n = 0), and B the reduced Maxwell-Stefan friction
// matrix of -grad x = B J (molar-average reference, total concentration 1):
//     B_ii = x_i / D_i3 + sum_{k != i} x_k / D_ik,   B_ij = -x_i (1/D_ij - 1/D_i3)   (i, j in {1, 2}).
// A_E is the K = I local flux operator of the Darcy path (projector + stabilisation), W the cell
// divergence (W = 1 per local edge moment at k = 0). The reference treats all three species with a
// regularised coupling and Picard iterations (vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:111-146,
// include/problem_device.cuh:12-28, src/solver_driver.cpp:202-240); here the third species is
// eliminated and B is frozen at x^n (one linear solve per step).
//
// B is not symmetric, so the system is solved by right-preconditioned GMRES(m) (classical
// Gram-Schmidt applied twice, device vectors, Hessenberg and Givens rotations on the host), FP64 or
// FP32 inner under FP64 iterative refinement, with a block-diagonal preconditioner: the 2x2 species
// block of the assembled flux diagonal per flux dof, and for each species one smoothed-aggregation
// V-cycle on its pressure Schur block (|E|/dt) I + W diag(F^{-1})_ss W^T (without the hierarchy:
// the 2x2 cell blocks (|E|/dt) I + sum_i F_{g_i}^{-1}). The hierarchy is built from the first state
// stepped after configuration and kept (a fixed preconditioner for GMRES).
#include <algorithm>
#include <cmath>

#include "vg_apply.cuh"
#include "vg_solver.hpp"

namespace vg {

namespace {

constexpr int MS_THREADS = 256;
constexpr int MS_BLOCKS = 148 * 4;
constexpr int MS_MAXM = 32;  // restart length + 1 (columns of the Krylov basis)

inline int ms_blocks(long long n) { return int(std::min<long long>((n + MS_THREADS - 1) / MS_THREADS, 1 << 20)); }

__device__ __forceinline__ bool ms_slot(const Piece* pieces, int npieces, Piece& P, int& lane) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int pc = int(t / PIECE);
    lane = int(t % PIECE);
    if (pc >= npieces) return false;
    P = pieces[pc];
    return lane < P.count;
}

__device__ __forceinline__ int packed_index(int i, int j, int n) {  // i <= j
    return i * n - i * (i - 1) / 2 + (j - i);
}

__device__ __forceinline__ void red_add_t(float* p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void red_add_t(double* p, double v) { atomicAdd(p, v); }

// B per cell from the cell mole fractions of the state (x1 at xofs, x2 at xofs + nc)
__global__ void k_ms_coeff(const double* state, long long xofs, int nc, double i12, double i13, double i23,
                           double* B64, float* B32) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const double x1 = state[xofs + c], x2 = state[xofs + nc + c], x3 = 1.0 - x1 - x2;
        const double b[4] = {x1 * i13 + x2 * i12 + x3 * i13, -x1 * (i12 - i13), -x2 * (i12 - i23),
                             x2 * i23 + x1 * i12 + x3 * i23};
        for (int z = 0; z < 4; ++z) {
            B64[4LL * c + z] = b[z];
            B32[4LL * c + z] = float(b[z]);
        }
    }
}

template <typename T>
struct MsArgs {
    const T* x;
    T* y;            // flux entries zero on entry
    const T* A;      // K = I packed local operators, piece layout
    const int* map;
    const int* slot_cell;
    const Piece* pieces;
    int npieces, nc;
    long long nf;
    const T* B;      // 4 per cell
    const T* mdt;    // |E| / dt per cell
    const int* mask; // boundary flux dofs (J.n = 0)
};

// y = K x; one lane per cell, both species; masked flux rows are identity rows
template <typename T>
__global__ void __launch_bounds__(MS_THREADS) k_ms_apply(MsArgs<T> a) {
    Piece P;
    int lane;
    if (!ms_slot(a.pieces, a.npieces, P, lane)) return;
    const int n = P.n;
    const int cell = a.slot_cell[P.slot + lane];
    int g[MAX_NE];
    T u0[MAX_NE], u1[MAX_NE], y0[MAX_NE], y1[MAX_NE];
    for (int i = 0; i < n; ++i) {
        int gi = a.map[P.map_off + (long long)i * PIECE + lane];
        g[i] = gi;
        int idx = gi < 0 ? ~gi : gi;
        T s = gi < 0 ? T(-1) : T(1);
        bool m = a.mask[idx] != 0;
        u0[i] = m ? T(0) : s * a.x[idx];
        u1[i] = m ? T(0) : s * a.x[a.nf + idx];
        y0[i] = T(0);
        y1[i] = T(0);
    }
    const T* Ap = a.A + P.a_off + lane;
    for (int i = 0; i < n; ++i)
        for (int c = i; c < n; ++c) {
            const T v = Ap[(long long)packed_index(i, c, n) * PIECE];
            y0[i] += v * u0[c];
            y1[i] += v * u1[c];
            if (c != i) {
                y0[c] += v * u0[i];
                y1[c] += v * u1[i];
            }
        }
    const T b00 = a.B[4LL * cell], b01 = a.B[4LL * cell + 1], b10 = a.B[4LL * cell + 2], b11 = a.B[4LL * cell + 3];
    const long long p0 = 2 * a.nf + cell, p1 = 2 * a.nf + a.nc + cell;
    const T pr0 = a.x[p0], pr1 = a.x[p1];
    T d0 = T(0), d1 = T(0);
    for (int i = 0; i < n; ++i) {
        const int idx = g[i] < 0 ? ~g[i] : g[i];
        const T s = g[i] < 0 ? T(-1) : T(1);
        d0 += u0[i];
        d1 += u1[i];
        if (a.mask[idx]) {
            a.y[idx] = a.x[idx];
            a.y[a.nf + idx] = a.x[a.nf + idx];
        } else {
            red_add_t(a.y + idx, s * (b00 * y0[i] + b01 * y1[i] - pr0));
            red_add_t(a.y + a.nf + idx, s * (b10 * y0[i] + b11 * y1[i] - pr1));
        }
    }
    const T m = a.mdt[cell];
    a.y[p0] = d0 + m * pr0;
    a.y[p1] = d1 + m * pr1;
}

// preconditioner: assembled 2x2 flux blocks D_g = sum_E A_E,ii B_E (at most two addends per dof)
__global__ void k_ms_pc_flux(const double* A, const int* map, const Piece* pieces, int npieces, const int* slot_cell,
                             const double* B, const int* mask, double* D) {
    Piece P;
    int lane;
    if (!ms_slot(pieces, npieces, P, lane)) return;
    const int cell = slot_cell[P.slot + lane];
    for (int i = 0; i < P.n; ++i) {
        int gi = map[P.map_off + (long long)i * PIECE + lane], idx = gi < 0 ? ~gi : gi;
        if (mask[idx]) continue;
        const double aii = A[P.a_off + (long long)packed_index(i, i, P.n) * PIECE + lane];
        for (int z = 0; z < 4; ++z) atomicAdd(D + 4LL * idx + z, aii * B[4LL * cell + z]);
    }
}

__device__ __forceinline__ void inv2(const double* m, double* o) {
    const double det = m[0] * m[3] - m[1] * m[2];
    const double id = det != 0.0 ? 1.0 / det : 0.0;
    o[0] = m[3] * id;
    o[1] = -m[1] * id;
    o[2] = -m[2] * id;
    o[3] = m[0] * id;
}

__global__ void k_ms_pc_flux_inv(const double* D, const int* mask, long long nf, double* F64, float* F32) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < nf; g += (long long)gridDim.x * blockDim.x) {
        double o[4] = {1, 0, 0, 1};
        if (!mask[g]) inv2(D + 4 * g, o);
        for (int z = 0; z < 4; ++z) {
            F64[4 * g + z] = o[z];
            F32[4 * g + z] = float(o[z]);
        }
    }
}

__global__ void k_ms_pc_cell(const int* map, const Piece* pieces, int npieces, const int* slot_cell, const int* mask,
                             const double* F, const double* mdt, double* C64, float* C32) {
    Piece P;
    int lane;
    if (!ms_slot(pieces, npieces, P, lane)) return;
    const int cell = slot_cell[P.slot + lane];
    double s[4] = {mdt[cell], 0, 0, mdt[cell]};
    for (int i = 0; i < P.n; ++i) {
        int gi = map[P.map_off + (long long)i * PIECE + lane], idx = gi < 0 ? ~gi : gi;
        if (mask[idx]) continue;
        for (int z = 0; z < 4; ++z) s[z] += F[4LL * idx + z];
    }
    double o[4];
    inv2(s, o);
    for (int z = 0; z < 4; ++z) {
        C64[4LL * cell + z] = o[z];
        C32[4LL * cell + z] = float(o[z]);
    }
}

template <typename T>
__global__ void k_ms_pc_apply(const T* r, T* z, const T* F, const T* C, long long nf, int nc) {
    const long long n = nf + nc;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        long long i0, i1;
        const T* m;
        if (t < nf) {
            i0 = t;
            i1 = nf + t;
            m = F + 4 * t;
        } else {
            const long long c = t - nf;
            i0 = 2 * nf + c;
            i1 = 2 * nf + nc + c;
            m = C + 4 * c;
        }
        const T a = r[i0], b = r[i1];
        z[i0] = m[0] * a + m[1] * b;
        z[i1] = m[2] * a + m[3] * b;
    }
}

// partial dot products of w with the first cnt columns of V (column stride ld), one row of
// MS_MAXM partials per block
// (with self: w.w in slot cnt, cnt < MS_MAXM)
template <typename T>
__global__ void __launch_bounds__(MS_THREADS) k_mdot(const T* V, long long ld, int cnt, const T* w, long long n,
                                                     double* partials, int self) {
    double acc[MS_MAXM];
#pragma unroll
    for (int k = 0; k < MS_MAXM; ++k) acc[k] = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double wi = double(w[i]);
#pragma unroll
        for (int k = 0; k < MS_MAXM; ++k) {
            if (k < cnt) acc[k] += double(V[k * ld + i]) * wi;
            if (self && k == cnt) acc[k] += wi * wi;
        }
    }
    cnt += self;
    __shared__ double sh[MS_THREADS / 32][MS_MAXM];
    const int wid = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < MS_MAXM; ++k) {
        if (k >= cnt) break;
        double v = acc[k];
        for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (l == 0) sh[wid][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < cnt) {
        double s = 0;
        for (int q = 0; q < MS_THREADS / 32; ++q) s += sh[q][threadIdx.x];
        partials[(long long)blockIdx.x * MS_MAXM + threadIdx.x] = s;
    }
}

__global__ void k_mdot_finish(const double* partials, int nb, int cnt, double* out) {
    const int k = threadIdx.x;
    if (k >= cnt) return;
    double s = 0;
    for (int b = 0; b < nb; ++b) s += partials[(long long)b * MS_MAXM + k];
    out[k] = s;
}

// w -= sum_k h[k] V[:, k]
template <typename T>
__global__ void k_gs_update(const T* V, long long ld, int cnt, const double* h, T* w, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        T s = T(0);
        for (int k = 0; k < cnt; ++k) s += T(h[k]) * V[k * ld + i];
        w[i] -= s;
    }
}

template <typename T>
__global__ void k_scale_to(const T* w, double a, T* v, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = T(a * double(w[i]));
}

// t = sum_k y[k] V[:, k]
template <typename T>
__global__ void k_combine(const T* V, long long ld, int cnt, const double* y, T* t, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = 0; k < cnt; ++k) s += y[k] * double(V[k * ld + i]);
        t[i] = T(s);
    }
}

template <typename T>
__global__ void k_axpy_t(T* x, const T* d, double a, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] += T(a * double(d[i]));
}

__global__ void k_ms_rhs(const double* old_state, const double* mdt, long long nf, int nc, double* b) {
    const long long n = 2 * nf + 2LL * nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (i < 2 * nf) {
            b[i] = 0.0;
        } else {
            const int c = int((i - 2 * nf) % nc);
            b[i] = mdt[c] * old_state[i];
        }
    }
}

__global__ void k_ms_mdt(const double* L, int nc, double dt, double* m64, float* m32) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        m64[c] = L[c] / dt;
        m32[c] = float(L[c] / dt);
    }
}

__global__ void k_d2f(const double* in, float* out, long long n, double scale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = float(scale * in[i]);
}

__global__ void k_sub(const double* b, const double* y, double* r, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        r[i] = b[i] - y[i];
}

__global__ void k_addf(double* x, const float* d, double a, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] += a * double(d[i]);
}

}  // namespace

void Solver::ms_configure(double d12, double d13, double d23, double dt) {
    if (!built) throw Error(VG_ESTATE, "vg_build must run before vg_ms_configure");
    if (k != 0) throw Error(VG_EINVAL, "Maxwell-Stefan is implemented for k = 0");
    if (bc != VG_BC_FLUX)
        throw Error(VG_EINVAL, "Maxwell-Stefan needs the no-flux boundary (build the handle with VG_BC_FLUX)");
    if (!(d12 > 0 && d13 > 0 && d23 > 0 && dt > 0)) throw Error(VG_EINVAL, "diffusivities and dt must be positive");
    ms_.i12 = 1.0 / d12;
    ms_.i13 = 1.0 / d13;
    ms_.i23 = 1.0 / d23;
    ms_.dt = dt;
    ms_.N = 2LL * nf + 2LL * m.nc;
    const long long Nm = ms_.N;
    ms_.B64.resize(4 * size_t(m.nc));
    ms_.B32.resize(4 * size_t(m.nc));
    ms_.F64.resize(4 * size_t(nf));
    ms_.F32.resize(4 * size_t(nf));
    ms_.C64.resize(4 * size_t(m.nc));
    ms_.C32.resize(4 * size_t(m.nc));
    ms_.D.resize(4 * size_t(nf));
    ms_.m64.resize(m.nc);
    ms_.m32.resize(m.nc);
    ms_.A32.resize(a_total_);
    k_d2f<<<MS_BLOCKS, MS_THREADS>>>(d_A0_.data(), ms_.A32.data(), a_total_, 1.0);
    k_ms_mdt<<<ms_blocks(m.nc), MS_THREADS>>>(d_L_.data(), m.nc, dt, ms_.m64.data(), ms_.m32.data());
    VG_CUDA(cudaGetLastError());
    ms_.V64.resize(size_t(MS_MAXM) * Nm);
    ms_.V32.resize(size_t(MS_MAXM) * Nm);
    for (auto* b : {&ms_.b, &ms_.r, &ms_.y, &ms_.d, &ms_.t64}) b->resize(Nm);
    for (auto* b : {&ms_.r32, &ms_.d32, &ms_.t32, &ms_.w32}) b->resize(Nm);
    ms_.w64.resize(Nm);
    ms_.partials.resize(size_t(MS_BLOCKS) * MS_MAXM);
    ms_.h.resize(MS_MAXM);
    VG_CUDA(cudaDeviceSynchronize());
    ms_.amg_ready = false;
    ms_.ready = true;
}

template <typename T>
void Solver::ms_apply(const T* x, T* y) {
    MsArgs<T> a{};
    a.x = x;
    a.y = y;
    if constexpr (sizeof(T) == 8) {
        a.A = d_A0_.data();
        a.B = ms_.B64.data();
        a.mdt = ms_.m64.data();
    } else {
        a.A = ms_.A32.data();
        a.B = ms_.B32.data();
        a.mdt = ms_.m32.data();
    }
    a.map = d_map_.data();
    a.slot_cell = d_slot_cell_.data();
    a.pieces = d_pieces_.data();
    a.npieces = int(pieces_.size());
    a.nc = m.nc;
    a.nf = nf;
    a.mask = d_mask_.data();
    VG_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * 2 * nf, nullptr));
    k_ms_apply<T><<<ms_blocks((long long)pieces_.size() * PIECE), MS_THREADS>>>(a);
    VG_CUDA(cudaGetLastError());
    ++n_apply;
    ++n_launch;
}

template <typename T>
void Solver::ms_precond(const T* r, T* z) {
    const T* F = sizeof(T) == 8 ? reinterpret_cast<const T*>(ms_.F64.data()) : reinterpret_cast<const T*>(ms_.F32.data());
    const T* C = sizeof(T) == 8 ? reinterpret_cast<const T*>(ms_.C64.data()) : reinterpret_cast<const T*>(ms_.C32.data());
    k_ms_pc_apply<T><<<MS_BLOCKS, MS_THREADS>>>(r, z, F, C, nf, m.nc);
    VG_CUDA(cudaGetLastError());
    if (ms_.amg_ready)  // pressure blocks: one V-cycle per species (replaces the 2x2 cell blocks)
        for (int s = 0; s < 2; ++s)
            ms_.amg[s].vcycle(r + 2 * nf + (long long)s * m.nc, z + 2 * nf + (long long)s * m.nc, nullptr);
}

// S_s = diag(|E|/dt) + W diag((F_g^{-1})_ss) W^T on the cell graph (k = 0: W = +-1 per local edge,
// opposite signs across a shared edge), free flux dofs only
void Solver::ms_build_amg() {
    std::vector<double> F = ms_.F64.download(), mdt = ms_.m64.download();
    std::vector<int> mask(nf);
    VG_CUDA(cudaMemcpy(mask.data(), d_mask_.data(), sizeof(int) * nf, cudaMemcpyDeviceToHost));
    std::vector<int> ec(2 * size_t(m.ne), -1);
    for (int c = 0; c < m.nc; ++c)
        for (int j = m.cptr[c]; j < m.cptr[c + 1]; ++j) {
            int e = m.gedges[j];
            if (ec[2 * e] < 0)
                ec[2 * e] = c;
            else
                ec[2 * e + 1] = c;
        }
    for (int s = 0; s < 2; ++s) {
        HostCsr S;
        S.n = S.m = m.nc;
        S.ptr.assign(m.nc + 1, 0);
        std::vector<std::pair<int, double>> row;
        for (int c = 0; c < m.nc; ++c) {
            row.clear();
            double diag = mdt[c];
            for (int j = m.cptr[c]; j < m.cptr[c + 1]; ++j) {
                int e = m.gedges[j];
                if (mask[e]) continue;
                const double w = F[4 * size_t(e) + 3 * s];
                diag += w;
                int o = ec[2 * e] == c ? ec[2 * e + 1] : ec[2 * e];
                if (o >= 0) row.push_back({o, -w});
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
        ms_.amg[s].setup(S, nullptr);
    }
    ms_.amg_ready = true;
}

// dot products of w with columns 0..cnt-1 of V (host result)
template <typename T>
void Solver::ms_dots(const T* V, long long ld, int cnt, const T* w, double* out, int self) {
    k_mdot<T><<<MS_BLOCKS, MS_THREADS>>>(V, ld, cnt, w, ms_.N, ms_.partials.data(), self);
    k_mdot_finish<<<1, MS_MAXM>>>(ms_.partials.data(), MS_BLOCKS, cnt + self, ms_.h.data());
    VG_CUDA(cudaGetLastError());
    VG_CUDA(cudaMemcpy(out, ms_.h.data(), sizeof(double) * (cnt + self), cudaMemcpyDeviceToHost));
}

// right-preconditioned GMRES(m) on K d = r from d = 0; returns iterations, relative reduction in *rel
template <typename T>
int Solver::ms_gmres(const T* r, T* d, double tol, int maxit, int mres, double* rel) {
    const long long Nm = ms_.N;
    T* V = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.V64.data()) : reinterpret_cast<T*>(ms_.V32.data());
    T* w = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.w64.data()) : reinterpret_cast<T*>(ms_.w32.data());
    T* t = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.t64.data()) : reinterpret_cast<T*>(ms_.t32.data());
    const int m = std::max(1, std::min(mres, MS_MAXM - 1));
    VG_CUDA(cudaMemsetAsync(d, 0, sizeof(T) * Nm, nullptr));
    // residual of the current iterate, kept in t (r initially)
    VG_CUDA(cudaMemcpyAsync(t, r, sizeof(T) * Nm, cudaMemcpyDeviceToDevice, nullptr));
    double nr = 0;
    ms_dots(t, 0, 1, t, &nr, 0);
    const double beta0 = std::sqrt(nr);
    *rel = 1.0;
    if (!(beta0 > 0)) return 0;
    int its = 0;
    std::vector<double> H(size_t(MS_MAXM) * MS_MAXM), cs(MS_MAXM), sn(MS_MAXM), g(MS_MAXM + 1), h(MS_MAXM + 1),
        h2(MS_MAXM), y(MS_MAXM);
    double beta = beta0;
    while (its < maxit) {
        k_scale_to<T><<<MS_BLOCKS, MS_THREADS>>>(t, 1.0 / beta, V, Nm);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        bool done = false;
        for (; j < m && its < maxit; ++j) {
            ++its;
            ms_precond<T>(V + (long long)j * Nm, t);
            ms_apply<T>(t, w);
            // classical Gram-Schmidt applied twice (the second pass restores orthogonality lost to
            // cancellation); the norm of the result rides on the second projection's pass
            ms_dots(V, Nm, j + 1, w, h.data(), 0);
            VG_CUDA(cudaMemcpy(ms_.h.data(), h.data(), sizeof(double) * (j + 1), cudaMemcpyHostToDevice));
            k_gs_update<T><<<MS_BLOCKS, MS_THREADS>>>(V, Nm, j + 1, ms_.h.data(), w, Nm);
            ms_dots(V, Nm, j + 1, w, h2.data(), 0);
            VG_CUDA(cudaMemcpy(ms_.h.data(), h2.data(), sizeof(double) * (j + 1), cudaMemcpyHostToDevice));
            k_gs_update<T><<<MS_BLOCKS, MS_THREADS>>>(V, Nm, j + 1, ms_.h.data(), w, Nm);
            for (int i = 0; i <= j; ++i) h[i] += h2[i];
            double nw = 0;
            ms_dots(w, 0, 1, w, &nw, 0);
            const double hn = std::sqrt(std::max(nw, 0.0));
            if (hn > 0) k_scale_to<T><<<MS_BLOCKS, MS_THREADS>>>(w, 1.0 / hn, V + (long long)(j + 1) * Nm, Nm);
            // Givens rotations of column j
            for (int i = 0; i < j; ++i) {
                const double a = h[i], b = h[i + 1];
                h[i] = cs[i] * a + sn[i] * b;
                h[i + 1] = -sn[i] * a + cs[i] * b;
            }
            const double den = std::hypot(h[j], hn);
            cs[j] = den > 0 ? h[j] / den : 1.0;
            sn[j] = den > 0 ? hn / den : 0.0;
            h[j] = den;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            for (int i = 0; i <= j; ++i) H[size_t(i) * MS_MAXM + j] = h[i];
            *rel = std::fabs(g[j + 1]) / beta0;
            if (*rel <= tol || !(hn > 0)) {
                ++j;
                done = true;
                break;
            }
        }
        // y = H^{-1} g (upper triangular), d += M^{-1} V y
        for (int i = j - 1; i >= 0; --i) {
            double s = g[i];
            for (int c = i + 1; c < j; ++c) s -= H[size_t(i) * MS_MAXM + c] * y[c];
            y[i] = H[size_t(i) * MS_MAXM + i] != 0 ? s / H[size_t(i) * MS_MAXM + i] : 0.0;
        }
        VG_CUDA(cudaMemcpy(ms_.h.data(), y.data(), sizeof(double) * j, cudaMemcpyHostToDevice));
        k_combine<T><<<MS_BLOCKS, MS_THREADS>>>(V, Nm, j, ms_.h.data(), w, Nm);
        ms_precond<T>(w, t);
        k_axpy_t<T><<<MS_BLOCKS, MS_THREADS>>>(d, t, 1.0, Nm);
        VG_CUDA(cudaGetLastError());
        if (done) break;
        // restart: t = r - K d
        ms_apply<T>(d, w);
        if constexpr (sizeof(T) == 8) {
            k_sub<<<MS_BLOCKS, MS_THREADS>>>(reinterpret_cast<const double*>(r), reinterpret_cast<const double*>(w),
                                            reinterpret_cast<double*>(t), Nm);
        } else {
            VG_CUDA(cudaMemcpyAsync(t, r, sizeof(T) * Nm, cudaMemcpyDeviceToDevice, nullptr));
            k_axpy_t<T><<<MS_BLOCKS, MS_THREADS>>>(t, w, -1.0, Nm);
        }
        double nt = 0;
        ms_dots(t, 0, 1, t, &nt, 0);
        beta = std::sqrt(nt);
        *rel = beta / beta0;
        if (*rel <= tol || !(beta > 0)) break;
    }
    return its;
}

__global__ void k_cell_areas(const double* L, int nc, int q, double* out) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) out[c] = L[(long long)c * q];
}

// physical cell measures int_E det J (the first moment of the multiplier vector, m_0 = 1)
void Solver::cell_areas(double* out) {
    if (!built) throw Error(VG_ESTATE, "vg_build must run before vg_cell_areas");
    k_cell_areas<<<ms_blocks(m.nc), MS_THREADS>>>(d_L_.data(), m.nc, q, out);
    VG_CUDA(cudaGetLastError());
    VG_CUDA(cudaDeviceSynchronize());
}

void Solver::ms_coefficients(const double* state) {
    if (!ms_.ready) throw Error(VG_ESTATE, "vg_ms_configure must run first");
    k_ms_coeff<<<ms_blocks(m.nc), MS_THREADS>>>(state, 2 * nf, m.nc, ms_.i12, ms_.i13, ms_.i23, ms_.B64.data(),
                                               ms_.B32.data());
    VG_CUDA(cudaGetLastError());
}

void Solver::ms_step(const double* old_state, double* new_state, const vg_solve_opts& o, vg_solve_info& info) {
    if (!ms_.ready) throw Error(VG_ESTATE, "vg_ms_configure must run before vg_ms_step");
    if (!(o.tol > 0) || o.maxit < 1 || (o.mode == VG_SOLVE_MIXED && !(o.inner_tol > 0 && o.inner_tol < 1)))
        throw Error(VG_EINVAL, "invalid solve options");
    info = vg_solve_info{};
    const long long Nm = ms_.N;
    VG_CUDA(cudaDeviceSynchronize());
    VG_CUDA(cudaEventRecord(ev0_, nullptr));
    // coefficients and preconditioner at x^n
    ms_coefficients(old_state);
    ms_.D.zero();
    k_ms_pc_flux<<<ms_blocks((long long)pieces_.size() * PIECE), MS_THREADS>>>(
        d_A0_.data(), d_map_.data(), d_pieces_.data(), int(pieces_.size()), d_slot_cell_.data(), ms_.B64.data(),
        d_mask_.data(), ms_.D.data());
    k_ms_pc_flux_inv<<<MS_BLOCKS, MS_THREADS>>>(ms_.D.data(), d_mask_.data(), nf, ms_.F64.data(), ms_.F32.data());
    k_ms_pc_cell<<<ms_blocks((long long)pieces_.size() * PIECE), MS_THREADS>>>(
        d_map_.data(), d_pieces_.data(), int(pieces_.size()), d_slot_cell_.data(), d_mask_.data(), ms_.F64.data(),
        ms_.m64.data(), ms_.C64.data(), ms_.C32.data());
    if (!ms_.amg_ready) {
        VG_CUDA(cudaDeviceSynchronize());
        try {
            ms_build_amg();
        } catch (const Error&) {
            ms_.amg_ready = false;  // the 2x2 cell blocks stay in use
        }
    }
    k_ms_rhs<<<MS_BLOCKS, MS_THREADS>>>(old_state, ms_.m64.data(), nf, m.nc, ms_.b.data());
    VG_CUDA(cudaGetLastError());
    // initial guess: the old state
    if (new_state != old_state)
        VG_CUDA(cudaMemcpyAsync(new_state, old_state, sizeof(double) * Nm, cudaMemcpyDeviceToDevice, nullptr));
    auto true_residual = [&](double* nb_out) {
        ms_apply<double>(new_state, ms_.y.data());
        k_sub<<<MS_BLOCKS, MS_THREADS>>>(ms_.b.data(), ms_.y.data(), ms_.r.data(), Nm);
        double nr = 0, nb = 0;
        ms_dots(ms_.r.data(), 0, 1, ms_.r.data(), &nr, 0);
        ms_dots(ms_.b.data(), 0, 1, ms_.b.data(), &nb, 0);
        if (nb_out) *nb_out = std::sqrt(nb);
        return std::sqrt(nr) / (nb > 0 ? std::sqrt(nb) : 1.0);
    };
    double nb = 0;
    double rel = true_residual(&nb);
    int total = 0, outer = 0;
    const int mres = 30;
    if (o.mode == VG_SOLVE_FP64) {
        for (outer = 0; outer < 4 && rel > o.tol && total < o.maxit; ++outer) {
            double r_in = 0;
            const double rn = rel * nb;
            total += ms_gmres<double>(ms_.r.data(), ms_.d.data(), std::min(0.5, 0.5 * o.tol * nb / rn), o.maxit - total,
                                      mres, &r_in);
            k_axpy_t<double><<<MS_BLOCKS, MS_THREADS>>>(new_state, ms_.d.data(), 1.0, Nm);
            rel = true_residual(nullptr);
        }
    } else {
        for (outer = 0; outer < o.max_outer && rel > o.tol && total < o.maxit; ++outer) {
            const double rn = rel * nb;
            k_d2f<<<MS_BLOCKS, MS_THREADS>>>(ms_.r.data(), ms_.r32.data(), Nm, 1.0 / rn);
            double r_in = 0;
            total += ms_gmres<float>(ms_.r32.data(), ms_.d32.data(), o.inner_tol, o.maxit - total, mres, &r_in);
            k_addf<<<MS_BLOCKS, MS_THREADS>>>(new_state, ms_.d32.data(), rn, Nm);
            rel = true_residual(nullptr);
        }
    }
    VG_CUDA(cudaEventRecord(ev1_, nullptr));
    VG_CUDA(cudaEventSynchronize(ev1_));
    float ms = 0;
    VG_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    info.iterations = total;
    info.outer = outer;
    info.residual = rel;
    info.seconds = ms * 1e-3;
    n_iter += total;
    ++n_solve;
    if (!(rel <= o.tol))
        throw Error(VG_ENOCONV, "Maxwell-Stefan step did not converge: iterations=" + std::to_string(total) +
                                    " true_relative_residual=" + std::to_string(rel));
}

template void Solver::ms_apply<double>(const double*, double*);
template void Solver::ms_apply<float>(const float*, float*);

}  // namespace vg
