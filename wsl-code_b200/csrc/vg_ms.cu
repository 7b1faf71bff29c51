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
// eliminated; B is taken at x^n (one linear solve per step, the default) or, with Picard
// iterations (vg_ms_set_picard), re-evaluated at the latest iterate until the step is fully implicit.
//
// B is not symmetric, so the system is solved by right-preconditioned GMRES(m) (classical
// Gram-Schmidt, a second pass where the first lost too much of |w|; the Arnoldi loop of a cycle is a captured CUDA graph whose Hessenberg
// column, Givens rotations and residual estimate are formed on the device), FP64 or
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
#ifndef VG_MS_RESTART
#define VG_MS_RESTART 10  // GMRES restart length (< MS_MAXM); 10 measured fastest with 8 at 250k cells
                          // (step 26.6 -> 21.0 ms FP64 against 30: less Gram-Schmidt work, same iterations)
#endif

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

// one cell, both species (NE edges; NE = 0: runtime count up to MAX_NE, arrays in local memory)
template <typename T, int NE>
__device__ __forceinline__ void ms_cell(const MsArgs<T>& a, const Piece& P, int lane) {
    constexpr int M = NE > 0 ? NE : MAX_NE;
    const int n = NE > 0 ? NE : P.n;
    const int cell = a.slot_cell[P.slot + lane];
    int g[M];
    T u0[M], u1[M], y0[M], y1[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
        if (i >= n) break;
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
    int e = 0;
#pragma unroll
    for (int i = 0; i < M; ++i) {
        if (i >= n) break;
#pragma unroll
        for (int c = i; c < M; ++c) {
            if (c >= n) break;
            const T v = Ap[(long long)(e++) * PIECE];
            y0[i] += v * u0[c];
            y1[i] += v * u1[c];
            if (c != i) {
                y0[c] += v * u0[i];
                y1[c] += v * u1[i];
            }
        }
    }
    const T b00 = a.B[4LL * cell], b01 = a.B[4LL * cell + 1], b10 = a.B[4LL * cell + 2], b11 = a.B[4LL * cell + 3];
    const long long p0 = 2 * a.nf + cell, p1 = 2 * a.nf + a.nc + cell;
    const T pr0 = a.x[p0], pr1 = a.x[p1];
    T d0 = T(0), d1 = T(0);
#pragma unroll
    for (int i = 0; i < M; ++i) {
        if (i >= n) break;
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

// y = K x; one lane per cell, both species; masked flux rows are identity rows. Cells with 3..9
// edges here (fixed-size register arrays), larger polygons in k_ms_apply_large
template <typename T>
__global__ void __launch_bounds__(MS_THREADS) k_ms_apply(MsArgs<T> a) {
    Piece P;
    int lane;
    if (!ms_slot(a.pieces, a.npieces, P, lane)) return;
    switch (P.n) {
    case 3: ms_cell<T, 3>(a, P, lane); break;
    case 4: ms_cell<T, 4>(a, P, lane); break;
    case 5: ms_cell<T, 5>(a, P, lane); break;
    case 6: ms_cell<T, 6>(a, P, lane); break;
    case 7: ms_cell<T, 7>(a, P, lane); break;
    case 8: ms_cell<T, 8>(a, P, lane); break;
    case 9: ms_cell<T, 9>(a, P, lane); break;
    default: break;
    }
}

template <typename T>
__global__ void __launch_bounds__(MS_THREADS) k_ms_apply_large(MsArgs<T> a) {
    Piece P;
    int lane;
    if (!ms_slot(a.pieces, a.npieces, P, lane)) return;
    if (P.n < 3 || P.n > 9) ms_cell<T, 0>(a, P, lane);
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

// GMRES scalars on the device. The Arnoldi loop of one cycle runs as a CUDA graph (a conditional
// while node around one iteration), so the Hessenberg column, the Givens rotations and the
// residual estimate are formed on the device and the host reads them once per cycle.
struct MsKrylov {
    double H[MS_MAXM * MS_MAXM];  // H[i * MS_MAXM + c]: R factor of the Hessenberg matrix
    double cs[MS_MAXM], sn[MS_MAXM], g[MS_MAXM + 1], y[MS_MAXM];
    double hd[3 * MS_MAXM];  // [0, 32): first Gram-Schmidt pass, [32, 64): second, [64]: |w|^2, [65]: |t|^2
    double beta0, tol, rel;
    int j, its, m, maxit, done, reorth;  // reorth: second Gram-Schmidt passes run in this solve
};

// Selective reorthogonalisation (Daniel, Gragg, Kaufman and Stewart, Math. Comp. 30 (1976); the
// "twice is enough" analysis of Giraud, Langou and Rozloznik, Comput. Math. Appl. 50 (2005)): the
// second classical Gram-Schmidt pass runs only when the first removed more than half of |w|^2,
// i.e. when |w'|^2 < REORTH_ETA2 |w|^2; otherwise w' is already orthogonal to the basis to working
// precision and the second pass would subtract nothing. hd[cnt] holds |w|^2 before the first pass
// (written by that pass's dot products), hd[2 MS_MAXM] |w'|^2 after it.
constexpr double REORTH_ETA2 = 0.5;
__device__ __forceinline__ bool reorth_skip(const double* hd, int cnt) {
    return hd[2 * MS_MAXM] >= REORTH_ETA2 * hd[cnt];
}

// one V-cycle-sized work split: block b owns rows [b chunk, (b + 1) chunk); chunk is a multiple of 4
template <typename T>
__device__ __forceinline__ double dot4(const T (&a)[4], const T (&b)[4]) {
    return double(a[0]) * double(b[0]) + double(a[1]) * double(b[1]) + double(a[2]) * double(b[2]) +
           double(a[3]) * double(b[3]);
}

// sum of the per-block values v[0..cnt) over the grid in a fixed order; the last block to arrive
// writes out[0..cnt) and resets the counter. sh holds the block's per-warp values on entry.
__device__ void ms_grid_sum(double (*sh)[MS_MAXM], int cnt, double* partials, unsigned* counter, double* out) {
    __shared__ bool last;
    if (threadIdx.x < cnt) {
        double s = 0;
        for (int q = 0; q < MS_THREADS / 32; ++q) s += sh[q][threadIdx.x];
        partials[(long long)blockIdx.x * MS_MAXM + threadIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int wid = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int k = wid; k < cnt; k += MS_THREADS / 32) {
        double s = 0;
        for (int b = l; b < gridDim.x; b += 32) s += __ldcg(partials + (long long)b * MS_MAXM + k);
        for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if (l == 0) out[k] = s;
    }
    if (threadIdx.x == 0) *counter = 0;
}

// out[k] = V[:, k] . w for k < cnt, cnt = (cnt_dev ? *cnt_dev : 0) + cnt_add. Block b stages its
// rows of w in shared memory and streams the cnt columns over them (four at a time, 16-byte
// loads); the column stride ld and chunk are multiples of 4. self_dot: also out[cnt] = w . w (the
// first Gram-Schmidt pass, for the reorthogonalisation test). reo: the second pass; when
// reorth_skip(reo, cnt) holds, out[0..cnt) = 0 and nothing is read.
template <typename T>
__global__ void __launch_bounds__(MS_THREADS) k_mdot(const T* V, long long ld, const int* cnt_dev, int cnt_add,
                                                     const T* w, long long n, long long chunk, double* partials,
                                                     unsigned* counter, double* out, int self_dot,
                                                     const double* reo) {
    extern __shared__ __align__(16) unsigned char ms_smem[];
    T* ws = reinterpret_cast<T*>(ms_smem);
    __shared__ double sh[MS_THREADS / 32][MS_MAXM];
    const int cnt = min((cnt_dev ? *cnt_dev : 0) + cnt_add, MS_MAXM);
    if (reo && reorth_skip(reo, cnt)) {
        if (blockIdx.x == 0 && threadIdx.x < cnt) out[threadIdx.x] = 0.0;
        return;
    }
    const bool sd = self_dot && cnt < MS_MAXM;
    double aw = 0;
    const long long lo = blockIdx.x * chunk;
    const int len = int(max(0LL, min(n, lo + chunk) - lo));
    const int len4 = len & ~3;
    for (int i = 4 * threadIdx.x; i < len4; i += 4 * MS_THREADS) {
        T v[4];
        ld4(w + lo + i, v);
        st4(ws + i, v);
    }
    for (int i = len4 + threadIdx.x; i < len; i += MS_THREADS) ws[i] = w[lo + i];
    __syncthreads();
    const int wid = threadIdx.x >> 5, l = threadIdx.x & 31;
    // four columns at a time, rows unrolled by two: about eight 16-byte loads in flight per thread
    for (int k = 0; k < cnt; k += 4) {
        const int nk = min(4, cnt - k);
        const T* v0 = V + k * ld + lo;
        const T* v1 = nk > 1 ? v0 + ld : v0;
        const T* v2 = nk > 2 ? v0 + 2 * ld : v0;
        const T* v3 = nk > 3 ? v0 + 3 * ld : v0;
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll 2
        for (int i = 4 * threadIdx.x; i < len4; i += 4 * MS_THREADS) {
            T x[4], p0[4], p1[4], p2[4], p3[4];
            ld4(v0 + i, p0);
            ld4(v1 + i, p1);
            ld4(v2 + i, p2);
            ld4(v3 + i, p3);
            ld4(ws + i, x);
            a0 += dot4(p0, x);
            a1 += dot4(p1, x);
            a2 += dot4(p2, x);
            a3 += dot4(p3, x);
            if (sd && k == 0) aw += dot4(x, x);
        }
        for (int i = len4 + threadIdx.x; i < len; i += MS_THREADS) {
            const double xi = double(ws[i]);
            a0 += double(v0[i]) * xi;
            a1 += double(v1[i]) * xi;
            a2 += double(v2[i]) * xi;
            a3 += double(v3[i]) * xi;
            if (sd && k == 0) aw += xi * xi;
        }
        for (int off = 16; off; off >>= 1) {
            a0 += __shfl_down_sync(0xffffffffu, a0, off);
            a1 += __shfl_down_sync(0xffffffffu, a1, off);
            a2 += __shfl_down_sync(0xffffffffu, a2, off);
            a3 += __shfl_down_sync(0xffffffffu, a3, off);
        }
        if (l == 0) {
            sh[wid][k] = a0;
            if (nk > 1) sh[wid][k + 1] = a1;
            if (nk > 2) sh[wid][k + 2] = a2;
            if (nk > 3) sh[wid][k + 3] = a3;
        }
    }
    if (sd) {
        for (int off = 16; off; off >>= 1) aw += __shfl_down_sync(0xffffffffu, aw, off);
        if (l == 0) sh[wid][cnt] = aw;
    }
    __syncthreads();
    ms_grid_sum(sh, cnt + (sd ? 1 : 0), partials, counter, out);
}

// w -= sum_k h[k] V[:, k] (cnt columns, as in k_mdot); with nrm: |w|^2 of the result -> nrm[0].
// reo: the second pass; skipped when reorth_skip(reo, cnt) holds (w and nrm keep the first pass's
// values), otherwise counted in *runs.
template <typename T>
__global__ void __launch_bounds__(MS_THREADS) k_gs_update(const T* V, long long ld, const int* cnt_dev, int cnt_add,
                                                          const double* h, T* w, long long n, double* partials,
                                                          unsigned* counter, double* nrm, const double* reo,
                                                          int* runs) {
    __shared__ T hs[MS_MAXM];
    __shared__ double sh[MS_THREADS / 32][MS_MAXM];
    const int cnt = min((cnt_dev ? *cnt_dev : 0) + cnt_add, MS_MAXM);
    if (reo) {
        // every block reads nrm[0] here, before any block can reach the grid sum that rewrites it
        if (reorth_skip(reo, cnt)) return;
        if (runs && blockIdx.x == 0 && threadIdx.x == 0) *runs += 1;
    }
    if (threadIdx.x < cnt) hs[threadIdx.x] = T(h[threadIdx.x]);
    __syncthreads();
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, nth = (long long)gridDim.x * blockDim.x;
    const long long n4 = n & ~3LL;
    double acc = 0;
    for (long long i = 4 * tid; i < n4; i += 4 * nth) {
        T s[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) {
            T a[4];
            ld4(V + k * ld + i, a);
#pragma unroll
            for (int q = 0; q < 4; ++q) s[q] += hs[k] * a[q];
        }
        T x[4];
        ld4(w + i, x);
#pragma unroll
        for (int q = 0; q < 4; ++q) x[q] -= s[q];
        st4(w + i, x);
        acc += dot4(x, x);
    }
    for (long long i = n4 + tid; i < n; i += nth) {
        T s = T(0);
        for (int k = 0; k < cnt; ++k) s += hs[k] * V[k * ld + i];
        const T x = w[i] - s;
        w[i] = x;
        acc += double(x) * double(x);
    }
    if (!nrm) return;
    for (int off = 16; off; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5][0] = acc;
    __syncthreads();
    ms_grid_sum(sh, 1, partials, counter, nrm);
}

// v = w / sqrt(nrm2[0]) into column (*col + 1) of V and into vnext (the next preconditioner input)
template <typename T>
__global__ void __launch_bounds__(MS_THREADS) k_scale_norm(const T* w, const double* nrm2, T* V, long long ld,
                                                           const int* col, T* vnext, long long n) {
    const double nr = sqrt(fmax(nrm2[0], 0.0));
    const double a = nr > 0 ? 1.0 / nr : 0.0;
    T* v = V + (long long)(col[0] + 1) * ld;
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, nth = (long long)gridDim.x * blockDim.x;
    const long long n4 = n & ~3LL;
    for (long long i = 4 * tid; i < n4; i += 4 * nth) {
        T x[4];
        ld4(w + i, x);
#pragma unroll
        for (int q = 0; q < 4; ++q) x[q] = T(a * double(x[q]));
        st4(v + i, x);
        st4(vnext + i, x);
    }
    for (long long i = n4 + tid; i < n; i += nth) v[i] = vnext[i] = T(a * double(w[i]));
}

// start of a cycle: beta = sqrt(|t|^2) (hd[65]); V[:, 0] = vnext = t / beta, g = beta e_0, j = 0
template <typename T>
__global__ void __launch_bounds__(MS_THREADS) k_cycle_start(const T* t, T* V, T* vnext, long long n, MsKrylov* K,
                                                            int first) {
    const double beta = sqrt(fmax(K->hd[65], 0.0));
    const double a = beta > 0 ? 1.0 / beta : 0.0;
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, nth = (long long)gridDim.x * blockDim.x;
    const long long n4 = n & ~3LL;
    for (long long i = 4 * tid; i < n4; i += 4 * nth) {
        T x[4];
        ld4(t + i, x);
#pragma unroll
        for (int q = 0; q < 4; ++q) x[q] = T(a * double(x[q]));
        st4(V + i, x);
        st4(vnext + i, x);
    }
    for (long long i = n4 + tid; i < n; i += nth) V[i] = vnext[i] = T(a * double(t[i]));
    if (tid == 0) {
        for (int i = 0; i <= MS_MAXM; ++i) K->g[i] = 0.0;
        K->g[0] = beta;
        K->j = 0;
        if (first) K->beta0 = beta;
    }
}

__global__ void k_kry_init(MsKrylov* K, double tol, int m, int maxit) {
    K->tol = tol;
    K->m = m;
    K->maxit = maxit;
    K->its = 0;
    K->done = 0;
    K->rel = 1.0;
    K->reorth = 0;
}

// end of an Arnoldi step: Hessenberg column j from the two Gram-Schmidt passes, previous rotations,
// new rotation, residual estimate |g_{j+1}| / beta0; the loop continues while the cycle has room,
// the estimate is above tol and the new vector is nonzero
__global__ void k_givens(MsKrylov* K, cudaGraphConditionalHandle cond) {
    const int j = K->j;
    double h[MS_MAXM + 1];
    for (int i = 0; i <= j; ++i) h[i] = K->hd[i] + K->hd[MS_MAXM + i];
    const double hn = sqrt(fmax(K->hd[2 * MS_MAXM], 0.0));
    for (int i = 0; i < j; ++i) {
        const double a = h[i], b = h[i + 1];
        h[i] = K->cs[i] * a + K->sn[i] * b;
        h[i + 1] = -K->sn[i] * a + K->cs[i] * b;
    }
    const double den = hypot(h[j], hn);
    K->cs[j] = den > 0 ? h[j] / den : 1.0;
    K->sn[j] = den > 0 ? hn / den : 0.0;
    h[j] = den;
    K->g[j + 1] = -K->sn[j] * K->g[j];
    K->g[j] = K->cs[j] * K->g[j];
    for (int i = 0; i <= j; ++i) K->H[i * MS_MAXM + j] = h[i];
    K->rel = fabs(K->g[j + 1]) / K->beta0;
    K->its += 1;
    K->j = j + 1;
    K->done = (K->rel <= K->tol || !(hn > 0)) ? 1 : 0;
    const bool more = !K->done && K->j < K->m && K->its < K->maxit;
    cudaGraphSetConditional(cond, more ? 1u : 0u);
}

// y = R^{-1} g over the j columns of the cycle
__global__ void k_trisolve(MsKrylov* K) {
    const int j = K->j;
    for (int i = j - 1; i >= 0; --i) {
        double s = K->g[i];
        for (int c = i + 1; c < j; ++c) s -= K->H[i * MS_MAXM + c] * K->y[c];
        const double d = K->H[i * MS_MAXM + i];
        K->y[i] = d != 0 ? s / d : 0.0;
    }
}

// t = sum_{k < *cnt} y[k] V[:, k]
template <typename T>
__global__ void __launch_bounds__(MS_THREADS) k_combine(const T* V, long long ld, const int* cnt_dev, const double* y,
                                                        T* t, long long n) {
    __shared__ double ys[MS_MAXM];
    const int cnt = min(*cnt_dev, MS_MAXM);
    if (threadIdx.x < cnt) ys[threadIdx.x] = y[threadIdx.x];
    __syncthreads();
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, nth = (long long)gridDim.x * blockDim.x;
    const long long n4 = n & ~3LL;
    for (long long i = 4 * tid; i < n4; i += 4 * nth) {
        double s[4] = {0, 0, 0, 0};
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) {
            T a[4];
            ld4(V + k * ld + i, a);
#pragma unroll
            for (int q = 0; q < 4; ++q) s[q] += ys[k] * double(a[q]);
        }
        T o[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] = T(s[q]);
        st4(t + i, o);
    }
    for (long long i = n4 + tid; i < n; i += nth) {
        double s = 0;
        for (int k = 0; k < cnt; ++k) s += ys[k] * double(V[k * ld + i]);
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
    ms_destroy_graphs();
    ms_.i12 = 1.0 / d12;
    ms_.i13 = 1.0 / d13;
    ms_.i23 = 1.0 / d23;
    ms_.dt = dt;
    ms_.N = 2LL * nf + 2LL * m.nc;
    ms_large_ = false;
    for (const auto& P : pieces_) ms_large_ = ms_large_ || P.n < 3 || P.n > 9;
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
    VG_CUDA(cudaDeviceSynchronize());  // inputs written on other streams
    k_d2f<<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(d_A0_.data(), ms_.A32.data(), a_total_, 1.0);
    k_ms_mdt<<<ms_blocks(m.nc), MS_THREADS, 0, stream_>>>(d_L_.data(), m.nc, dt, ms_.m64.data(), ms_.m32.data());
    VG_CUDA(cudaGetLastError());
    // Krylov basis with a column stride that keeps every column 16-byte aligned for 4-wide access
    ms_.ld = (Nm + 63) / 64 * 64;
    ms_.V64.resize(size_t(MS_MAXM) * ms_.ld);
    ms_.V32.resize(size_t(MS_MAXM) * ms_.ld);
    for (auto* b : {&ms_.b, &ms_.r, &ms_.y, &ms_.d, &ms_.t64, &ms_.vn64}) b->resize(Nm);
    for (auto* b : {&ms_.r32, &ms_.d32, &ms_.t32, &ms_.w32, &ms_.vn32}) b->resize(Nm);
    ms_.w64.resize(Nm);
    // dot-product split: at least one block per SM slot, at most 8192 rows (64 KB of FP64 staging) per block
    ms_.chunk = std::min<long long>(8192, ((Nm + MS_BLOCKS - 1) / MS_BLOCKS + 3) / 4 * 4);
    ms_.dblocks = int((Nm + ms_.chunk - 1) / ms_.chunk);
    ms_.partials.resize(size_t(std::max(ms_.dblocks, MS_BLOCKS)) * MS_MAXM);
    ms_.counter.resize(1);
    VG_CUDA(cudaMemsetAsync(ms_.counter.data(), 0, sizeof(unsigned), stream_));
    ms_.kry.resize((sizeof(MsKrylov) + 7) / 8);
    VG_CUDA(cudaMemsetAsync(ms_.kry.data(), 0, sizeof(MsKrylov), stream_));
    VG_CUDA(cudaFuncSetAttribute(k_mdot<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8192 * 8));
    VG_CUDA(cudaFuncSetAttribute(k_mdot<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8192 * 4));
    VG_CUDA(cudaStreamSynchronize(stream_));
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
    VG_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * 2 * nf, stream_));
    k_ms_apply<T><<<ms_blocks((long long)pieces_.size() * PIECE), MS_THREADS, 0, stream_>>>(a);
    if (ms_large_) k_ms_apply_large<T><<<ms_blocks((long long)pieces_.size() * PIECE), MS_THREADS, 0, stream_>>>(a);
    VG_CUDA(cudaGetLastError());
    ++n_apply;
    ++n_launch;
}

template <typename T>
void Solver::ms_precond(const T* r, T* z) {
    const T* F = sizeof(T) == 8 ? reinterpret_cast<const T*>(ms_.F64.data()) : reinterpret_cast<const T*>(ms_.F32.data());
    const T* C = sizeof(T) == 8 ? reinterpret_cast<const T*>(ms_.C64.data()) : reinterpret_cast<const T*>(ms_.C32.data());
    k_ms_pc_apply<T><<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(r, z, F, C, nf, m.nc);
    VG_CUDA(cudaGetLastError());
    if (ms_.amg_ready) {  // pressure blocks: one V-cycle per species (replaces the 2x2 cell blocks)
        // the two species' cycles are independent chains of small kernels: the second runs on a
        // second stream beside the first
        VG_CUDA(cudaEventRecord(ev_fork_, stream_));
        VG_CUDA(cudaStreamWaitEvent(side_, ev_fork_, 0));
        ms_.amg[1].vcycle(r + 2 * nf + m.nc, z + 2 * nf + m.nc, side_);
        VG_CUDA(cudaEventRecord(ev_join_, side_));
        ms_.amg[0].vcycle(r + 2 * nf, z + 2 * nf, stream_);
        VG_CUDA(cudaStreamWaitEvent(stream_, ev_join_, 0));
    }
}

// S_s = diag(|E|/dt) + W diag((F_g^{-1})_ss) W^T on the cell graph (k = 0: W = +-1 per local edge,
// opposite signs across a shared edge), free flux dofs only
void Solver::ms_build_amg() {
    ms_destroy_graphs();  // the captured loop holds the previous hierarchy's buffers
    VG_CUDA(cudaStreamSynchronize(stream_));
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
    VG_CUDA(cudaDeviceSynchronize());
    ms_.amg_ready = true;
}

// |x|^2 into device memory
template <typename T>
void Solver::ms_norm2(const T* x, double* dst) {
    k_mdot<T><<<ms_.dblocks, MS_THREADS, ms_.chunk * sizeof(T), stream_>>>(
        x, 0, nullptr, 1, x, ms_.N, ms_.chunk, ms_.partials.data(), ms_.counter.data(), dst, 0, nullptr);
    VG_CUDA(cudaGetLastError());
}

// |x| on the host
template <typename T>
double Solver::ms_norm(const T* x) {
    MsKrylov* K = reinterpret_cast<MsKrylov*>(ms_.kry.data());
    ms_norm2<T>(x, K->hd + 2 * MS_MAXM + 1);
    double h = 0;
    VG_CUDA(cudaMemcpyAsync(&h, K->hd + 2 * MS_MAXM + 1, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    VG_CUDA(cudaStreamSynchronize(stream_));
    return std::sqrt(std::max(h, 0.0));
}

void Solver::ms_destroy_graphs() {
    for (int p = 0; p < 2; ++p) {
        if (ms_.gexec[p]) cudaGraphExecDestroy(ms_.gexec[p]);
        if (ms_.graph[p]) cudaGraphDestroy(ms_.graph[p]);
        ms_.gexec[p] = nullptr;
        ms_.graph[p] = nullptr;
    }
}

// one Arnoldi step on the stream being captured: z = M^{-1} v_j, w = K z, classical Gram-Schmidt
// with a second pass where the first removed more than half of |w|^2 (it restores the
// orthogonality lost to cancellation), v_{j+1} = w/|w|,
// then the Givens update that sets the loop condition. The column index j lives on the device.
template <typename T>
void Solver::ms_arnoldi_step(cudaGraphConditionalHandle cond) {
    const long long Nm = ms_.N, ld = ms_.ld;
    T* V = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.V64.data()) : reinterpret_cast<T*>(ms_.V32.data());
    T* w = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.w64.data()) : reinterpret_cast<T*>(ms_.w32.data());
    T* t = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.t64.data()) : reinterpret_cast<T*>(ms_.t32.data());
    T* vn = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.vn64.data()) : reinterpret_cast<T*>(ms_.vn32.data());
    MsKrylov* K = reinterpret_cast<MsKrylov*>(ms_.kry.data());
    double* part = ms_.partials.data();
    unsigned* ctr = ms_.counter.data();
    const size_t smem = ms_.chunk * sizeof(T);
    ms_precond<T>(vn, t);
    ms_apply<T>(t, w);
    // first pass (with |w|^2 for the test), then the second only where the test asks for it
    for (int pass = 0; pass < 2; ++pass) {
        double* hd = K->hd + pass * MS_MAXM;
        const double* reo = pass ? K->hd : nullptr;
        k_mdot<T><<<ms_.dblocks, MS_THREADS, smem, stream_>>>(V, ld, &K->j, 1, w, Nm, ms_.chunk, part, ctr, hd,
                                                              pass ? 0 : 1, reo);
        k_gs_update<T><<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(V, ld, &K->j, 1, hd, w, Nm, part, ctr,
                                                              K->hd + 2 * MS_MAXM, reo, &K->reorth);
    }
    k_scale_norm<T><<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(w, K->hd + 2 * MS_MAXM, V, ld, &K->j, vn, Nm);
    k_givens<<<1, 1, 0, stream_>>>(K, cond);
    VG_CUDA(cudaGetLastError());
}

// the Arnoldi loop of one cycle as a CUDA graph: a conditional while node around one step
template <typename T>
void Solver::ms_build_graph(int p) {
    VG_CUDA(cudaGraphCreate(&ms_.graph[p], 0));
    cudaGraphConditionalHandle h;
    VG_CUDA(cudaGraphConditionalHandleCreate(&h, ms_.graph[p], 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    VG_CUDA(cudaGraphAddNode(&node, ms_.graph[p], nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    VG_CUDA(cudaStreamBeginCaptureToGraph(stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const long long napply = n_apply, nlaunch = n_launch;
    const long long l0 = ms_.amg[0].launches, l1 = ms_.amg[1].launches;
    try {
        ms_arnoldi_step<T>(h);
    } catch (...) {
        cudaGraph_t dummy;
        cudaStreamEndCapture(stream_, &dummy);
        throw;
    }
    n_apply = napply;
    n_launch = nlaunch;
    ms_.amg[0].launches = l0;
    ms_.amg[1].launches = l1;
    VG_CUDA(cudaStreamEndCapture(stream_, &body));
    VG_CUDA(cudaGraphInstantiate(&ms_.gexec[p], ms_.graph[p], 0));
}

// right-preconditioned GMRES(m) on K d = r from d = 0; returns iterations, relative reduction in *rel.
// Per cycle: the captured Arnoldi loop, y = R^{-1} g, d += M^{-1} V y on the device, one host read
// of the cycle's outcome; on restart t = r - K d and one host read of |t|.
template <typename T>
int Solver::ms_gmres(const T* r, T* d, double tol, int maxit, int mres, double* rel) {
    const long long Nm = ms_.N, ld = ms_.ld;
    T* V = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.V64.data()) : reinterpret_cast<T*>(ms_.V32.data());
    T* w = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.w64.data()) : reinterpret_cast<T*>(ms_.w32.data());
    T* t = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.t64.data()) : reinterpret_cast<T*>(ms_.t32.data());
    T* vn = sizeof(T) == 8 ? reinterpret_cast<T*>(ms_.vn64.data()) : reinterpret_cast<T*>(ms_.vn32.data());
    MsKrylov* K = reinterpret_cast<MsKrylov*>(ms_.kry.data());
    const int p = sizeof(T) == 4 ? 1 : 0;
    const int m = std::max(1, std::min(mres, MS_MAXM - 1));
    VG_CUDA(cudaMemsetAsync(d, 0, sizeof(T) * Nm, stream_));
    // residual of the current iterate, kept in t (r initially)
    VG_CUDA(cudaMemcpyAsync(t, r, sizeof(T) * Nm, cudaMemcpyDeviceToDevice, stream_));
    k_kry_init<<<1, 1, 0, stream_>>>(K, tol, m, maxit);
    ms_norm2<T>(t, K->hd + 2 * MS_MAXM + 1);
    double nr = 0;
    VG_CUDA(cudaMemcpyAsync(&nr, K->hd + 2 * MS_MAXM + 1, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    VG_CUDA(cudaStreamSynchronize(stream_));
    const double beta0 = std::sqrt(std::max(nr, 0.0));
    *rel = 1.0;
    if (!(beta0 > 0)) return 0;
    if (!ms_.gexec[p]) ms_build_graph<T>(p);
    struct {
        double rel;
        int its, done, reorth;
    } out{};
    for (int first = 1;; first = 0) {
        k_cycle_start<T><<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(t, V, vn, Nm, K, first);
        VG_CUDA(cudaGraphLaunch(ms_.gexec[p], stream_));
        k_trisolve<<<1, 1, 0, stream_>>>(K);
        k_combine<T><<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(V, ld, &K->j, K->y, w, Nm);
        ms_precond<T>(w, t);
        k_axpy_t<T><<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(d, t, 1.0, Nm);
        VG_CUDA(cudaGetLastError());
        VG_CUDA(cudaMemcpyAsync(&out.rel, &K->rel, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        VG_CUDA(cudaMemcpyAsync(&out.its, &K->its, sizeof(int), cudaMemcpyDeviceToHost, stream_));
        VG_CUDA(cudaMemcpyAsync(&out.done, &K->done, sizeof(int), cudaMemcpyDeviceToHost, stream_));
        VG_CUDA(cudaMemcpyAsync(&out.reorth, &K->reorth, sizeof(int), cudaMemcpyDeviceToHost, stream_));
        VG_CUDA(cudaStreamSynchronize(stream_));
        *rel = out.rel;
        if (out.done || out.its >= maxit) break;
        // restart: t = r - K d
        ms_apply<T>(d, w);
        if constexpr (sizeof(T) == 8) {
            k_sub<<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(reinterpret_cast<const double*>(r),
                                                         reinterpret_cast<const double*>(w),
                                                         reinterpret_cast<double*>(t), Nm);
        } else {
            VG_CUDA(cudaMemcpyAsync(t, r, sizeof(T) * Nm, cudaMemcpyDeviceToDevice, stream_));
            k_axpy_t<T><<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(t, w, -1.0, Nm);
        }
        ms_norm2<T>(t, K->hd + 2 * MS_MAXM + 1);
        VG_CUDA(cudaMemcpyAsync(&nr, K->hd + 2 * MS_MAXM + 1, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        VG_CUDA(cudaStreamSynchronize(stream_));
        const double beta = std::sqrt(std::max(nr, 0.0));
        *rel = beta / beta0;
        if (*rel <= tol || !(beta > 0)) break;
    }
    ms_arnoldi_steps_ += out.its;
    ms_reorth_passes_ += out.reorth;
    return out.its;
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
    k_ms_coeff<<<ms_blocks(m.nc), MS_THREADS, 0, stream_>>>(state, 2 * nf, m.nc, ms_.i12, ms_.i13, ms_.i23, ms_.B64.data(),
                                               ms_.B32.data());
    VG_CUDA(cudaGetLastError());
}

void Solver::ms_set_picard(int max_iterations, double tol) {
    if (max_iterations < 1 || !(tol > 0)) throw Error(VG_EINVAL, "Picard needs max_iterations >= 1 and tol > 0");
    ms_picard_max_ = max_iterations;
    ms_picard_tol_ = tol;
}

// One backward-Euler step. With one Picard iteration (the default) the friction matrix is taken at
// x^n and one linear system is solved (linearly implicit). With more, the friction matrix is
// re-evaluated at the latest iterate and the system solved again, until the relative change of
// the iterate is at most the Picard tolerance and the nonlinear residual ||b - K(x) x|| / ||b||,
// with K(x) at the accepted state, is at most max(Picard tolerance, 5 linear tolerance): the
// acceptance of the reference's time loop (vem/CurvedVEM_Darcy_gpu/src/solver_driver.cpp:209-240).
void Solver::ms_step(const double* old_state, double* new_state, const vg_solve_opts& o, vg_solve_info& info) {
    if (!ms_.ready) throw Error(VG_ESTATE, "vg_ms_configure must run before vg_ms_step");
    if (!(o.tol > 0) || o.maxit < 1 || (o.mode == VG_SOLVE_MIXED && !(o.inner_tol > 0 && o.inner_tol < 1)))
        throw Error(VG_EINVAL, "invalid solve options");
    info = vg_solve_info{};
    ms_last_picard_ = 0;
    ms_last_change_ = ms_last_nonlinear_ = 0.0;
    const long long Nm = ms_.N;
    const int P = ms_picard_max_;
    VG_CUDA(cudaDeviceSynchronize());  // the states may come from any stream
    VG_CUDA(cudaEventRecord(ev0_, stream_));
    if (P > 1) {
        ms_.prev.resize(Nm);
        VG_CUDA(cudaMemcpyAsync(ms_.prev.data(), old_state, sizeof(double) * Nm, cudaMemcpyDeviceToDevice, stream_));
    }
    // friction coefficients and the block preconditioner at a state
    auto prepare = [&](const double* coeff_state) {
        ms_coefficients(coeff_state);
        VG_CUDA(cudaMemsetAsync(ms_.D.data(), 0, sizeof(double) * ms_.D.size(), stream_));
        k_ms_pc_flux<<<ms_blocks((long long)pieces_.size() * PIECE), MS_THREADS, 0, stream_>>>(
            d_A0_.data(), d_map_.data(), d_pieces_.data(), int(pieces_.size()), d_slot_cell_.data(), ms_.B64.data(),
            d_mask_.data(), ms_.D.data());
        k_ms_pc_flux_inv<<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(ms_.D.data(), d_mask_.data(), nf, ms_.F64.data(),
                                                                ms_.F32.data());
        k_ms_pc_cell<<<ms_blocks((long long)pieces_.size() * PIECE), MS_THREADS, 0, stream_>>>(
            d_map_.data(), d_pieces_.data(), int(pieces_.size()), d_slot_cell_.data(), d_mask_.data(), ms_.F64.data(),
            ms_.m64.data(), ms_.C64.data(), ms_.C32.data());
        VG_CUDA(cudaGetLastError());
    };
    prepare(old_state);
    if (!ms_.amg_ready) {
        VG_CUDA(cudaStreamSynchronize(stream_));
        try {
            ms_build_amg();
        } catch (const Error&) {
            ms_.amg_ready = false;  // the 2x2 cell blocks stay in use
        }
    }
    k_ms_rhs<<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(old_state, ms_.m64.data(), nf, m.nc, ms_.b.data());
    VG_CUDA(cudaGetLastError());
    // initial guess: the old state
    if (new_state != old_state)
        VG_CUDA(cudaMemcpyAsync(new_state, old_state, sizeof(double) * Nm, cudaMemcpyDeviceToDevice, stream_));
    auto true_residual = [&](double* nb_out) {
        ms_apply<double>(new_state, ms_.y.data());
        k_sub<<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(ms_.b.data(), ms_.y.data(), ms_.r.data(), Nm);
        const double nr = ms_norm<double>(ms_.r.data()), nbv = ms_norm<double>(ms_.b.data());
        if (nb_out) *nb_out = nbv;
        return nr / (nbv > 0 ? nbv : 1.0);
    };
    int total = 0, outer = 0;
    double rel = 0;
    bool accepted = P == 1;
    const int mres = VG_MS_RESTART;
    for (int pic = 0; pic < P; ++pic) {
        if (pic > 0) {
            // the next linear system: friction at the latest iterate, started from it
            VG_CUDA(cudaMemcpyAsync(ms_.prev.data(), new_state, sizeof(double) * Nm, cudaMemcpyDeviceToDevice,
                                    stream_));
            prepare(ms_.prev.data());
        }
        double nb = 0;
        rel = true_residual(&nb);
        int steps = 0;
        if (o.mode == VG_SOLVE_FP64) {
            for (steps = 0; steps < 4 && rel > o.tol && total < o.maxit; ++steps) {
                double r_in = 0;
                const double rn = rel * nb;
                total += ms_gmres<double>(ms_.r.data(), ms_.d.data(), std::min(0.5, 0.5 * o.tol * nb / rn),
                                          o.maxit - total, mres, &r_in);
                k_axpy_t<double><<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(new_state, ms_.d.data(), 1.0, Nm);
                rel = true_residual(nullptr);
            }
        } else {
            for (steps = 0; steps < o.max_outer && rel > o.tol && total < o.maxit; ++steps) {
                const double rn = rel * nb;
                k_d2f<<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(ms_.r.data(), ms_.r32.data(), Nm, 1.0 / rn);
                double r_in = 0;
                // reduction asked of this FP32 solve: inner_tol, or less when less reaches tol
                const double itol = std::min(0.5, std::max(o.inner_tol, 0.5 * o.tol / rel));
                total += ms_gmres<float>(ms_.r32.data(), ms_.d32.data(), itol, o.maxit - total, mres, &r_in);
                k_addf<<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(new_state, ms_.d32.data(), rn, Nm);
                rel = true_residual(nullptr);
            }
        }
        outer += steps;
        ms_last_picard_ = pic + 1;
        if (P == 1) break;
        if (!(rel <= o.tol)) break;  // the linear solve failed: reported below
        // relative change of the iterate (the reference's measure: all unknowns, against max(1, |x|))
        k_sub<<<MS_BLOCKS, MS_THREADS, 0, stream_>>>(new_state, ms_.prev.data(), ms_.y.data(), Nm);
        const double change = ms_norm<double>(ms_.y.data()) / std::max(1.0, ms_norm<double>(new_state));
        ms_last_change_ = change;
        if (change <= ms_picard_tol_) {
            // nonlinear residual with the friction matrix at the accepted state
            prepare(new_state);
            const double nonlinear = true_residual(nullptr);
            ms_last_nonlinear_ = nonlinear;
            if (nonlinear <= std::max(ms_picard_tol_, 5.0 * o.tol)) {
                accepted = true;
                break;
            }
        }
    }
    VG_CUDA(cudaEventRecord(ev1_, stream_));
    VG_CUDA(cudaEventSynchronize(ev1_));
    float ms = 0;
    VG_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    info.iterations = total;
    info.outer = outer;
    info.residual = rel;
    info.seconds = ms * 1e-3;
    n_iter += total;
    ++n_solve;
    for (auto& a : ms_.amg)
        if (a.ready() && a.failed()) throw Error(VG_ECUDA, "multigrid copy wait timed out");
    if (!(rel <= o.tol))
        throw Error(VG_ENOCONV, "Maxwell-Stefan step did not converge: iterations=" + std::to_string(total) +
                                    " true_relative_residual=" + std::to_string(rel));
    if (!accepted)
        throw Error(VG_ENOCONV, "Maxwell-Stefan Picard iteration did not converge in " + std::to_string(P) +
                                    " iterations: relative change " + std::to_string(ms_last_change_));
}

template void Solver::ms_apply<double>(const double*, double*);
template void Solver::ms_apply<float>(const float*, float*);

}  // namespace vg
