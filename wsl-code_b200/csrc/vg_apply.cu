// Matrix-free saddle-point apply, one thread per polygon.
//
//   y = sum_E R_E^T S_E [A_E, -W_E^T; s W_E, 0] S_E R_E x  (+ multiplier row/column, BC mask)
//
// replaces element_apply + finish_apply (vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:198-279).
// The reference applies the factored form P^T AG P + alpha (I - DP)^T (I - DP) with one block
// per cell re-reading ragged factors from global memory; here the local flux operator is the
// packed symmetric A_E formed once by the setup kernel. One warp handles one piece (up to 32
// cells of one edge count inside one compact mesh region, vg_common.cuh); every entry of the
// piece is one coalesced load of the warp, all operator loads are issued before the dependent
// gathers of x, and the local matvec runs in registers (fully unrolled for k in {0, 1} and
// n_e in 3..9, a generic loop otherwise). The whole apply is a single launch.
//
// Scatter: flux edge moments are shared by at most two cells. They are accumulated with one
// atomicAdd per local edge dof into a zeroed y; with at most two addends onto 0 the result is
// independent of the order (IEEE addition is commutative), so the apply is bitwise
// deterministic. Interior moments, pressure rows and masked (essential-BC) rows have a single
// owner and are plain stores.
//
// s = psign: +1 gives the reference sign [A, -W^T; W, 0]; -1 the symmetric form used by MINRES.
// Optionally the local quadratic form x^T K x is reduced (deterministic two-level sum, last block
// finishes), which MINRES needs as delta_j before it can update its Lanczos vectors.
#include "vg_apply.cuh"

namespace vg {

namespace {

__device__ __forceinline__ void block_reduce2(double& a, double& b, double (*sh)[2]) {
    for (int off = 16; off; off >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, off);
        b += __shfl_down_sync(0xffffffffu, b, off);
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sh[w][0] = a;
        sh[w][1] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = 0;
        b = 0;
        for (int i = 0; i < APPLY_THREADS / 32; ++i) {
            a += sh[i][0];
            b += sh[i][1];
        }
    }
}

// partial sums of (quad, multiplier row) of this block; the last block to finish sums all
// partials in a fixed order and writes quad to red[0] and the multiplier row of y
template <typename T>
__device__ void finish_reduction(const ApplyArgs<T>& a, double quad, double msum) {
    __shared__ double sh[APPLY_THREADS / 32][2];
    __shared__ bool last;
    block_reduce2(quad, msum, sh);
    if (threadIdx.x == 0) {
        a.partials[2 * blockIdx.x] = quad;
        a.partials[2 * blockIdx.x + 1] = msum;
        __threadfence();
        unsigned done = atomicAdd(a.counter, 1u);
        last = done == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int nb = gridDim.x, t = threadIdx.x;
    double q = 0, s = 0;
    for (int i = t; i < nb; i += APPLY_THREADS) {
        q += __ldcg(a.partials + 2 * i);
        s += __ldcg(a.partials + 2 * i + 1);
    }
    __shared__ double tq[APPLY_THREADS], ts[APPLY_THREADS];
    tq[t] = q;
    ts[t] = s;
    __syncthreads();
    for (int st = APPLY_THREADS / 2; st; st >>= 1) {
        if (t < st) {
            tq[t] += tq[t + st];
            ts[t] += ts[t + st];
        }
        __syncthreads();
    }
    if (t == 0) {
        if (a.red) a.red[0] = tq[0];
        if (a.mult) a.y[a.N - 1] = T(a.psign * ts[0]);
        *a.counter = 0u;
    }
}

// one lane = one cell of the piece; K and NE compile-time
template <typename T, int K, int NE>
__device__ __forceinline__ void piece_apply(const ApplyArgs<T>& a, const Piece& P, int lane, double& quad,
                                            double& msum) {
    constexpr int Q = (K + 1) * (K + 2) / 2, NI = Q - 1 + K * (K + 1) / 2, ED = (K + 1) * NE, N = ED + NI;
    constexpr int NPK = N * (N + 1) / 2, NW = K == 0 ? 1 : Q * N;
    // small blocks (k = 0): every operator load is issued before the dependent gathers of x
    constexpr bool PRE = NPK <= 48;
    constexpr int NAV = PRE ? NPK : 1;
    if (lane >= P.count) return;
    const T* A = a.A + P.a_off + lane;
    T av[NAV];
    if (PRE) {
#pragma unroll
        for (int e = 0; e < NAV; ++e) av[e] = __ldg(A + e * PIECE);
    }
    const T* W = a.W + P.w_off + lane;
    int g[N];
#pragma unroll
    for (int i = 0; i < N; ++i) g[i] = __ldg(a.map + P.map_off + i * PIECE + lane);
    const int cell = __ldg(a.slot_cell + P.slot + lane);
    const long long pb = a.nf + (long long)cell * Q;
    T u[N], yu[N], pr[Q];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        int idx = g[i] < 0 ? ~g[i] : g[i];
        T xv = a.x[idx];
        if (i < ED && a.constrained && a.mask[idx]) xv = T(0);
        u[i] = g[i] < 0 ? -xv : xv;
        yu[i] = T(0);
    }
#pragma unroll
    for (int r = 0; r < Q; ++r) pr[r] = a.x[pb + r];
    int e = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
#pragma unroll
        for (int c = i; c < N; ++c) {
            T v = PRE ? av[PRE ? e : 0] : __ldg(A + e * PIECE);
            ++e;
            yu[i] += v * u[c];
            if (c != i) yu[c] += v * u[i];
        }
    }
    if (a.red) {
#pragma unroll
        for (int i = 0; i < N; ++i) quad += double(u[i]) * double(yu[i]);
    }
    T yp[Q];
#pragma unroll
    for (int r = 0; r < Q; ++r) yp[r] = T(0);
    if (K == 0) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            yu[i] -= pr[0];
            yp[0] += u[i];
        }
    } else {
#pragma unroll
        for (int r = 0; r < Q; ++r)
#pragma unroll
            for (int i = 0; i < N; ++i) {
                T w = __ldg(W + (r * N + i) * PIECE);
                yu[i] -= w * pr[r];
                yp[r] += w * u[i];
            }
    }
    if (a.red) {
#pragma unroll
        for (int r = 0; r < Q; ++r) quad += (double(a.psign) - 1.0) * double(pr[r]) * double(yp[r]);
    }
#pragma unroll
    for (int i = 0; i < ED; ++i) {
        int idx = g[i] < 0 ? ~g[i] : g[i];
        if (a.constrained && a.mask[idx]) {
            T xv = a.x[idx];
            a.y[idx] = xv;
            quad += double(xv) * double(xv);
        } else {
            atomicAdd(a.y + idx, g[i] < 0 ? -yu[i] : yu[i]);
        }
    }
#pragma unroll
    for (int i = ED; i < N; ++i) a.y[g[i]] = yu[i];
    if (a.mult) {
        T lam = a.x[a.N - 1];
#pragma unroll
        for (int r = 0; r < Q; ++r) {
            T l = a.L[(long long)cell * Q + r];
            yp[r] += l * lam;
            msum += double(l) * double(pr[r]);
        }
        if (a.red) quad += 2.0 * double(a.psign) * double(lam) * msum;
    }
#pragma unroll
    for (int r = 0; r < Q; ++r) a.y[pb + r] = a.psign * yp[r];
}

// generic path: any k, any edge count up to MAX_NE, local arrays in thread-local memory
constexpr int GEN_MAXN = 5 * MAX_NE + 24;
template <typename T>
__device__ void piece_apply_generic(const ApplyArgs<T>& a, const Piece& P, int lane, double& quad, double& msum) {
    if (lane >= P.count) return;
    const int K = a.k, Q = (K + 1) * (K + 2) / 2, NE = P.ne, ED = (K + 1) * NE, N = P.n;
    int g[GEN_MAXN];
    T u[GEN_MAXN], yu[GEN_MAXN], pr[15], yp[15];
    for (int i = 0; i < N; ++i) {
        int gi = a.map[P.map_off + (long long)i * PIECE + lane];
        g[i] = gi;
        int idx = gi < 0 ? ~gi : gi;
        T xv = a.x[idx];
        if (i < ED && a.constrained && a.mask[idx]) xv = T(0);
        u[i] = gi < 0 ? -xv : xv;
        yu[i] = T(0);
    }
    const int cell = a.slot_cell[P.slot + lane];
    const long long pb = a.nf + (long long)cell * Q;
    for (int r = 0; r < Q; ++r) {
        pr[r] = a.x[pb + r];
        yp[r] = T(0);
    }
    const T* A = a.A + P.a_off + lane;
    long long e = 0;
    for (int i = 0; i < N; ++i)
        for (int c = i; c < N; ++c) {
            T v = A[(e++) * PIECE];
            yu[i] += v * u[c];
            if (c != i) yu[c] += v * u[i];
        }
    if (a.red)
        for (int i = 0; i < N; ++i) quad += double(u[i]) * double(yu[i]);
    if (K == 0) {
        for (int i = 0; i < N; ++i) {
            yu[i] -= pr[0];
            yp[0] += u[i];
        }
    } else {
        const T* W = a.W + P.w_off + lane;
        for (int r = 0; r < Q; ++r)
            for (int i = 0; i < N; ++i) {
                T w = W[(long long)(r * N + i) * PIECE];
                yu[i] -= w * pr[r];
                yp[r] += w * u[i];
            }
    }
    if (a.red)
        for (int r = 0; r < Q; ++r) quad += (double(a.psign) - 1.0) * double(pr[r]) * double(yp[r]);
    for (int i = 0; i < ED; ++i) {
        int gi = g[i], idx = gi < 0 ? ~gi : gi;
        if (a.constrained && a.mask[idx]) {
            T xv = a.x[idx];
            a.y[idx] = xv;
            quad += double(xv) * double(xv);
        } else {
            atomicAdd(a.y + idx, gi < 0 ? -yu[i] : yu[i]);
        }
    }
    for (int i = ED; i < N; ++i) a.y[g[i]] = yu[i];
    if (a.mult) {
        T lam = a.x[a.N - 1];
        for (int r = 0; r < Q; ++r) {
            T l = a.L[(long long)cell * Q + r];
            yp[r] += l * lam;
            msum += double(l) * double(pr[r]);
        }
        if (a.red) quad += 2.0 * double(a.psign) * double(lam) * msum;
    }
    for (int r = 0; r < Q; ++r) a.y[pb + r] = a.psign * yp[r];
}

template <typename T, int K>
__global__ void __launch_bounds__(APPLY_THREADS) apply_kernel(ApplyArgs<T> a) {
    if (a.flags && a.flags[0]) return;  // solver converged: skip
    const int warp = (blockIdx.x * APPLY_THREADS + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    double quad = 0, msum = 0;
    if (warp < a.npieces) {
        const Piece P = a.pieces[warp];
        if (K == 0 || K == 1) {
            switch (P.ne) {
            case 3: piece_apply<T, K, 3>(a, P, lane, quad, msum); break;
            case 4: piece_apply<T, K, 4>(a, P, lane, quad, msum); break;
            case 5: piece_apply<T, K, 5>(a, P, lane, quad, msum); break;
            case 6: piece_apply<T, K, 6>(a, P, lane, quad, msum); break;
            case 7: piece_apply<T, K, 7>(a, P, lane, quad, msum); break;
            case 8: piece_apply<T, K, 8>(a, P, lane, quad, msum); break;
            case 9: piece_apply<T, K, 9>(a, P, lane, quad, msum); break;
            default: piece_apply_generic<T>(a, P, lane, quad, msum);
            }
        } else {
            piece_apply_generic<T>(a, P, lane, quad, msum);
        }
    }
    if (a.red || a.mult) finish_reduction(a, quad, msum);
}

}  // namespace

int apply_blocks(int npieces) { return (npieces * 32 + APPLY_THREADS - 1) / APPLY_THREADS; }

template <typename T>
void launch_apply(ApplyArgs<T> a, cudaStream_t s) {
    int blocks = apply_blocks(a.npieces);
    if (blocks == 0) return;
    if (a.k == 0)
        apply_kernel<T, 0><<<blocks, APPLY_THREADS, 0, s>>>(a);
    else if (a.k == 1)
        apply_kernel<T, 1><<<blocks, APPLY_THREADS, 0, s>>>(a);
    else
        apply_kernel<T, 2><<<blocks, APPLY_THREADS, 0, s>>>(a);
    VG_CUDA(cudaGetLastError());
}

template void launch_apply<double>(ApplyArgs<double>, cudaStream_t);
template void launch_apply<float>(ApplyArgs<float>, cudaStream_t);

}  // namespace vg
