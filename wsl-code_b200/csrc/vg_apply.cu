// Matrix-free saddle-point apply, one thread per polygon.
//
//   y = sum_E R_E^T S_E [A_E, -W_E^T; s W_E, 0] S_E R_E x  (+ multiplier row/column, BC mask)
//
// replaces element_apply + finish_apply (vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:198-279).
// The reference applies the factored form P^T AG P + alpha (I - DP)^T (I - DP) with one block
// per cell re-reading ragged factors from global memory; here the local flux operator is the
// packed symmetric A_E formed once by the setup kernel, stored slot-major inside each edge-count
// bucket so that consecutive threads read consecutive words of every entry (fully coalesced
// streams), and the whole local matvec runs in registers (fully unrolled for k in {0, 1} and
// n_e <= 12, a generic loop otherwise).
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

template <int NT>
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
        for (int i = 0; i < NT / 32; ++i) {
            a += sh[i][0];
            b += sh[i][1];
        }
    }
}

// partial sums of (quad, multiplier row) of this block; the last block of the whole apply sums
// all partials in a fixed order and writes quad to red[0] and the multiplier row of y
template <typename T>
__device__ void finish_reduction(const ApplyArgs<T>& a, double quad, double msum) {
    __shared__ double sh[8][2];
    __shared__ bool last;
    block_reduce2<256>(quad, msum, sh);
    if (threadIdx.x == 0) {
        a.partials[2 * (a.block_off + blockIdx.x)] = quad;
        a.partials[2 * (a.block_off + blockIdx.x) + 1] = msum;
        __threadfence();
        unsigned done = atomicAdd(a.counter, 1u);
        last = done == unsigned(a.total_blocks - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    int nb = a.total_blocks, t = threadIdx.x;
    int chunk = (nb + 255) / 256, lo = t * chunk, hi = min(nb, lo + chunk);
    double q = 0, s = 0;
    for (int i = lo; i < hi; ++i) {
        q += __ldcg(a.partials + 2 * i);
        s += __ldcg(a.partials + 2 * i + 1);
    }
    __shared__ double tq[256], ts[256];
    tq[t] = q;
    ts[t] = s;
    __syncthreads();
    for (int st = 128; st; st >>= 1) {
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

template <typename T, int K, int NE>
__global__ void __launch_bounds__(256) apply_tpl(ApplyArgs<T> a, Bucket b) {
    constexpr int Q = (K + 1) * (K + 2) / 2, NI = Q - 1 + K * (K + 1) / 2, ED = (K + 1) * NE, N = ED + NI;
    if (a.flags && a.flags[0]) return;  // solver converged: skip
    const int m = b.count;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double quad = 0, msum = 0;
    if (j < m) {
        int g[N];
        T u[N], yu[N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            int gi = __ldg(a.map + b.map_off + (long long)i * m + j);
            g[i] = gi;
            int idx = gi < 0 ? ~gi : gi;
            T xv = a.x[idx];
            if (i < ED && a.constrained && a.mask[idx]) xv = T(0);
            u[i] = gi < 0 ? -xv : xv;
            yu[i] = T(0);
        }
        const int cell = __ldg(a.slot_cell + b.slot + j);
        const long long pb = a.nf + (long long)cell * Q;
        T pr[Q];
#pragma unroll
        for (int r = 0; r < Q; ++r) pr[r] = a.x[pb + r];
        const T* A = a.A + b.a_off + j;
        int e = 0;
#pragma unroll
        for (int i = 0; i < N; ++i) {
#pragma unroll
            for (int c = i; c < N; ++c) {
                T v = __ldg(A + (long long)(e++) * m);
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
            const T* W = a.W + b.w_off + j;
#pragma unroll
            for (int r = 0; r < Q; ++r)
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    T w = __ldg(W + (long long)(r * N + i) * m);
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
            int gi = g[i], idx = gi < 0 ? ~gi : gi;
            if (a.constrained && a.mask[idx]) {
                T xv = a.x[idx];
                a.y[idx] = xv;
                quad += double(xv) * double(xv);
            } else {
                atomicAdd(a.y + idx, gi < 0 ? -yu[i] : yu[i]);
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
    if (a.red || a.mult) finish_reduction(a, quad, msum);
}

// generic path: any k, any edge count up to MAX_NE, local arrays in thread-local memory
constexpr int GEN_MAXN = 5 * MAX_NE + 24;
template <typename T>
__global__ void __launch_bounds__(256) apply_generic(ApplyArgs<T> a, Bucket b, int K) {
    if (a.flags && a.flags[0]) return;
    const int Q = (K + 1) * (K + 2) / 2, NE = b.ne, ED = (K + 1) * NE, N = b.n;
    const int m = b.count;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double quad = 0, msum = 0;
    if (j < m) {
        int g[GEN_MAXN];
        T u[GEN_MAXN], yu[GEN_MAXN], pr[15], yp[15];
        for (int i = 0; i < N; ++i) {
            int gi = a.map[b.map_off + (long long)i * m + j];
            g[i] = gi;
            int idx = gi < 0 ? ~gi : gi;
            T xv = a.x[idx];
            if (i < ED && a.constrained && a.mask[idx]) xv = T(0);
            u[i] = gi < 0 ? -xv : xv;
            yu[i] = T(0);
        }
        const int cell = a.slot_cell[b.slot + j];
        const long long pb = a.nf + (long long)cell * Q;
        for (int r = 0; r < Q; ++r) {
            pr[r] = a.x[pb + r];
            yp[r] = T(0);
        }
        const T* A = a.A + b.a_off + j;
        long long e = 0;
        for (int i = 0; i < N; ++i)
            for (int c = i; c < N; ++c) {
                T v = A[(e++) * m];
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
            const T* W = a.W + b.w_off + j;
            for (int r = 0; r < Q; ++r)
                for (int i = 0; i < N; ++i) {
                    T w = W[(long long)(r * N + i) * m];
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
    if (a.red || a.mult) finish_reduction(a, quad, msum);
}

template <typename T, int K, int NE>
void launch_one(const ApplyArgs<T>& a, const Bucket& b, int blocks, cudaStream_t s) {
    apply_tpl<T, K, NE><<<blocks, 256, 0, s>>>(a, b);
}

template <typename T, int K>
bool launch_k(const ApplyArgs<T>& a, const Bucket& b, int blocks, cudaStream_t s) {
    switch (b.ne) {
    case 3: launch_one<T, K, 3>(a, b, blocks, s); return true;
    case 4: launch_one<T, K, 4>(a, b, blocks, s); return true;
    case 5: launch_one<T, K, 5>(a, b, blocks, s); return true;
    case 6: launch_one<T, K, 6>(a, b, blocks, s); return true;
    case 7: launch_one<T, K, 7>(a, b, blocks, s); return true;
    case 8: launch_one<T, K, 8>(a, b, blocks, s); return true;
    case 9: launch_one<T, K, 9>(a, b, blocks, s); return true;
    case 10: launch_one<T, K, 10>(a, b, blocks, s); return true;
    case 11: launch_one<T, K, 11>(a, b, blocks, s); return true;
    case 12: launch_one<T, K, 12>(a, b, blocks, s); return true;
    }
    return false;
}

}  // namespace

int apply_blocks(const std::vector<Bucket>& buckets) {
    int t = 0;
    for (const auto& b : buckets) t += (b.count + 255) / 256;
    return t;
}

template <typename T>
void launch_apply(ApplyArgs<T> a, const std::vector<Bucket>& buckets, int k, cudaStream_t s) {
    a.total_blocks = apply_blocks(buckets);
    int off = 0;
    for (const auto& b : buckets) {
        int blocks = (b.count + 255) / 256;
        if (blocks == 0) continue;
        a.block_off = off;
        bool done = false;
        if (k == 0)
            done = launch_k<T, 0>(a, b, blocks, s);
        else if (k == 1)
            done = launch_k<T, 1>(a, b, blocks, s);
        if (!done) apply_generic<T><<<blocks, 256, 0, s>>>(a, b, k);
        VG_CUDA(cudaGetLastError());
        off += blocks;
    }
}

template void launch_apply<double>(ApplyArgs<double>, const std::vector<Bucket>&, int, cudaStream_t);
template void launch_apply<float>(ApplyArgs<float>, const std::vector<Bucket>&, int, cudaStream_t);

}  // namespace vg
