// Matrix-free saddle-point apply.
//
//   y = sum_E R_E^T S_E [A_E, -W_E^T; s W_E, 0] S_E R_E x  (+ multiplier row/column, BC mask)
//
// replaces element_apply + finish_apply (vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:198-279).
// The reference applies the factored form P^T AG P + alpha (I - DP)^T (I - DP) with one block
// per cell re-reading ragged factors from global memory; here the local flux operator is the
// packed symmetric A_E formed once by the setup kernel, and one lane handles one polygon.
//
// Two kernels share the per-cell body:
//
// * apply_bulk_kernel (k <= 1, the production path): the operator of every piece (up to 32
//   cells of one edge count, vg_common.cuh) is one contiguous record of the record stream
//   (A_E, W_E, signed map and cell ids, lane-strided). Persistent CTAs own contiguous runs of
//   records; one producer thread streams them with cp.async.bulk into a ring of shared-memory
//   stages (mbarrier completion), consumer warps (two groups, each owning alternate stages) run
//   the cell bodies out of shared memory and release each stage on an "empty" mbarrier. Bytes in flight are set by the ring, not by how
//   many warps fit on an SM, so the stream runs at HBM speed with few resident warps. Every
//   wait is bounded (globaltimer); a wait that gives up sets an error word, drains the copies
//   it issued and returns.
// * apply_kernel (any k): one warp per piece reading the strided global arrays (used for
//   k >= 2 and for pieces whose record does not fit a stage).
//
// Scatter: flux edge moments are shared by at most two cells. They are accumulated with one
// reduction (red.global.add) per local edge dof into a zeroed y; with at most two addends onto 0 the result is
// independent of the order (IEEE addition is commutative), so the apply is bitwise
// deterministic. Interior moments, pressure rows and masked (essential-BC) rows have a single
// owner and are plain stores.
//
// s = psign: +1 gives the reference sign [A, -W^T; W, 0]; -1 the symmetric form used by MINRES.
// Optionally the local quadratic form x^T K x is reduced (deterministic two-level sum, last block
// finishes), which MINRES needs as delta_j before it can update its Lanczos vectors.
#include <algorithm>

#include "vg_apply.cuh"
#include "vg_pipe.cuh"

namespace vg {

namespace {

#ifndef VG_BULK_CONSUMERS
#define VG_BULK_CONSUMERS 8
#endif
#ifndef VG_STAGE_MIN_KB
#define VG_STAGE_MIN_KB 24  // FP64 records; FP32 records use two thirds of it
#endif
#ifndef VG_CTAS_PER_SM
#define VG_CTAS_PER_SM 2  // FP64; FP32 (fewer registers per cell) runs one more CTA per SM
#endif
#ifndef VG_BULK_DIRECT_SPEC
#define VG_BULK_DIRECT_SPEC 0  // 1: the streamed kernel's direct (oversized) pieces use the specialised bodies too
#endif
#ifndef VG_BULK_GROUPS
#define VG_BULK_GROUPS 2
#endif
constexpr int BULK_CONSUMERS = VG_BULK_CONSUMERS;       // consumer warps per CTA
// The consumer warps form BULK_GROUPS groups; group g consumes the stages of batches i with
// i % BULK_GROUPS == g. A stage holds only 3-4 piece records at k = 0, so a group of a few warps
// is enough for it, and each warp waits on, walks and releases only its group's stages instead of
// every stage. The stage count is a multiple of BULK_GROUPS, so a ring slot is always consumed by
// the same group and every waiter is at most one phase ahead of its slot's barrier.
constexpr int BULK_GROUPS = VG_BULK_GROUPS;
constexpr int GROUP_WARPS = BULK_CONSUMERS / BULK_GROUPS;
static_assert(BULK_CONSUMERS % BULK_GROUPS == 0, "consumer warps split evenly into groups");
// smallest shared-memory stage and resident CTAs per SM (k = 0), by element size: measured at 1M
// cells, FP32 runs 3 CTAs of 72 registers per thread with 16 KB stages (apply 39.0 -> 38.0 us),
// FP64 stays at 2 CTAs of 96 registers (3 CTAs spill and take 70 us instead of 56)
constexpr int stage_min(int elem_bytes) { return (elem_bytes == 4 ? 2 * VG_STAGE_MIN_KB / 3 : VG_STAGE_MIN_KB) << 10; }
constexpr int ctas_per_sm(int elem_bytes) { return elem_bytes == 4 ? VG_CTAS_PER_SM + 1 : VG_CTAS_PER_SM; }
constexpr int BULK_THREADS = 32 * (BULK_CONSUMERS + 1);  // + one producer warp
constexpr int MAX_STAGES = 4;
constexpr int MAX_RING_BYTES = 200 << 10;                // dynamic shared memory of the ring

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

// partial sums of (quad, multiplier row) of this block; the last block to finish sums all
// partials in a fixed order and writes quad to red[0] and the multiplier row of y
template <typename T, int NT>
__device__ void finish_reduction(const ApplyArgs<T>& a, double quad, double msum) {
    __shared__ double sh[NT / 32][2];
    __shared__ bool last;
    block_reduce2<NT>(quad, msum, sh);
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
    for (int i = t; i < nb; i += NT) {
        q += __ldcg(a.partials + 2 * i);
        s += __ldcg(a.partials + 2 * i + 1);
    }
    __shared__ double tq[NT], ts[NT];
    tq[t] = q;
    ts[t] = s;
    __syncthreads();
    // fixed-order tree: fold the block onto the largest power of two, then halve
    constexpr int P2 = NT >= 512 ? 512 : NT >= 256 ? 256 : NT >= 128 ? 128 : 64;
    if (P2 < NT && t < NT - P2) {
        tq[t] += tq[t + P2];
        ts[t] += ts[t + P2];
    }
    __syncthreads();
    for (int st = P2 / 2; st; st >>= 1) {
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

// scatter-add without a returned value (red, not atom): a persistent warp must not wait for the
// round trip of its previous piece's adds (same rounding as atomicAdd)
__device__ __forceinline__ void red_add(float* p, float v) {
    asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void red_add(double* p, double v) {
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// operator sources of one lane: strided global arrays or a record in shared memory
template <typename T>
struct GlobalSrc {
    const T* A;
    const T* W;
    const int* m;
    // operator entries are read once per apply: streaming loads (evict first)
    __device__ __forceinline__ T a(int e) const { return __ldcs(A + (long long)e * PIECE); }
    __device__ __forceinline__ T w(int j) const { return __ldcs(W + (long long)j * PIECE); }
    __device__ __forceinline__ int g(int i) const { return __ldcs(m + (long long)i * PIECE); }
};

template <typename T>
struct SmemSrc {
    const T* A;
    const T* W;
    const int* m;
    __device__ __forceinline__ T a(int e) const { return A[e * PIECE]; }
    __device__ __forceinline__ T w(int j) const { return W[j * PIECE]; }
    __device__ __forceinline__ int g(int i) const { return m[i * PIECE]; }
};

// one cell; K and NE compile-time. PRE: issue every operator load before the dependent gathers
template <typename T, int K, int NE, bool PRE, class Src>
__device__ __forceinline__ void cell_apply(const ApplyArgs<T>& a, const Src& src, int prow, double& quad,
                                           double& msum) {
    constexpr int Q = (K + 1) * (K + 2) / 2, NI = Q - 1 + K * (K + 1) / 2, ED = (K + 1) * NE, N = ED + NI;
    constexpr int NPK = N * (N + 1) / 2;
    constexpr int NAV = PRE ? NPK : 1;
    T av[NAV];
    if (PRE) {
#pragma unroll
        for (int e = 0; e < NAV; ++e) av[e] = src.a(e);
    }
    int g[N];
#pragma unroll
    for (int i = 0; i < N; ++i) g[i] = src.g(i);
    const long long pb = prow;
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
            T v = PRE ? av[PRE ? e : 0] : src.a(e);
            ++e;
            yu[i] += v * u[c];
            if (c != i) yu[c] += v * u[i];
        }
    }
    if (a.red) {
        // the cell's share of delta = x^T K x, summed in the operator's precision and promoted
        // once (an FP32 inner solve needs no FP64 products; fewer conversions per cell)
        T qc = T(0);
#pragma unroll
        for (int i = 0; i < N; ++i) qc += u[i] * yu[i];
        quad += double(qc);
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
                T w = src.w(r * N + i);
                yu[i] -= w * pr[r];
                yp[r] += w * u[i];
            }
    }
    if (a.red && a.psign != T(1)) {
        T qp = T(0);
#pragma unroll
        for (int r = 0; r < Q; ++r) qp += pr[r] * yp[r];
        quad += (double(a.psign) - 1.0) * double(qp);
    }
#pragma unroll
    for (int i = 0; i < ED; ++i) {
        int idx = g[i] < 0 ? ~g[i] : g[i];
        if (a.constrained && a.mask[idx]) {
            T xv = a.x[idx];
            a.y[idx] = xv;
            quad += double(xv) * double(xv);
        } else {
            red_add(a.y + idx, g[i] < 0 ? -yu[i] : yu[i]);
        }
    }
#pragma unroll
    for (int i = ED; i < N; ++i) a.y[g[i]] = yu[i];
    if (a.mult) {
        T lam = a.x[a.N - 1];
#pragma unroll
        for (int r = 0; r < Q; ++r) {
            T l = a.L[(pb - a.nf) + r];
            yp[r] += l * lam;
            msum += double(l) * double(pr[r]);
        }
        if (a.red) quad += 2.0 * double(a.psign) * double(lam) * msum;
    }
#pragma unroll
    for (int r = 0; r < Q; ++r) a.y[pb + r] = a.psign * yp[r];
}

// generic cell body: any k, any edge count up to MAX_NE, local arrays in thread-local memory
constexpr int GEN_MAXN = 5 * MAX_NE + 24;
template <typename T, class Src>
__device__ void cell_apply_generic(const ApplyArgs<T>& a, const Src& src, int ne, int n, int prow, double& quad,
                                   double& msum) {
    const int K = a.k, Q = (K + 1) * (K + 2) / 2, ED = (K + 1) * ne, N = n;
    int g[GEN_MAXN];
    T u[GEN_MAXN], yu[GEN_MAXN], pr[15], yp[15];
    for (int i = 0; i < N; ++i) {
        int gi = src.g(i);
        g[i] = gi;
        int idx = gi < 0 ? ~gi : gi;
        T xv = a.x[idx];
        if (i < ED && a.constrained && a.mask[idx]) xv = T(0);
        u[i] = gi < 0 ? -xv : xv;
        yu[i] = T(0);
    }
    const long long pb = prow;
    for (int r = 0; r < Q; ++r) {
        pr[r] = a.x[pb + r];
        yp[r] = T(0);
    }
    int e = 0;
    for (int i = 0; i < N; ++i)
        for (int c = i; c < N; ++c) {
            T v = src.a(e++);
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
        for (int r = 0; r < Q; ++r)
            for (int i = 0; i < N; ++i) {
                T w = src.w(r * N + i);
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
            red_add(a.y + idx, gi < 0 ? -yu[i] : yu[i]);
        }
    }
    for (int i = ED; i < N; ++i) a.y[g[i]] = yu[i];
    if (a.mult) {
        T lam = a.x[a.N - 1];
        for (int r = 0; r < Q; ++r) {
            T l = a.L[(pb - a.nf) + r];
            yp[r] += l * lam;
            msum += double(l) * double(pr[r]);
        }
        if (a.red) quad += 2.0 * double(a.psign) * double(lam) * msum;
    }
    for (int r = 0; r < Q; ++r) a.y[pb + r] = a.psign * yp[r];
}

template <int K, int NE>
__host__ __device__ constexpr bool prefetch_all() {
    constexpr int N = (K + 1) * NE + (K + 1) * (K + 2) / 2 - 1 + K * (K + 1) / 2;
    return N * (N + 1) / 2 <= 48;
}

// one lane of a piece read from the strided global arrays. SPEC: the cell bodies specialised by
// edge count; without it every piece takes the generic body (the streamed kernel's rare pieces too
// large for a stage, where a second set of specialised bodies would only add code)
template <typename T, int K, bool SPEC = true>
__device__ __forceinline__ void piece_global(const ApplyArgs<T>& a, const Piece& P, int lane, double& quad,
                                             double& msum) {
    if (lane >= P.count) return;
    GlobalSrc<T> src{a.A + P.a_off + lane, a.W + P.w_off + lane, a.map + P.map_off + lane};
    const int prow = __ldg(a.prow + P.slot + lane);  // first pressure row of the cell
    if constexpr (SPEC && (K == 0 || K == 1)) {
        switch (P.ne) {
        case 3: cell_apply<T, K, 3, prefetch_all<K, 3>()>(a, src, prow, quad, msum); return;
        case 4: cell_apply<T, K, 4, prefetch_all<K, 4>()>(a, src, prow, quad, msum); return;
        case 5: cell_apply<T, K, 5, prefetch_all<K, 5>()>(a, src, prow, quad, msum); return;
        case 6: cell_apply<T, K, 6, prefetch_all<K, 6>()>(a, src, prow, quad, msum); return;
        case 7: cell_apply<T, K, 7, prefetch_all<K, 7>()>(a, src, prow, quad, msum); return;
        case 8: cell_apply<T, K, 8, prefetch_all<K, 8>()>(a, src, prow, quad, msum); return;
        case 9: cell_apply<T, K, 9, prefetch_all<K, 9>()>(a, src, prow, quad, msum); return;
        default: break;
        }
    }
    cell_apply_generic<T>(a, src, P.ne, P.n, prow, quad, msum);
}

// one lane of a piece record in shared memory: header int4 {ne, n, count, bytes}
template <typename T, int K>
__device__ __forceinline__ void piece_record(const ApplyArgs<T>& a, const unsigned char* r, int4 h, int lane,
                                             double& quad, double& msum) {
    if (lane >= h.z) return;
    const int ne = h.x, n = h.y, npk = n * (n + 1) / 2, nw = K == 0 ? 0 : ((K + 1) * (K + 2) / 2) * n;
    const T* A = reinterpret_cast<const T*>(r + 16) + lane;
    const int* m = reinterpret_cast<const int*>(reinterpret_cast<const T*>(r + 16) + (npk + nw) * PIECE) + lane;
    SmemSrc<T> src{A, A + npk * PIECE, m};
    const int prow = m[n * PIECE];  // first pressure row of the cell
    switch (ne) {
    case 3: cell_apply<T, K, 3, false>(a, src, prow, quad, msum); return;
    case 4: cell_apply<T, K, 4, false>(a, src, prow, quad, msum); return;
    case 5: cell_apply<T, K, 5, false>(a, src, prow, quad, msum); return;
    case 6: cell_apply<T, K, 6, false>(a, src, prow, quad, msum); return;
    case 7: cell_apply<T, K, 7, false>(a, src, prow, quad, msum); return;
    case 8: cell_apply<T, K, 8, false>(a, src, prow, quad, msum); return;
    case 9: cell_apply<T, K, 9, false>(a, src, prow, quad, msum); return;
    default: cell_apply_generic<T>(a, src, ne, n, prow, quad, msum);
    }
}

template <typename T, int K>
__global__ void __launch_bounds__(APPLY_THREADS) apply_kernel(ApplyArgs<T> a) {
    if (a.flags && a.flags[0]) return;  // solver converged: skip
    const int warp = (blockIdx.x * APPLY_THREADS + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    double quad = 0, msum = 0;
    if (warp < a.npieces) piece_global<T, K>(a, a.pieces[warp], lane, quad, msum);
    if (a.red || a.mult) finish_reduction<T, APPLY_THREADS>(a, quad, msum);
}

template <typename T, int K>
__global__ void __launch_bounds__(BULK_THREADS, K == 0 ? ctas_per_sm(int(sizeof(T))) : 1)
    apply_bulk_kernel(ApplyArgs<T> a) {
    if (a.flags && a.flags[0]) return;  // solver converged: skip
    extern __shared__ __align__(128) unsigned char ring[];
    __shared__ __align__(8) unsigned long long full[MAX_STAGES], empty[MAX_STAGES];
    // descriptor of the batch in each stage, written by the producer before its arrival on
    // full[s] (release) and read by the consumers after their wait (acquire)
    __shared__ int st_first[MAX_STAGES], st_count[MAX_STAGES], st_direct[MAX_STAGES];
    __shared__ int abort_flag, issued_sh;
    __shared__ __align__(8) unsigned long long never;  // test hook: a barrier nothing arrives on
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b0 = a.cta_batch[blockIdx.x], nb = a.cta_batch[blockIdx.x + 1] - b0;
    const int S = a.stages, SB = a.stage_bytes;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], GROUP_WARPS);
        }
        mbar_init(&never, 1);
        abort_flag = 0;
        issued_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    double quad = 0, msum = 0;
    if (warp == 0) {
        if (lane == 0) {  // producer
            const unsigned long long pol = evict_first_policy();
            int issued = 0;
            bool ok = true;
            for (int i = 0; i < nb; ++i) {
                const int s = i % S;
                if (i >= S && !mbar_wait(&empty[s], unsigned((i / S) - 1) & 1u, &abort_flag)) {
                    ok = false;
                    break;
                }
                const ApplyBatch B = a.batches[b0 + i];
                st_first[s] = B.first;
                st_count[s] = B.count;
                st_direct[s] = B.bytes == 0;
                mbar_expect_tx(&full[s], unsigned(B.bytes));
                if (B.bytes) bulk_g2s(ring + size_t(s) * SB, a.rec + B.off, unsigned(B.bytes), &full[s], pol);
                issued = i + 1;
            }
            issued_sh = issued;
            if (!ok) {
                abort_flag = 1;
                *reinterpret_cast<volatile int*>(a.err) = 1;
            }
        }
    } else {  // consumers
        const int cw = warp - 1, grp = cw / GROUP_WARPS, gw = cw % GROUP_WARPS;
        // test hook (failure-path tests only): the first consumer warp 0 to find the flag set
        // clears it and, at the last batch of its group, waits on a barrier nothing arrives on, so
        // that its bounded wait runs out; the flag is loaded while the first stage is still in flight
        int stall_req = 0;
        if (cw == 0 && lane == 0 && a.stall) stall_req = *reinterpret_cast<volatile int*>(a.stall);
        for (int i = grp; i < nb; i += BULK_GROUPS) {
            const int s = i % S;
            bool ok = __all_sync(0xffffffffu, mbar_wait(&full[s], unsigned(i / S) & 1u, &abort_flag));
            if (cw == 0 && i + BULK_GROUPS >= nb) {
                int st = 0;
                if (lane == 0 && stall_req) st = atomicExch(a.stall, 0);
                if (__shfl_sync(0xffffffffu, st, 0)) ok = __all_sync(0xffffffffu, mbar_wait(&never, 0u, &abort_flag));
            }
            if (!ok) {
                if (lane == 0) {
                    abort_flag = 1;
                    *reinterpret_cast<volatile int*>(a.err) = 1;
                }
                break;
            }
            const int first = st_first[s], count = st_count[s];
            if (st_direct[s]) {
                for (int j = gw; j < count; j += GROUP_WARPS)
                    piece_global<T, K, VG_BULK_DIRECT_SPEC != 0>(a, a.pieces[first + j], lane, quad, msum);
            } else {
                const unsigned char* r = ring + size_t(s) * SB;
                for (int j = 0; j < count; ++j) {
                    const int4 h = *reinterpret_cast<const int4*>(r);
                    if ((first + j) % GROUP_WARPS == gw) piece_record<T, K>(a, r, h, lane, quad, msum);
                    r += h.w;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
    }
    __syncthreads();
    if (abort_flag && threadIdx.x == 0) {
        // a wait gave up (producer or consumers): the copies still in flight (at most one per
        // stage, the last ones issued) land before the CTA exits; bounded as well
        for (int i = max(0, issued_sh - S); i < issued_sh; ++i) mbar_wait(&full[i % S], unsigned(i / S) & 1u, nullptr);
    }
    if (a.red || a.mult) finish_reduction<T, BULK_THREADS>(a, quad, msum);
}

template <typename T>
__global__ void k_pack(const Piece* pieces, int np, const long long* rec_off, const T* A, const T* W, const int* map,
                       const int* prow, int k, unsigned char* out) {
    const int p = int((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (p >= np) return;
    const Piece P = pieces[p];
    unsigned char* r = out + rec_off[p];
    const int n = P.n, npk = n * (n + 1) / 2, nw = k ? dimP(k) * n : 0;
    if (lane == 0) *reinterpret_cast<int4*>(r) = make_int4(P.ne, n, P.count, int(rec_off[p + 1] - rec_off[p]));
    T* As = reinterpret_cast<T*>(r + 16);
    for (int e = 0; e < npk; ++e) As[e * PIECE + lane] = A[P.a_off + (long long)e * PIECE + lane];
    for (int j = 0; j < nw; ++j) As[(npk + j) * PIECE + lane] = W[P.w_off + (long long)j * PIECE + lane];
    int* m = reinterpret_cast<int*>(As + (npk + nw) * PIECE);
    for (int i = 0; i < n; ++i) m[i * PIECE + lane] = map[P.map_off + (long long)i * PIECE + lane];
    m[n * PIECE + lane] = prow[P.slot + lane];
}

}  // namespace

int apply_blocks(int npieces) { return (npieces * 32 + APPLY_THREADS - 1) / APPLY_THREADS; }

long long record_bytes(const Piece& P, int k, int elem_bytes) {
    const long long n = P.n, npk = n * (n + 1) / 2, nw = k ? (long long)dimP(k) * n : 0;
    return 16 + (npk + nw) * PIECE * elem_bytes + (n + 1) * PIECE * 4;
}

StreamPlan plan_stream(const std::vector<Piece>& pieces, int k, int elem_bytes, int sm_count) {
    StreamPlan pl;
    const int np = int(pieces.size());
    pl.rec_off.assign(np + 1, 0);
    long long common = 0;
    for (int p = 0; p < np; ++p) {
        const long long rb = record_bytes(pieces[p], k, elem_bytes);
        pl.rec_off[p + 1] = pl.rec_off[p] + rb;
        if (pieces[p].ne <= 9) common = std::max(common, rb);
    }
    pl.bytes = pl.rec_off[np];
    // stage: at least stage_min and the largest record of a polygon with <= 9 edges; bigger records
    // (and anything above 96 KB) are read from the strided arrays
    long long sb = std::max<long long>(stage_min(elem_bytes), (common + 1023) / 1024 * 1024);
    sb = std::min<long long>(sb, 96 << 10);
    pl.stage_bytes = int(sb);
    pl.stages = int(std::max<long long>(2, std::min<long long>(MAX_STAGES, MAX_RING_BYTES / sb)));
    pl.stages -= pl.stages % BULK_GROUPS;  // a ring slot always belongs to one consumer group
    static_assert(2 % BULK_GROUPS == 0 && MAX_STAGES % BULK_GROUPS == 0, "at least one stage per group");
    const int per_sm = int(std::max<long long>(
        1, std::min<long long>(k == 0 ? ctas_per_sm(elem_bytes) : 1, (227 << 10) / (pl.stages * sb + 8192))));
    // batches: runs of whole records up to one stage
    ApplyBatch cur{0, 0, 0, 0, {0, 0, 0}};
    std::vector<long long> work;
    auto flush = [&]() {
        if (cur.count) {
            pl.batches.push_back(cur);
            work.push_back(cur.bytes);
        }
        cur = ApplyBatch{0, 0, 0, 0, {0, 0, 0}};
    };
    for (int p = 0; p < np; ++p) {
        const long long rb = pl.rec_off[p + 1] - pl.rec_off[p];
        if (rb > sb) {
            flush();
            pl.batches.push_back(ApplyBatch{pl.rec_off[p], 0, p, 1, {0, 0, 0}});
            work.push_back(rb);
            continue;
        }
        if (cur.count && cur.bytes + rb > sb) flush();
        if (!cur.count) {
            cur.off = pl.rec_off[p];
            cur.first = p;
        }
        cur.bytes += int(rb);
        cur.count += 1;
    }
    flush();
    const int nbat = int(pl.batches.size());
    pl.ncta = std::max(0, std::min(nbat, sm_count * per_sm));
    pl.cta_batch.assign(pl.ncta + 1, nbat);
    if (pl.ncta) {
        long long total = 0;
        for (long long w : work) total += w;
        int c = 0;
        long long acc = 0;
        pl.cta_batch[0] = 0;
        for (int b = 0; b < nbat && c + 1 < pl.ncta; ++b) {
            acc += work[b];
            // cut after batch b once this CTA reached its share (and enough batches remain)
            if (acc * pl.ncta >= (long long)(c + 1) * total && nbat - (b + 1) >= pl.ncta - (c + 1))
                pl.cta_batch[++c] = b + 1;
        }
        while (c + 1 < pl.ncta) {  // not reached for sane inputs; keep ranges nonempty and ordered
            ++c;
            pl.cta_batch[c] = std::min(nbat, pl.cta_batch[c - 1] + 1);
        }
        pl.cta_batch[pl.ncta] = nbat;
    }
    return pl;
}

template <typename T>
void pack_stream(const Piece* pieces, int npieces, const long long* rec_off, const T* A, const T* W, const int* map,
                 const int* prow, int k, unsigned char* out, cudaStream_t s) {
    if (npieces == 0) return;
    k_pack<T><<<(npieces * 32 + 255) / 256, 256, 0, s>>>(pieces, npieces, rec_off, A, W, map, prow, k, out);
    VG_CUDA(cudaGetLastError());
}

void prepare_stream_kernels() {
    // one limit for every plan (stages x stage bytes never exceeds it), so handles with different
    // plans in one process do not lower each other's limit
    const int lim = MAX_RING_BYTES;
    VG_CUDA(cudaFuncSetAttribute(apply_bulk_kernel<double, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    VG_CUDA(cudaFuncSetAttribute(apply_bulk_kernel<float, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    VG_CUDA(cudaFuncSetAttribute(apply_bulk_kernel<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    VG_CUDA(cudaFuncSetAttribute(apply_bulk_kernel<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
}

template <typename T>
void launch_apply(ApplyArgs<T> a, cudaStream_t s) {
    if (a.rec && a.k <= 1) {
        if (a.ncta == 0) return;
        if (a.stages < BULK_GROUPS || a.stages % BULK_GROUPS)
            throw Error(VG_EINVAL, "apply ring: stage count not a multiple of the consumer groups");
        const size_t smem = size_t(a.stages) * a.stage_bytes;
        if (a.k == 0)
            apply_bulk_kernel<T, 0><<<a.ncta, BULK_THREADS, smem, s>>>(a);
        else
            apply_bulk_kernel<T, 1><<<a.ncta, BULK_THREADS, smem, s>>>(a);
        VG_CUDA(cudaGetLastError());
        return;
    }
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
template void pack_stream<double>(const Piece*, int, const long long*, const double*, const double*, const int*,
                                  const int*, int, unsigned char*, cudaStream_t);
template void pack_stream<float>(const Piece*, int, const long long*, const float*, const float*, const int*,
                                 const int*, int, unsigned char*, cudaStream_t);

}  // namespace vg
