// Smoothed-aggregation AMG: host setup, device V-cycle (see vg_amg.hpp).
//
// Setup (host, once per operator): strength of connection |a_ij| >= theta sqrt(a_ii a_jj);
// three-phase greedy aggregation in row order (rows are cells in Hilbert order, so aggregates are
// compact); tentative prolongator = aggregate indicator; prolongator smoothed by one damped Jacobi
// step P = (I - omega D^{-1} A) P_tent with omega = 4 / (3 rho(D^{-1} A)); Galerkin coarse operator
// R A P with R = P^T; stop at <= COARSE_MAX rows and invert the coarsest matrix densely on the
// device (one dense matrix-vector product replaces the levels below).
// Cycle (device): symmetric V(1,1) cycle with damped Jacobi (same omega) — a fixed symmetric
// positive definite operator, as MINRES requires of its preconditioner.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <numeric>

#include "vg_amg.hpp"
#include "vg_pipe.cuh"

namespace vg {

namespace {

// ---------------------------------------------------------------------------------------------
// host sparse kernels
// ---------------------------------------------------------------------------------------------
HostCsr transpose(const HostCsr& A) {
    HostCsr T;
    T.n = A.m;
    T.m = A.n;
    T.ptr.assign(T.n + 1, 0);
    for (int c : A.col) T.ptr[c + 1]++;
    for (int i = 0; i < T.n; ++i) T.ptr[i + 1] += T.ptr[i];
    T.col.resize(A.col.size());
    T.val.resize(A.val.size());
    std::vector<int> fill(T.ptr.begin(), T.ptr.end() - 1);
    for (int i = 0; i < A.n; ++i)
        for (int j = A.ptr[i]; j < A.ptr[i + 1]; ++j) {
            int d = fill[A.col[j]]++;
            T.col[d] = i;
            T.val[d] = A.val[j];
        }
    return T;
}

// transpose and, for every entry of the result, its position in A
HostCsr transpose_map(const HostCsr& A, std::vector<int>& pos) {
    HostCsr T;
    T.n = A.m;
    T.m = A.n;
    T.ptr.assign(T.n + 1, 0);
    for (int c : A.col) T.ptr[c + 1]++;
    for (int i = 0; i < T.n; ++i) T.ptr[i + 1] += T.ptr[i];
    T.col.resize(A.col.size());
    T.val.resize(A.val.size());
    pos.assign(A.col.size(), 0);
    std::vector<int> fill(T.ptr.begin(), T.ptr.end() - 1);
    for (int i = 0; i < A.n; ++i)
        for (int j = A.ptr[i]; j < A.ptr[i + 1]; ++j) {
            int d = fill[A.col[j]]++;
            T.col[d] = i;
            T.val[d] = A.val[j];
            pos[d] = j;
        }
    return T;
}

HostCsr spgemm(const HostCsr& A, const HostCsr& B) {
    HostCsr C;
    C.n = A.n;
    C.m = B.m;
    C.ptr.assign(C.n + 1, 0);
    std::vector<int> mark(B.m, -1), cols;
    std::vector<double> acc(B.m, 0.0);
    for (int i = 0; i < A.n; ++i) {
        cols.clear();
        for (int j = A.ptr[i]; j < A.ptr[i + 1]; ++j) {
            int k = A.col[j];
            double a = A.val[j];
            for (int t = B.ptr[k]; t < B.ptr[k + 1]; ++t) {
                int c = B.col[t];
                if (mark[c] != i) {
                    mark[c] = i;
                    acc[c] = 0.0;
                    cols.push_back(c);
                }
                acc[c] += a * B.val[t];
            }
        }
        std::sort(cols.begin(), cols.end());
        for (int c : cols) {
            C.col.push_back(c);
            C.val.push_back(acc[c]);
        }
        C.ptr[i + 1] = int(C.col.size());
    }
    return C;
}

// rows i -> rows[i] and columns j -> cols[j] (either may be null), columns sorted per row
HostCsr permute_csr(const HostCsr& S, const std::vector<int>* rows, const std::vector<int>* cols) {
    HostCsr T;
    T.n = S.n;
    T.m = S.m;
    T.ptr.assign(S.n + 1, 0);
    std::vector<int> old_of(S.n);
    for (int i = 0; i < S.n; ++i) old_of[rows ? (*rows)[i] : i] = i;
    std::vector<std::pair<int, double>> row;
    for (int t = 0; t < S.n; ++t) {
        const int i = old_of[t];
        row.clear();
        for (int j = S.ptr[i]; j < S.ptr[i + 1]; ++j) row.push_back({cols ? (*cols)[S.col[j]] : S.col[j], S.val[j]});
        std::sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (const auto& e : row) {
            T.col.push_back(e.first);
            T.val.push_back(e.second);
        }
        T.ptr[t + 1] = int(T.col.size());
    }
    return T;
}

double diag_of(const HostCsr& A, int i) {
    for (int j = A.ptr[i]; j < A.ptr[i + 1]; ++j)
        if (A.col[j] == i) return A.val[j];
    return 0.0;
}

// largest eigenvalue of D^{-1} A by power iteration (seeded start vector)
double rho_dinv_a(const HostCsr& A, const std::vector<double>& dinv) {
    int n = A.n;
    std::vector<double> v(n), w(n);
    unsigned s = 12345u;
    for (int i = 0; i < n; ++i) {
        s = s * 1103515245u + 12345u;
        v[i] = 0.5 + (s >> 16) / 65536.0;
    }
    double lam = 1.0;
    for (int it = 0; it < 20; ++it) {
        double nv = 0;
        for (int i = 0; i < n; ++i) {
            double a = 0;
            for (int j = A.ptr[i]; j < A.ptr[i + 1]; ++j) a += A.val[j] * v[A.col[j]];
            w[i] = dinv[i] * a;
            nv += w[i] * w[i];
        }
        nv = std::sqrt(nv);
        if (!(nv > 0)) break;
        double dv = 0;
        for (int i = 0; i < n; ++i) dv += w[i] * v[i];
        double vv = 0;
        for (int i = 0; i < n; ++i) vv += v[i] * v[i];
        lam = dv / vv;
        for (int i = 0; i < n; ++i) v[i] = w[i] / nv;
    }
    return std::max(lam, 1e-300);
}

// three-phase greedy aggregation on the strong-connection graph
std::vector<int> aggregate(const HostCsr& A, double theta, int& nagg) {
    int n = A.n;
    std::vector<double> d(n);
    for (int i = 0; i < n; ++i) d[i] = std::fabs(diag_of(A, i));
    auto strong = [&](int i, int j, double a) {
        return j != i && std::fabs(a) >= theta * std::sqrt(d[i] * d[j]);
    };
    std::vector<int> agg(n, -1);
    nagg = 0;
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        bool free = true;
        for (int j = A.ptr[i]; j < A.ptr[i + 1] && free; ++j)
            if (strong(i, A.col[j], A.val[j]) && agg[A.col[j]] >= 0) free = false;
        if (!free) continue;
        agg[i] = nagg;
        for (int j = A.ptr[i]; j < A.ptr[i + 1]; ++j)
            if (strong(i, A.col[j], A.val[j])) agg[A.col[j]] = nagg;
        ++nagg;
    }
    std::vector<int> first(agg);
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        double best = -1;
        int bj = -1;
        for (int j = A.ptr[i]; j < A.ptr[i + 1]; ++j) {
            int c = A.col[j];
            if (strong(i, c, A.val[j]) && first[c] >= 0 && std::fabs(A.val[j]) > best) {
                best = std::fabs(A.val[j]);
                bj = c;
            }
        }
        if (bj >= 0) agg[i] = first[bj];
    }
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        agg[i] = nagg;
        for (int j = A.ptr[i]; j < A.ptr[i + 1]; ++j)
            if (strong(i, A.col[j], A.val[j]) && agg[A.col[j]] < 0) agg[A.col[j]] = nagg;
        ++nagg;
    }
    return agg;
}

// P = (I - omega D^{-1} A) P_tent
HostCsr smoothed_prolongator(const HostCsr& A, const std::vector<int>& agg, int nagg, const std::vector<double>& dinv,
                             double omega) {
    HostCsr P;
    P.n = A.n;
    P.m = nagg;
    P.ptr.assign(A.n + 1, 0);
    std::vector<int> mark(nagg, -1), cols;
    std::vector<double> acc(nagg, 0.0);
    for (int i = 0; i < A.n; ++i) {
        cols.clear();
        auto add = [&](int c, double v) {
            if (mark[c] != i) {
                mark[c] = i;
                acc[c] = 0.0;
                cols.push_back(c);
            }
            acc[c] += v;
        };
        add(agg[i], 1.0);
        for (int j = A.ptr[i]; j < A.ptr[i + 1]; ++j) add(agg[A.col[j]], -omega * dinv[i] * A.val[j]);
        std::sort(cols.begin(), cols.end());
        for (int c : cols)
            if (acc[c] != 0.0) {
                P.col.push_back(c);
                P.val.push_back(acc[c]);
            }
        P.ptr[i + 1] = int(P.col.size());
    }
    return P;
}

// Pt = (I - omega D^{-1} A) P from P and the product A P: the union of their row patterns, no entry
// dropped (the pattern stays valid for the values of a refresh)
HostCsr transfer_smooth(const HostCsr& P, const HostCsr& AP, const std::vector<double>& dinv, double omega) {
    HostCsr Q;
    Q.n = P.n;
    Q.m = P.m;
    Q.ptr.assign(P.n + 1, 0);
    for (int i = 0; i < P.n; ++i) {
        const double f = omega * dinv[i];
        int a = P.ptr[i], b = AP.ptr[i];
        const int ae = P.ptr[i + 1], be = AP.ptr[i + 1];
        while (a < ae || b < be) {
            const int ca = a < ae ? P.col[a] : P.m, cb = b < be ? AP.col[b] : P.m;
            const int c = std::min(ca, cb);
            const double pv = ca == c ? P.val[a++] : 0.0;
            const double apv = cb == c ? AP.val[b++] : 0.0;
            Q.col.push_back(c);
            Q.val.push_back(pv - f * apv);
        }
        Q.ptr[i + 1] = int(Q.col.size());
    }
    return Q;
}

// dense copy of the coarsest matrix, row-major; a tiny diagonal shift keeps a semi-definite
// coarsest matrix (constants in the kernel) invertible
std::vector<double> dense_of(const HostCsr& A) {
    const int n = A.n;
    std::vector<double> a(size_t(n) * n, 0.0);
    double tr = 0;
    for (int i = 0; i < n; ++i)
        for (int j = A.ptr[i]; j < A.ptr[i + 1]; ++j) {
            a[size_t(i) * n + A.col[j]] += A.val[j];
            if (A.col[j] == i) tr += A.val[j];
        }
    for (int i = 0; i < n; ++i) a[size_t(i) * n + i] += 1e-12 * tr / n;
    return a;
}

// ---------------------------------------------------------------------------------------------
// device kernels (SELL-32, one thread per row)
// ---------------------------------------------------------------------------------------------
constexpr int TPB = 256;
constexpr int CSR_CAP = 2048;  // entries staged per CSR row block
constexpr int CSR_RPT = 4;     // rows per thread of a CSR row block (at most CSR_RPT * TPB rows)

// the first SELL_PRE entries of a row (columns and values) loaded before the programmatic-launch
// wait: the matrix is written only at set-up and refresh, never by a kernel of the cycle
constexpr int SELL_PRE = 8;
template <typename T>
struct SellRow {
    int c[SELL_PRE];
    T v[SELL_PRE];
    int w = 0;
    long long o = 0;
};

template <typename T>
__device__ __forceinline__ void sell_fetch(const DevSell<T>& M, int r, SellRow<T>& R) {
    const int s = r >> 5, l = r & 31;
    R.o = __ldg(M.soff + s) + l;
    R.w = __ldg(M.width + s);
#pragma unroll
    for (int k = 0; k < SELL_PRE; ++k) {
        R.c[k] = k < R.w ? __ldg(M.col + R.o + 32 * k) : 0;
        R.v[k] = k < R.w ? __ldg(M.val + R.o + 32 * k) : T(0);
    }
}

// sum_k val_k x(col_k) in entry order (fixed summation order)
template <typename T>
__device__ __forceinline__ T sell_finish(const DevSell<T>& M, const SellRow<T>& R, const T* x) {
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < SELL_PRE; ++k)
        if (k < R.w) acc += R.v[k] * x[R.c[k]];
    for (int k = SELL_PRE; k < R.w; ++k) acc += __ldg(M.val + R.o + 32 * k) * x[__ldg(M.col + R.o + 32 * k)];
    return acc;
}

// residual of one Jacobi step from zero, r = b - (A S) b, on the SELL-32 finest level (the stored
// values are those of A S, so only b is gathered), written as the prolongation's term
// q = S (b + r). b is written by an earlier kernel: read with plain loads after the
// programmatic-launch wait (never ld.global.nc, which the compiler may move above it)
template <typename T>
__global__ void __launch_bounds__(TPB) k_sell_residual(DevSell<T> A, const T* dinv, T omega, const T* b, T* q) {
    pdl_trigger();
    const int i = blockIdx.x * TPB + threadIdx.x;
    SellRow<T> R;
    if (i < A.n) sell_fetch<T>(A, i, R);
    const T di = i < A.n ? __ldg(dinv + i) : T(0);
    pdl_wait();
    if (i < A.n) {
        const T bi = b[i], ri = bi - sell_finish<T>(A, R, b);
        q[i] = omega * di * (bi + ri);
    }
}

// ---- CSR in row blocks (the CSR-stream scheme of Greathouse and Daga, SC 2014, with the entries
// staged by bulk copies): row block b covers rows [rb[b].x, rb[b + 1].x) (at most CSR_RPT * TPB)
// and entries [rb[b].y, rb[b + 1].y) (at most CSR_CAP unless one row alone is longer). A CTA walks
// row blocks b = blockIdx.x, + gridDim.x, ... through a two-stage ring: the column indices and
// values of the next row block are copied into shared memory (cp.async.bulk on an mbarrier, 16-byte
// aligned supersets of the ranges) while the current one gathers x and sums; one thread per row
// sums its products in order (or, for long rows, 8 threads per row in a fixed strided order and
// shuffle tree), so the result does not depend on the launch shape. Vectors written
// by earlier kernels of the cycle are read with plain loads after the programmatic-launch wait
// (never ld.global.nc, which the compiler may move above it); the matrix may be read before it.
// op: 0 y = M x (restriction); 1 y = r + M x (prolongation, r holding S (b + residual) of the
//     composite cycle); 2 y = omega dinv (b + (b - M x)) (that smoothed residual term, with x = b
//     and M = A S)
template <typename T>
struct CsrSmem {
    static constexpr int col_bytes = (CSR_CAP + 8) * 4;
    static constexpr int val_bytes = (CSR_CAP + 8) * int(sizeof(T));
    static constexpr int stage_bytes = col_bytes + val_bytes;
    static constexpr int prod_off = 2 * stage_bytes;
    static constexpr int total = prod_off + CSR_CAP * int(sizeof(T));
    static_assert(col_bytes % 16 == 0 && val_bytes % 16 == 0, "16-byte stage layout");
};

template <int OP, typename T, int LPR>
__global__ void __launch_bounds__(TPB) k_csr(DevCsr<T> M, const T* dinv, T omega, const T* b, const T* x, T* y,
                                             const T* r) {
    // LPR threads per row: 1 (each thread sums up to CSR_RPT rows) or 8 for long rows (a row's
    // products summed by 8 threads, strided, then a fixed shuffle tree; at most TPB / 8 rows)
    constexpr int RQ = LPR == 1 ? CSR_RPT : 1;
    using L = CsrSmem<T>;
    constexpr int J = CSR_CAP / TPB;
    constexpr int VA = 16 / int(sizeof(T));  // values per 16 bytes
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) unsigned long long full[2];
    __shared__ T red[TPB / 32];
    T* prod = reinterpret_cast<T*>(sm + L::prod_off);
    const int t = threadIdx.x, G = gridDim.x, nblk = M.nblk;
    // copy row block blk into stage s (thread 0); empty and long-row blocks are not staged
    auto issue = [&](int blk, int s) {
        const int2 a = __ldg(M.rb + blk), z = __ldg(M.rb + blk + 1);
        const int ne = z.y - a.y;
        if (ne <= 0 || ne > CSR_CAP) return;
        const int c0 = a.y & ~3, c1 = (z.y + 3) & ~3, v0 = a.y & ~(VA - 1), v1 = (z.y + VA - 1) & ~(VA - 1);
        unsigned char* st = sm + s * L::stage_bytes;
        mbar_expect_tx(&full[s], unsigned((c1 - c0) * 4 + (v1 - v0) * int(sizeof(T))));
        bulk_g2s(st, M.col + c0, unsigned((c1 - c0) * 4), &full[s]);
        bulk_g2s(st + L::col_bytes, M.val + v0, unsigned((v1 - v0) * int(sizeof(T))), &full[s]);
    };
    pdl_trigger();
    if (t == 0) {  // the matrix does not depend on earlier kernels: its first two row blocks are copied before the wait
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
        if (blockIdx.x < nblk) issue(blockIdx.x, 0);
        if (blockIdx.x + G < nblk) issue(blockIdx.x + G, 1);
    }
    __syncthreads();
    pdl_wait();
    unsigned par0 = 0u, par1 = 0u;  // phase parity of each stage's barrier
    for (int i = 0, blk = blockIdx.x; blk < nblk; ++i, blk += G) {
        const int s = i & 1;
        const int2 a = __ldg(M.rb + blk), z = __ldg(M.rb + blk + 1);
        const int ne = z.y - a.y;
        const bool staged = ne > 0 && ne <= CSR_CAP;
        int lo[RQ], hi[RQ];
        T ep[RQ], dd[RQ];  // the epilogue's vector operands, loaded before the gathers (independent of them)
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
            const int row = LPR == 1 ? a.x + t + q * TPB : a.x + t / LPR;
            lo[q] = hi[q] = 0;
            ep[q] = dd[q] = T(0);
            if (row < z.x) {
                lo[q] = __ldg(M.ptr + row) - a.y;
                hi[q] = __ldg(M.ptr + row + 1) - a.y;
                if (OP == 1)
                    ep[q] = r[row];
                else if (OP == 2) {
                    ep[q] = b[row];
                    dd[q] = __ldg(dinv + row);
                }
            }
        }
        int c[J];
        T v[J];
        if (staged) {
            const bool ok = mbar_wait(&full[s], s ? par1 : par0, nullptr);
            if (s)
                par1 ^= 1u;
            else
                par0 ^= 1u;
            if (__syncthreads_or(!ok)) {  // a copy that never landed: flag it and stop (never in a correct run)
                if (t == 0) {
                    atomicExch(M.err, 1);
                    if (blk + G < nblk) mbar_wait(&full[s ^ 1], s ? par0 : par1, nullptr);
                }
                return;
            }
            const int* scol = reinterpret_cast<const int*>(sm + s * L::stage_bytes) + (a.y & 3);
            const T* sval = reinterpret_cast<const T*>(sm + s * L::stage_bytes + L::col_bytes) + (a.y & (VA - 1));
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int k = t + j * TPB;
                c[j] = k < ne ? scol[k] : 0;
                v[j] = k < ne ? sval[k] : T(0);
            }
        }
        __syncthreads();  // stage s consumed: refill it with the row block two steps ahead
        if (t == 0 && blk + 2 * G < nblk) {
            fence_proxy_async_smem();
            issue(blk + 2 * G, s);
        }
        T acc[RQ];
#pragma unroll
        for (int q = 0; q < RQ; ++q) acc[q] = T(0);
        if (staged) {
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int k = t + j * TPB;
                if (k < ne) prod[k] = v[j] * x[c[j]];
            }
            __syncthreads();
            if (LPR == 1) {
#pragma unroll
                for (int q = 0; q < RQ; ++q)
                    for (int k = lo[q]; k < hi[q]; ++k) acc[q] += prod[k];
            } else {
                for (int k = lo[0] + t % LPR; k < hi[0]; k += LPR) acc[0] += prod[k];
#pragma unroll
                for (int off = LPR / 2; off; off >>= 1) acc[0] += __shfl_down_sync(0xffffffffu, acc[0], off, LPR);
            }
            __syncthreads();  // prod is rewritten by the next row block
        } else if (ne > CSR_CAP) {  // one long row: strided partial sums, fixed-order block reduction
            T part = T(0);
            for (int k = t; k < ne; k += TPB)
                part += __ldg(M.val + a.y + k) * x[__ldg(M.col + a.y + k)];
            for (int off = 16; off; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
            if ((t & 31) == 0) red[t >> 5] = part;
            __syncthreads();
            if (t == 0) {
                T sum = T(0);
                for (int w = 0; w < TPB / 32; ++w) sum += red[w];
                acc[0] = sum;
            }
            __syncthreads();
        }
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
            const int row = LPR == 1 ? a.x + t + q * TPB : a.x + t / LPR;
            if (row >= z.x || (LPR > 1 && t % LPR != 0)) continue;
            if (OP == 0)
                y[row] = acc[q];
            else if (OP == 1)
                y[row] = ep[q] + acc[q];
            else {
                const T rr = ep[q] - acc[q];
                y[row] = omega * dd[q] * (ep[q] + rr);
            }
        }
    }
}

// ---- CSR in warp blocks: a warp takes up to 32 / LPR consecutive rows holding at most WS_CAP
// entries. Lane l loads the block's entries l, l + 32, ... (coalesced) into registers before the
// programmatic-launch wait (the matrix is never written by the cycle), gathers x after it and
// stores the products in the warp's slice of shared memory; the LPR lanes of a row then sum its
// products (LPR = 1: in order; LPR = 8 for long rows: strided, then a fixed shuffle tree), so the
// result is deterministic. A row longer than WS_CAP is a block of its own, summed by the whole
// warp from global memory (strided partial sums, fixed shuffle tree). Same ops as k_csr.
constexpr int WS_CAP = 128, WS_J = WS_CAP / 32, WS_WARPS = 8;
template <int OP, typename T, int LPR>
__global__ void __launch_bounds__(WS_WARPS * 32) k_csr_ws(DevCsr<T> M, const T* dinv, T omega, const T* b,
                                                          const T* x, T* y, const T* r) {
    __shared__ T prod[WS_WARPS][WS_CAP];
    pdl_trigger();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, blk = blockIdx.x * WS_WARPS + w;
    const int rl_i = lane / LPR, sub = lane % LPR;  // LPR lanes per row (at most 32 / LPR rows)
    const bool live = blk < M.nwb;
    int2 a = make_int2(0, 0), z = make_int2(0, 0);
    if (live) {
        a = __ldg(M.wb + blk);
        z = __ldg(M.wb + blk + 1);
    }
    const int ne = z.y - a.y, row = a.x + rl_i;
    const bool rl = row < z.x;
    const bool staged = ne <= WS_CAP;
    int lo = 0, hi = 0;
    if (rl) {
        lo = __ldg(M.ptr + row) - a.y;
        hi = __ldg(M.ptr + row + 1) - a.y;
    }
    int c[WS_J];
    T v[WS_J];
#pragma unroll
    for (int j = 0; j < WS_J; ++j) {
        const int k = lane + 32 * j;
        const bool in = staged && k < ne;
        c[j] = in ? __ldg(M.col + a.y + k) : 0;
        v[j] = in ? __ldg(M.val + a.y + k) : T(0);
    }
    const T dl = (OP == 2 && rl) ? __ldg(dinv + row) : T(0);
    pdl_wait();
    if (!live) return;
    T ep = T(0);
    if (rl) {
        if (OP == 1)
            ep = r[row];
        else if (OP == 2)
            ep = b[row];
    }
    T acc = T(0);
    if (staged) {
#pragma unroll
        for (int j = 0; j < WS_J; ++j) {
            const int k = lane + 32 * j;
            if (k < ne) prod[w][k] = v[j] * x[c[j]];
        }
        __syncwarp();
        if (LPR == 1) {
            if (rl)
                for (int k = lo; k < hi; ++k) acc += prod[w][k];
        } else {
            if (rl)
                for (int k = lo + sub; k < hi; k += LPR) acc += prod[w][k];
#pragma unroll
            for (int off = LPR / 2; off; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off, LPR);
        }
    } else {
        for (int k = lane; k < ne; k += 32) acc += __ldg(M.val + a.y + k) * x[__ldg(M.col + a.y + k)];
        for (int off = 16; off; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    }
    if (rl && (staged ? sub == 0 : lane == 0)) {
        if (OP == 0)
            y[row] = acc;
        else if (OP == 1)
            y[row] = ep + acc;
        else {
            const T rr = ep - acc;
            y[row] = omega * dl * (ep + rr);
        }
    }
}


template <int OP, typename T, int LPR>
void prepare_csr_op1() {
    VG_CUDA(cudaFuncSetAttribute(k_csr<OP, T, LPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, CsrSmem<T>::total));
    // the whole unified L1/shared array as shared memory: the occupancy the grid is sized for
    VG_CUDA(cudaFuncSetAttribute(k_csr<OP, T, LPR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 int(cudaSharedmemCarveoutMaxShared)));
}
template <int OP, typename T>
void prepare_csr_op() {
    prepare_csr_op1<OP, T, 1>();
    prepare_csr_op1<OP, T, 8>();
}

// kernel attributes on the current device (function attributes are per device) and the number of
// CTAs of each precision's CSR kernel the device holds at once: slots[0] FP32, slots[1] FP64
void prepare_csr_kernels(int slots[2]) {
    prepare_csr_op<0, float>();
    prepare_csr_op<1, float>();
    prepare_csr_op<2, float>();
    prepare_csr_op<0, double>();
    prepare_csr_op<1, double>();
    prepare_csr_op<2, double>();
    int dev = 0, n32 = 0, n64 = 0, sms = 0;
    VG_CUDA(cudaGetDevice(&dev));
    VG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    VG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n32, k_csr<0, float, 1>, TPB, CsrSmem<float>::total));
    VG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n64, k_csr<0, double, 1>, TPB, CsrSmem<double>::total));
    slots[0] = std::max(1, n32) * std::max(1, sms);
    slots[1] = std::max(1, n64) * std::max(1, sms);
}

template <typename T>
void launch_csr(int op, const DevCsr<T>& M, const T* dinv, T omega, const T* b, const T* x, T* y, const T* r,
                cudaStream_t s) {
    if (M.n <= 0 || M.nblk <= 0) return;
    const int grid = std::min(M.nblk, std::max(1, M.slots));
    const int sb = CsrSmem<T>::total;
    switch (op) {
    case 0:
        if (M.lpr > 1)
            launch_pdl(k_csr<0, T, 8>, grid, TPB, sb, s, M, dinv, omega, b, x, y, r);
        else
            launch_pdl(k_csr<0, T, 1>, grid, TPB, sb, s, M, dinv, omega, b, x, y, r);
        break;
    case 1:
        if (M.lpr > 1)
            launch_pdl(k_csr<1, T, 8>, grid, TPB, sb, s, M, dinv, omega, b, x, y, r);
        else
            launch_pdl(k_csr<1, T, 1>, grid, TPB, sb, s, M, dinv, omega, b, x, y, r);
        break;
    default:
        if (M.lpr > 1)
            launch_pdl(k_csr<2, T, 8>, grid, TPB, sb, s, M, dinv, omega, b, x, y, r);
        else
            launch_pdl(k_csr<2, T, 1>, grid, TPB, sb, s, M, dinv, omega, b, x, y, r);
        break;
    }
}

template <typename T>
void launch_ws(int op, const DevCsr<T>& M, const T* dinv, T omega, const T* b, const T* x, T* y, const T* r,
               cudaStream_t s) {
    if (M.n <= 0 || M.nwb <= 0) return;
    const int grid = (M.nwb + WS_WARPS - 1) / WS_WARPS;
    switch (op) {
    case 0:
        if (M.lpr > 1)
            launch_pdl(k_csr_ws<0, T, 8>, grid, WS_WARPS * 32, 0, s, M, dinv, omega, b, x, y, r);
        else
            launch_pdl(k_csr_ws<0, T, 1>, grid, WS_WARPS * 32, 0, s, M, dinv, omega, b, x, y, r);
        break;
    case 1:
        if (M.lpr > 1)
            launch_pdl(k_csr_ws<1, T, 8>, grid, WS_WARPS * 32, 0, s, M, dinv, omega, b, x, y, r);
        else
            launch_pdl(k_csr_ws<1, T, 1>, grid, WS_WARPS * 32, 0, s, M, dinv, omega, b, x, y, r);
        break;
    default:
        if (M.lpr > 1)
            launch_pdl(k_csr_ws<2, T, 8>, grid, WS_WARPS * 32, 0, s, M, dinv, omega, b, x, y, r);
        else
            launch_pdl(k_csr_ws<2, T, 1>, grid, WS_WARPS * 32, 0, s, M, dinv, omega, b, x, y, r);
        break;
    }
}

// the CSR product of the cycle in each precision's faster form (1M cells, A/B of builds): FP64 in
// warp blocks (FP64 solve 22.3 -> 21.5 ms; the row-block kernel holds 3 CTAs per SM in FP64), FP32
// in row blocks (warp blocks 14.34 -> 14.46 ms). Matrices of 16 or more entries per row (the
// restrictions, the denser coarse operators) are summed by 8 threads per row in both kernels
// (mixed 14.31 -> 14.13 ms, FP64 21.49 -> 21.14 ms)
template <typename T>
void launch_prod(int op, const DevCsr<T>& M, const T* dinv, T omega, const T* b, const T* x, T* y, const T* r,
                 cudaStream_t s) {
    if constexpr (sizeof(T) == 8)
        launch_ws<T>(op, M, dinv, omega, b, x, y, r, s);
    else
        launch_csr<T>(op, M, dinv, omega, b, x, y, r, s);
}

// coarsest level: z = Ainv b, one warp per row. The inverse does not change between cycles: its
// rows are loaded with an L2 evict-last hint, so that they stay resident in L2 while the operator
// records stream through with evict-first, and each warp loads its row into registers before the
// programmatic-launch wait (while the restriction before it still runs). After the wait only b is
// read. Lane l sums the entries l, l + 32, ... in order, then a fixed shuffle tree: deterministic.
constexpr int DENSE_WARPS = 4;  // rows per block
template <typename T>
struct DensePre {
    static constexpr int value = sizeof(T) == 4 ? 72 : 36;  // entries per lane held in registers
};

template <typename T>
__device__ __forceinline__ T ld_keep(const T* p, unsigned long long pol);
template <>
__device__ __forceinline__ float ld_keep<float>(const float* p, unsigned long long pol) {
    float v;
    asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
template <>
__device__ __forceinline__ double ld_keep<double>(const double* p, unsigned long long pol) {
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}

template <typename T>
__global__ void __launch_bounds__(DENSE_WARPS * 32) k_dense(int n, const T* Ainv, const T* b, T* z) {
    pdl_trigger();
    constexpr int PRE = DensePre<T>::value;
    const int lane = threadIdx.x & 31, row = blockIdx.x * DENSE_WARPS + (threadIdx.x >> 5);
    const bool live = row < n;
    const T* a = Ainv + (long long)(live ? row : 0) * n;
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    T av[PRE];
#pragma unroll
    for (int q = 0; q < PRE; ++q) {
        const int j = lane + 32 * q;
        av[q] = (live && j < n) ? ld_keep(a + j, pol) : T(0);
    }
    pdl_wait();
    if (!live) return;
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < PRE; ++q) {
        const int j = lane + 32 * q;
        if (j < n) acc += av[q] * b[j];
    }
    for (int j = lane + 32 * PRE; j < n; j += 32) acc += ld_keep(a + j, pol) * b[j];
    for (int off = 16; off; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) z[row] = acc;
}

// ---- dense inverse of the (symmetric positive definite) coarsest matrix on the device: in-place
// Gauss-Jordan without pivoting, one step per pivot k:
//   a_kk <- 1/p, a_kj <- a_kj/p, a_ik <- -a_ik/p, a_ij <- a_ij - a_ik a_kj / p   (p = a_kk)
// with column k and row k saved before the step, so every element reads only its own old value
__global__ void k_gj_save(const double* a, int n, int k, double* col, double* row) {
    int t = blockIdx.x * TPB + threadIdx.x;
    if (t < n) {
        col[t] = a[(long long)t * n + k];
        row[t] = a[(long long)k * n + t];
    }
}

__global__ void k_gj_step(double* a, int n, int k, const double* col, const double* row, unsigned long long* bad,
                          double* ncol, double* nrow) {
    long long t = blockIdx.x * (long long)TPB + threadIdx.x;
    if (t >= (long long)n * n) return;
    const int i = int(t / n), j = int(t % n);
    const double p = row[k];
    if (!(p > 0.0)) {  // not positive definite: reported, the result is not used
        if (t == 0) atomicExch(bad, 1ull);
        return;
    }
    double v;
    if (i == k && j == k)
        v = 1.0 / p;
    else if (i == k)
        v = row[j] / p;
    else if (j == k)
        v = -col[i] / p;
    else
        v = a[t] - col[i] * row[j] / p;
    a[t] = v;
    // the next step's saved column and row (ping-pong buffers): no separate save launch
    if (ncol) {
        if (j == k + 1) ncol[i] = v;
        if (i == k + 1) nrow[j] = v;
    }
}

// symmetric part in FP64 and FP32 (the exact inverse is symmetric)
__global__ void k_gj_sym(const double* a, int n, double* o64, float* o32) {
    long long t = blockIdx.x * (long long)TPB + threadIdx.x;
    if (t >= (long long)n * n) return;
    const int i = int(t / n), j = int(t % n);
    const double v = 0.5 * (a[t] + a[(long long)j * n + i]);
    o64[t] = v;
    o32[t] = float(v);
}

// ---- numeric refresh of a hierarchy with fixed structure (one thread per row, fixed order) -------
__device__ __forceinline__ int find_col(const int* col, int lo, int hi, int c) {
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (col[mid] < c)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;  // position of c when present
}

__global__ void k_diag_inv(const int* ptr, const int* col, const double* val, int n, double* d64, float* d32) {
    int r = blockIdx.x * TPB + threadIdx.x;
    if (r >= n) return;
    int lo = ptr[r], hi = ptr[r + 1];
    int j = find_col(col, lo, hi, r);
    double v = (j < hi && col[j] == r) ? val[j] : 0.0;
    double iv = v != 0.0 ? 1.0 / v : 0.0;
    d64[r] = iv;
    d32[r] = float(iv);
}

// P = (I - omega D^{-1} A) P_tent on the fixed pattern of P (rows in A's stored order)
__global__ void k_smooth_p(const int* aptr, const int* acol, const double* aval, const int* agg, const double* dinv,
                           double omega, const int* pptr, const int* pcol, double* pval, int n) {
    int t = blockIdx.x * TPB + threadIdx.x;
    if (t >= n) return;
    const int lo = pptr[t], hi = pptr[t + 1];
    for (int j = lo; j < hi; ++j) pval[j] = 0.0;
    int j = find_col(pcol, lo, hi, agg[t]);
    if (j < hi && pcol[j] == agg[t]) pval[j] += 1.0;
    const double f = -omega * dinv[t];
    for (int e = aptr[t]; e < aptr[t + 1]; ++e) {
        const int J = agg[acol[e]];
        j = find_col(pcol, lo, hi, J);
        if (j < hi && pcol[j] == J) pval[j] += f * aval[e];
    }
}

__global__ void k_take(const double* src, const int* map, double* dst, long long n) {
    for (long long i = blockIdx.x * (long long)TPB + threadIdx.x; i < n; i += (long long)gridDim.x * TPB)
        dst[i] = src[map[i]];
}

// C = R A P on C's fixed pattern, one coarse row per thread
__global__ void k_rap(const int* rptr, const int* rcol, const double* rval, const int* aptr, const int* acol,
                      const double* aval, const int* pptr, const int* pcol, const double* pval, const int* cptr,
                      const int* ccol, double* cval, int nc) {
    int I = blockIdx.x * TPB + threadIdx.x;
    if (I >= nc) return;
    const int lo = cptr[I], hi = cptr[I + 1];
    for (int j = lo; j < hi; ++j) cval[j] = 0.0;
    for (int u = rptr[I]; u < rptr[I + 1]; ++u) {
        const int t = rcol[u];
        const double rv = rval[u];
        for (int e = aptr[t]; e < aptr[t + 1]; ++e) {
            const int k = acol[e];
            const double ra = rv * aval[e];
            for (int w = pptr[k]; w < pptr[k + 1]; ++w) {
                const int J = pcol[w];
                const int j = find_col(ccol, lo, hi, J);
                if (j < hi && ccol[j] == J) cval[j] += ra * pval[w];
            }
        }
    }
}

// Pt = (I - omega D^{-1} A) P on Pt's fixed pattern, one row per thread: the products A P of the row
// summed in the order of the host set-up (A's entries, then P's), then Pt = P - omega d_i (A P)
__global__ void k_ptilde(const int* aptr, const int* acol, const double* aval, const double* dinv, double omega,
                         const int* pptr, const int* pcol, const double* pval, const int* qptr, const int* qcol,
                         double* qval, int n) {
    int t = blockIdx.x * TPB + threadIdx.x;
    if (t >= n) return;
    const int lo = qptr[t], hi = qptr[t + 1];
    for (int j = lo; j < hi; ++j) qval[j] = 0.0;
    for (int e = aptr[t]; e < aptr[t + 1]; ++e) {
        const int k = acol[e];
        const double a = aval[e];
        for (int w = pptr[k]; w < pptr[k + 1]; ++w) {
            const int j = find_col(qcol, lo, hi, pcol[w]);
            if (j < hi && qcol[j] == pcol[w]) qval[j] += a * pval[w];
        }
    }
    const double f = omega * dinv[t];
    int w = pptr[t];
    for (int j = lo; j < hi; ++j) {
        while (w < pptr[t + 1] && pcol[w] < qcol[j]) ++w;
        const double pv = (w < pptr[t + 1] && pcol[w] == qcol[j]) ? pval[w] : 0.0;
        qval[j] = pv - f * qval[j];
    }
}

// values of A S (columns scaled by omega D^{-1}) from A's stored CSR values, into CSR (pos null)
// or SELL slots
__global__ void k_scale_cols(const double* aval, const int* acol, const double* dinv, double omega,
                             const long long* pos, double* out, long long n) {
    for (long long i = blockIdx.x * (long long)TPB + threadIdx.x; i < n; i += (long long)gridDim.x * TPB) {
        const double v = aval[i] * (omega * dinv[acol[i]]);
        out[pos ? pos[i] : i] = v;
    }
}

__global__ void k_to32(const double* a, float* b, long long n) {
    for (long long i = blockIdx.x * (long long)TPB + threadIdx.x; i < n; i += (long long)gridDim.x * TPB)
        b[i] = float(a[i]);
}

// dense copy of a CSR matrix with the tiny diagonal shift of dense_of (one block)
__global__ void k_csr_dense(const int* ptr, const int* col, const double* val, int n, double* d) {
    __shared__ double tr[TPB];
    double t = 0;
    for (int r = threadIdx.x; r < n; r += TPB)
        for (int j = ptr[r]; j < ptr[r + 1]; ++j) {
            d[(long long)r * n + col[j]] += val[j];
            if (col[j] == r) t += val[j];
        }
    tr[threadIdx.x] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int i = 0; i < TPB; ++i) s += tr[i];
        tr[0] = s;
    }
    __syncthreads();
    const double shift = 1e-12 * tr[0] / n;
    for (int r = threadIdx.x; r < n; r += TPB) d[(long long)r * n + r] += shift;
}

inline int blocks(int n) { return (n + TPB - 1) / TPB; }

}  // namespace

void Amg::dense_inverse_device(const std::vector<double>& a, int n) {
    DevBuf<double> d;
    d.upload(a);
    dense_inverse_of(d.data(), n);
}

void Amg::dense_inverse_of(double* dd, int n) {
    DevBuf<double> col(n), row(n);
    DevBuf<unsigned long long> bad(1);
    struct {
        double* p;
        double* data() { return p; }
    } d{dd};
    bad.zero();
    const long long nn = (long long)n * n;
    const int nb = int((nn + TPB - 1) / TPB);
    DevBuf<double> col2(n), row2(n);
    double *c0 = col.data(), *r0 = row.data(), *c1 = col2.data(), *r1 = row2.data();
    k_gj_save<<<blocks(n), TPB>>>(d.data(), n, 0, c0, r0);
    for (int k = 0; k < n; ++k) {
        const bool more = k + 1 < n;
        k_gj_step<<<nb, TPB>>>(d.data(), n, k, c0, r0, bad.data(), more ? c1 : nullptr, more ? r1 : nullptr);
        std::swap(c0, c1);
        std::swap(r0, r1);
    }
    dinvc64_.resize(size_t(nn));
    dinvc32_.resize(size_t(nn));
    k_gj_sym<<<nb, TPB>>>(d.data(), n, dinvc64_.data(), dinvc32_.data());
    VG_CUDA(cudaGetLastError());
    unsigned long long b = 0;
    VG_CUDA(cudaMemcpy(&b, bad.data(), sizeof(b), cudaMemcpyDeviceToHost));
    if (b) throw Error(VG_ESINGULAR, "coarsest multigrid matrix is not positive definite");
}

Amg::~Amg() { release_streams(); }

void Amg::release_streams() {
    for (cudaEvent_t e : ev_fork_) cudaEventDestroy(e);
    for (cudaEvent_t e : ev_join_) cudaEventDestroy(e);
    ev_fork_.clear();
    ev_join_.clear();
    if (side_) cudaStreamDestroy(side_);
    side_ = nullptr;
}

void Amg::refresh(const double* a0) {
    if (levels_.empty()) throw Error(VG_ESTATE, "multigrid refresh before setup");
    PhaseTimer pt;
    const int nl = int(levels_.size());
    const double* aval = a0;
    for (int l = 0; l < nl; ++l) {
        Level& L = levels_[l];
        const long long nnz = (long long)L.pa_col.size();
        k_diag_inv<<<blocks(L.n), TPB>>>(L.dpa_ptr.data(), L.dpa_col.data(), aval, L.n, L.dinv64.data(),
                                         L.dinv32.data());
        VG_CUDA(cudaGetLastError());
        if (l == nl - 1) {  // coarsest: dense inverse of the refreshed matrix
            DevBuf<double> d(size_t(L.n) * L.n);
            d.zero();
            k_csr_dense<<<1, TPB>>>(L.dpa_ptr.data(), L.dpa_col.data(), aval, L.n, d.data());
            VG_CUDA(cudaGetLastError());
            VG_CUDA(cudaDeviceSynchronize());
            pt.mark("refresh: levels");
            dense_inverse_of(d.data(), L.n);
            pt.mark("refresh: coarsest inverse");
            break;
        }
        // A S for the residual
        if (L.A.csr) {
            k_scale_cols<<<148 * 4, TPB>>>(aval, L.dpa_col.data(), L.dinv64.data(), L.omega, nullptr, L.cA.v64.data(),
                                           nnz);
            k_to32<<<148 * 4, TPB>>>(L.cA.v64.data(), L.cA.v32.data(), nnz);
        } else {
            k_scale_cols<<<148 * 4, TPB>>>(aval, L.dpa_col.data(), L.dinv64.data(), L.omega, L.dsellpos.data(),
                                           L.dA_v64.data(), nnz);
            k_to32<<<148 * 4, TPB>>>(L.dA_v64.data(), L.dA_v32.data(), (long long)L.dA_v64.size());
        }
        // P, R = P^T (FP64: the next level's Galerkin product), Pt = (I - S A) P and Rt = Pt^T
        if (!L.fixedP)
            k_smooth_p<<<blocks(L.n), TPB>>>(L.dpa_ptr.data(), L.dpa_col.data(), aval, L.dagg.data(), L.dinv64.data(),
                                             L.omega, L.cP.ptr.data(), L.cP.col.data(), L.cP.v64.data(), L.n);
        k_take<<<148 * 4, TPB>>>(L.cP.v64.data(), L.dr2p.data(), L.cR.v64.data(), (long long)L.r2p.size());
        k_ptilde<<<blocks(L.n), TPB>>>(L.dpa_ptr.data(), L.dpa_col.data(), aval, L.dinv64.data(), L.omega,
                                       L.cP.ptr.data(), L.cP.col.data(), L.cP.v64.data(), L.cPt.ptr.data(),
                                       L.cPt.col.data(), L.cPt.v64.data(), L.n);
        const long long ptn = (long long)L.rt2pt.size();
        k_take<<<148 * 4, TPB>>>(L.cPt.v64.data(), L.drt2pt.data(), L.cRt.v64.data(), ptn);
        k_to32<<<148 * 4, TPB>>>(L.cPt.v64.data(), L.cPt.v32.data(), ptn);
        k_to32<<<148 * 4, TPB>>>(L.cRt.v64.data(), L.cRt.v32.data(), ptn);
        Level& C = levels_[l + 1];
        k_rap<<<blocks(L.nc), TPB>>>(L.cR.ptr.data(), L.cR.col.data(), L.cR.v64.data(), L.dpa_ptr.data(),
                                      L.dpa_col.data(), aval, L.cP.ptr.data(), L.cP.col.data(), L.cP.v64.data(),
                                      C.dpa_ptr.data(), C.dpa_col.data(), C.dvals.data(), L.nc);
        VG_CUDA(cudaGetLastError());
        aval = C.dvals.data();
    }
    VG_CUDA(cudaDeviceSynchronize());
}

long long Amg::nnz() const {
    long long t = 0;
    for (const auto& L : levels_) t += (long long)L.pa_col.size();
    return t;
}

void Amg::setup(const HostCsr& S0, const HostCsr* first_P, const std::vector<int>* fine_order) {
    PhaseTimer pt;
    levels_.clear();
    release_streams();
    HostCsr A = S0;
    const double theta = 0.08;
    // storage: SELL-32 (one thread per row) only for the regular fine-level operator; every other
    // matrix (rectangular transfers, the denser coarse operators) as CSR in row blocks (k_csr)
    auto to_sell = [&](const HostCsr& M, Sell& S, bool sell_ok) {
        S.n = M.n;
        double avg = M.n ? double(M.col.size()) / M.n : 0.0;
        if (!(sell_ok && avg <= 10.0)) {
            S.csr = true;
            S.cptr = M.ptr;
            S.ccol = M.col;
            S.cval = M.val;
            S.nslices = 0;
            // row blocks: at most CSR_RPT * TPB rows and about nnz / (4 blocks per SM) entries,
            // between 256 and CSR_CAP (a longer single row is a block of its own)
            const long long nnz = (long long)M.col.size();
            const int cap = int(std::min<long long>(CSR_CAP, std::max<long long>(256, (nnz + 591) / 592)));
            S.lpr = avg >= 16.0 ? 8 : 1;
            const int max_rows = S.lpr == 1 ? CSR_RPT * TPB : TPB / S.lpr;
            S.rb.assign({0, 0});
            for (int r = 0; r < M.n;) {
                const int start = r;
                long long nn = 0;
                while (r < M.n && r - start < max_rows) {
                    const int len = M.ptr[r + 1] - M.ptr[r];
                    if (r > start && nn + len > cap) break;
                    nn += len;
                    ++r;
                }
                S.rb.push_back(r);
                S.rb.push_back(M.ptr[r]);
            }
            S.wb.assign({0, 0});
            for (int r = 0; r < M.n;) {
                const int start = r;
                long long nn = 0;
                while (r < M.n && r - start < 32 / S.lpr) {
                    const int len = M.ptr[r + 1] - M.ptr[r];
                    if (r > start && nn + len > WS_CAP) break;
                    nn += len;
                    ++r;
                }
                S.wb.push_back(r);
                S.wb.push_back(M.ptr[r]);
            }
            return;
        }
        S.nslices = (M.n + 31) / 32;
        S.soff.assign(S.nslices + 1, 0);
        S.width.assign(S.nslices, 0);
        for (int s = 0; s < S.nslices; ++s) {
            int w = 0;
            for (int r = s * 32; r < std::min(M.n, s * 32 + 32); ++r) w = std::max(w, M.ptr[r + 1] - M.ptr[r]);
            S.width[s] = w;
            S.soff[s + 1] = S.soff[s] + 32LL * w;
        }
        S.col.assign(S.soff[S.nslices], 0);
        S.val.assign(S.soff[S.nslices], 0.0);
        for (int s = 0; s < S.nslices; ++s)
            for (int l = 0; l < 32; ++l) {
                int r = s * 32 + l;
                for (int k = 0; k < S.width[s]; ++k) {
                    long long o = S.soff[s] + 32LL * k + l;
                    if (r < M.n && k < M.ptr[r + 1] - M.ptr[r]) {
                        S.col[o] = M.col[M.ptr[r] + k];
                        S.val[o] = M.val[M.ptr[r] + k];
                    } else {
                        S.col[o] = 0;  // padding reads column 0 with value 0
                        S.val[o] = 0.0;
                    }
                }
            }
    };
    // CSR on the device (row blocks; column and value arrays padded by 4 entries: k_csr copies
    // 16-byte aligned supersets of each block's ranges)
    auto upload_csr = [](const Sell& S, CsrBufs& B) {
        B.rb.upload(S.rb);
        B.wb.upload(S.wb);
        B.ptr.upload(S.cptr);
        std::vector<int> cc(S.ccol);
        cc.resize(cc.size() + 4, 0);
        B.col.upload(cc);
        std::vector<double> vv(S.cval);
        vv.resize(vv.size() + 4, 0.0);
        B.v64.upload(vv);
        std::vector<float> f(vv.begin(), vv.end());
        B.v32.upload(f);
    };
    while (true) {
        Level L;
        L.n = A.n;
        L.dinv.resize(A.n);
        for (int i = 0; i < A.n; ++i) {
            double d = diag_of(A, i);
            L.dinv[i] = d != 0.0 ? 1.0 / d : 0.0;
        }
        // the finest level is coarsened in the given matrix's order (aggregation visits rows in
        // order) and stored in fine_order, the order of the vectors it will act on
        const bool fine = levels_.empty() && fine_order;
        const std::vector<double> dinv_own(L.dinv);  // in A's own order (smoothing, spectral radius)
        if (fine)
            for (int i = 0; i < A.n; ++i) L.dinv[(*fine_order)[i]] = dinv_own[i];
        // prolongator (smoothed aggregation, or the given one on the finest level)
        HostCsr P;
        int nagg = 0;
        bool last = A.n <= COARSE_MAX || levels_.size() >= 16;
        if (!last && levels_.empty() && first_P) {
            if (first_P->n != A.n || first_P->m <= 0 || first_P->m >= A.n)
                throw Error(VG_EINVAL, "first multigrid prolongator does not fit the matrix");
            L.omega = 4.0 / (3.0 * rho_dinv_a(A, dinv_own));
            P = *first_P;
            nagg = P.m;
            L.fixedP = true;
        } else if (!last) {
            std::vector<int> agg = aggregate(A, theta, nagg);
            if (nagg >= A.n || nagg == 0) {
                last = true;  // no coarsening possible
            } else {
                L.omega = 4.0 / (3.0 * rho_dinv_a(A, dinv_own));
                P = smoothed_prolongator(A, agg, nagg, dinv_own, L.omega);
                L.agg.resize(A.n);
                for (int i = 0; i < A.n; ++i) L.agg[fine ? (*fine_order)[i] : i] = agg[i];
            }
        }
        // stored operator: A S (columns scaled by omega D^{-1}) on a level with a coarser one; the
        // coarsest level keeps only its pattern (refresh) and is inverted densely
        {
            HostCsr Ast = fine ? permute_csr(A, fine_order, fine_order) : A;
            L.pa_ptr = Ast.ptr;
            L.pa_col = Ast.col;
            if (!last) {
                for (size_t j = 0; j < Ast.col.size(); ++j) Ast.val[j] *= L.omega * L.dinv[Ast.col[j]];
                to_sell(Ast, L.A, levels_.empty());
                if (!L.A.csr) {
                    L.sellpos.resize(Ast.col.size());
                    for (int r = 0; r < Ast.n; ++r)
                        for (int j = Ast.ptr[r]; j < Ast.ptr[r + 1]; ++j)
                            L.sellpos[j] = L.A.soff[r / 32] + 32LL * (j - Ast.ptr[r]) + r % 32;
                }
            }
        }
        if (last) {
            if (fine) A = permute_csr(A, fine_order, fine_order);
            levels_.push_back(std::move(L));
            break;
        }
        HostCsr R = transpose(P);
        HostCsr AP = spgemm(A, P);
        HostCsr Ac = spgemm(R, AP);
        HostCsr Pt = transfer_smooth(P, AP, dinv_own, L.omega);
        L.nc = nagg;
        {
            HostCsr Pst = fine ? permute_csr(P, fine_order, nullptr) : P;
            HostCsr Rst = transpose_map(Pst, L.r2p);
            L.cP.ptr.upload(Pst.ptr);
            L.cP.col.upload(Pst.col);
            L.cP.v64.upload(Pst.val);
            L.cR.ptr.upload(Rst.ptr);
            L.cR.col.upload(Rst.col);
            L.cR.v64.upload(Rst.val);
            HostCsr Ptst = fine ? permute_csr(Pt, fine_order, nullptr) : Pt;
            HostCsr Rtst = transpose_map(Ptst, L.rt2pt);
            to_sell(Ptst, L.Pt, false);
            to_sell(Rtst, L.Rt, false);
        }
        levels_.push_back(std::move(L));
        A = std::move(Ac);
        pt.mark("multigrid level (host)");
    }
    // coarsest level: dense inverse (bounded size; otherwise the caller keeps its diagonal preconditioner)
    if (A.n > DENSE_MAX) {
        levels_.clear();
        throw Error(VG_EINVAL, "multigrid coarsening stalled at " + std::to_string(A.n) + " rows");
    }
    ncoarse_ = A.n;
    dense_inverse_device(dense_of(A), A.n);
    pt.mark("coarsest dense inverse");
    if (PhaseTimer::stats_enabled()) {
        // diagnostics: rows and stored entries of every level (stderr)
        for (size_t l = 0; l < levels_.size(); ++l) {
            const Level& L = levels_[l];
            std::fprintf(stderr, "amg level %zu: rows %d A %zu (%s) Pt %zu Rt %zu omega %.3f\n", l, L.n,
                         L.pa_col.size(), L.A.csr ? "csr" : "sell", L.Pt.ccol.size(), L.Rt.ccol.size(), L.omega);
        }
        std::fprintf(stderr, "amg coarsest dense: %d rows\n", ncoarse_);
    }
    // uploads
    for (size_t l = 0; l < levels_.size(); ++l) {
        Level& L = levels_[l];
        const bool coarsest = l + 1 == levels_.size();
        if (!coarsest) {
            if (L.A.csr) {
                upload_csr(L.A, L.cA);
            } else {
                L.dA_soff.upload(L.A.soff);
                L.dA_w.upload(L.A.width);
                L.dA_col.upload(L.A.col);
                L.dA_v64.upload(L.A.val);
                std::vector<float> f(L.A.val.begin(), L.A.val.end());
                L.dA_v32.upload(f);
            }
            upload_csr(L.Pt, L.cPt);
            upload_csr(L.Rt, L.cRt);
            if (!L.agg.empty()) L.dagg.upload(L.agg);
            L.dr2p.upload(L.r2p);
            L.drt2pt.upload(L.rt2pt);
            if (!L.sellpos.empty()) L.dsellpos.upload(L.sellpos);
        }
        L.dpa_ptr.upload(L.pa_ptr);
        L.dpa_col.upload(L.pa_col);
        if (l > 0) L.dvals.resize(L.pa_col.size());  // written by refresh()
        L.dinv64.upload(L.dinv);
        std::vector<float> f(L.dinv.begin(), L.dinv.end());
        L.dinv32.upload(f);
        for (auto* b : {&L.x64, &L.b64, &L.r64}) b->resize(L.n);
        for (auto* b : {&L.x32, &L.b32, &L.r32}) b->resize(L.n);
    }
    err_.resize(1);
    err_.zero();
    prepare_csr_kernels(csr_slots_);
    VG_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
    ev_fork_.assign(levels_.size(), nullptr);
    ev_join_.assign(levels_.size(), nullptr);
    for (size_t l = 0; l < levels_.size(); ++l) {
        VG_CUDA(cudaEventCreateWithFlags(&ev_fork_[l], cudaEventDisableTiming));
        VG_CUDA(cudaEventCreateWithFlags(&ev_join_[l], cudaEventDisableTiming));
    }
    pt.mark("multigrid uploads");
}

template <typename T>
DevSell<T> Amg::view(const Level& L) const {
    DevSell<T> v;
    v.n = L.A.n;
    v.nslices = L.A.nslices;
    v.soff = L.dA_soff.data();
    v.width = L.dA_w.data();
    v.col = L.dA_col.data();
    if constexpr (sizeof(T) == 8)
        v.val = reinterpret_cast<const T*>(L.dA_v64.data());
    else
        v.val = reinterpret_cast<const T*>(L.dA_v32.data());
    return v;
}

template <typename T>
DevCsr<T> Amg::cview(const Sell& S, const CsrBufs& B) const {
    DevCsr<T> v;
    v.n = S.n;
    v.nblk = S.csr ? int(S.rb.size() / 2) - 1 : 0;
    v.slots = csr_slots_[sizeof(T) == 8 ? 1 : 0];
    v.lpr = S.lpr;
    v.err = const_cast<int*>(err_.data());
    v.rb = reinterpret_cast<const int2*>(B.rb.data());
    v.nwb = S.csr ? int(S.wb.size() / 2) - 1 : 0;
    v.wb = reinterpret_cast<const int2*>(B.wb.data());
    v.ptr = B.ptr.data();
    v.col = B.col.data();
    if constexpr (sizeof(T) == 8)
        v.val = reinterpret_cast<const T*>(B.v64.data());
    else
        v.val = reinterpret_cast<const T*>(B.v32.data());
    return v;
}

// one level of the composite V(1,1) cycle (the same operator as Jacobi pre-smoothing from zero,
// residual, restriction, coarse correction, prolongation and Jacobi post-smoothing):
//   side stream:  q = S (b + r), r = b - (A S) b   (stored in the level's r buffer)
//   this stream:  b_c = Rt b;  x_c = cycle(b_c);  z = q + Pt x_c
template <typename T>
void Amg::cycle(int l, const T* b, T* z, cudaStream_t s) {
    Level& L = levels_[l];
    auto buf = [&](DevBuf<double>& d64, DevBuf<float>& d32) -> T* {
        if constexpr (sizeof(T) == 8)
            return reinterpret_cast<T*>(d64.data());
        else
            return reinterpret_cast<T*>(d32.data());
    };
    if (l == int(levels_.size()) - 1) {
        const T* inv = sizeof(T) == 8 ? reinterpret_cast<const T*>(dinvc64_.data())
                                      : reinterpret_cast<const T*>(dinvc32_.data());
        launch_pdl(k_dense<T>, (ncoarse_ + DENSE_WARPS - 1) / DENSE_WARPS, DENSE_WARPS * 32, 0, s, ncoarse_, inv, b, z);
        ++launches;
        return;
    }
    Level& C = levels_[l + 1];
    const T* dinv = buf(L.dinv64, L.dinv32);
    T* r = buf(L.r64, L.r32);
    T* bc = buf(C.b64, C.b32);
    T* xc = buf(C.x64, C.x32);
    VG_CUDA(cudaEventRecord(ev_fork_[l], s));
    VG_CUDA(cudaStreamWaitEvent(side_, ev_fork_[l], 0));
    if (L.A.csr)
        launch_prod<T>(2, cview<T>(L.A, L.cA), dinv, T(L.omega), b, b, r, nullptr, side_);
    else
        launch_pdl(k_sell_residual<T>, blocks(L.n), TPB, 0, side_, view<T>(L), dinv, T(L.omega), b, r);
    VG_CUDA(cudaEventRecord(ev_join_[l], side_));
    launch_prod<T>(0, cview<T>(L.Rt, L.cRt), nullptr, T(0), nullptr, b, bc, nullptr, s);
    cycle<T>(l + 1, bc, xc, s);
    VG_CUDA(cudaStreamWaitEvent(s, ev_join_[l], 0));
    launch_prod<T>(1, cview<T>(L.Pt, L.cPt), dinv, T(L.omega), b, xc, z, r, s);
    launches += 3;
}

bool Amg::failed() {
    if (err_.size() == 0) return false;
    int e = 0;
    VG_CUDA(cudaMemcpy(&e, err_.data(), sizeof(int), cudaMemcpyDeviceToHost));
    if (e) err_.zero();
    return e != 0;
}

void Amg::vcycle(const double* b, double* z, cudaStream_t s) {
    cycle<double>(0, b, z, s);
    VG_CUDA(cudaGetLastError());
}

void Amg::vcycle(const float* b, float* z, cudaStream_t s) {
    cycle<float>(0, b, z, s);
    VG_CUDA(cudaGetLastError());
}

}  // namespace vg
