// Auxiliary per-cell kernels: preconditioner diagonal, right-hand-side lift, permeability rescale,
// adjoint contraction, FP64 axpy.
#include "vg_common.cuh"

namespace vg {

namespace {

__device__ __forceinline__ int packed_diag(int i, int n) { return i * n - i * (i - 1) / 2; }

// thread per slot: piece index and lane, false for padding lanes
__device__ __forceinline__ bool slot_of(const Piece* pieces, int npieces, Piece& P, int& lane) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int pc = int(t / PIECE);
    lane = int(t % PIECE);
    if (pc >= npieces) return false;
    P = pieces[pc];
    return lane < P.count;
}

// assembled diagonal of the flux block: d[g] += A_E,ii (at most two addends per edge dof)
__global__ void k_diag_flux(const double* A, const int* map, const Piece* pieces, int npieces, double* d) {
    Piece P;
    int lane;
    if (!slot_of(pieces, npieces, P, lane)) return;
    for (int i = 0; i < P.n; ++i) {
        int g = map[P.map_off + i * PIECE + lane];
        atomicAdd(d + (g < 0 ? ~g : g), A[P.a_off + (long long)packed_diag(i, P.n) * PIECE + lane]);
    }
}

// pressure diagonal S_rr = sum_i W_ri^2 / d_i over free flux dofs; multiplier contribution
__global__ void k_diag_finish(const double* W, const int* map, const int* slot_cell, const int* mask, const double* L,
                              const Piece* pieces, int npieces, int k, long long nf, double* d, double* contrib) {
    Piece P;
    int lane;
    if (!slot_of(pieces, npieces, P, lane)) return;
    const int q = (k + 1) * (k + 2) / 2, ed = (k + 1) * P.ne;
    const int cell = slot_cell[P.slot + lane];
    double c = 0;
    for (int r = 0; r < q; ++r) {
        double s = 0;
        for (int i = 0; i < P.n; ++i) {
            int g = map[P.map_off + i * PIECE + lane], idx = g < 0 ? ~g : g;
            if (mask && i < ed && mask[idx]) continue;
            double w = k == 0 ? 1.0 : W[P.w_off + (long long)(r * P.n + i) * PIECE + lane];
            s += w * w / fmax(fabs(d[idx]), 1e-300);
        }
        s = fmax(s, 1e-300);
        d[nf + (long long)cell * q + r] = s;
        double l = L[(long long)cell * q + r];
        c += l * l / s;
    }
    contrib[cell] = c;
}

__global__ void k_sum(const double* v, int n, double* out) {
    __shared__ double sh[256];
    int t = threadIdx.x;
    int chunk = (n + 255) / 256, lo = t * chunk, hi = min(n, lo + chunk);
    double s = 0;
    for (int i = lo; i < hi; ++i) s += v[i];
    sh[t] = s;
    __syncthreads();
    for (int st = 128; st; st >>= 1) {
        if (t < st) sh[t] += sh[t + st];
        __syncthreads();
    }
    if (t == 0) *out = sh[0];
}

__global__ void k_invert(double* d, const int* mask, long long nfp, int mult, long long N, const double* msum) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double v;
        if (i < nfp)
            v = (mask && mask[i]) ? 1.0 : 1.0 / fmax(fabs(d[i]), 1e-300);
        else
            v = 1.0 / fmax(*msum, 1e-300);
        d[i] = v;
    }
}

__global__ void k_lift(const int* mask, const double* g, const double* y, double* b, long long N) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        b[i] = mask[i] ? g[i] : b[i] - y[i];
}

__global__ void k_rescale(const double* theta, const int* slot_cell, const Piece* pieces, int npieces, const double* A0,
                          double* A64, float* A32) {
    Piece P;
    int lane;
    if (!slot_of(pieces, npieces, P, lane)) return;
    double et = exp(-theta[slot_cell[P.slot + lane]]);
    int npk = P.n * (P.n + 1) / 2;
    for (int e = 0; e < npk; ++e) {
        long long o = P.a_off + (long long)e * PIECE + lane;
        double v = et * A0[o];
        A64[o] = v;
        A32[o] = float(v);
    }
}

constexpr int ADJ_MAXN = 5 * MAX_NE + 24;

__global__ void k_contract(const double* A, const int* map, const int* slot_cell, const int* mask, const Piece* pieces,
                           int npieces, int k, const double* x, const double* mu, int constrained, double* g) {
    Piece P;
    int lane;
    if (!slot_of(pieces, npieces, P, lane)) return;
    const int ed = (k + 1) * P.ne;
    double u[ADJ_MAXN], w[ADJ_MAXN];
    for (int i = 0; i < P.n; ++i) {
        int gi = map[P.map_off + i * PIECE + lane], idx = gi < 0 ? ~gi : gi;
        double s = gi < 0 ? -1.0 : 1.0;
        u[i] = s * x[idx];
        w[i] = (constrained && i < ed && mask[idx]) ? 0.0 : s * mu[idx];
    }
    double acc = 0;
    long long e = 0;
    for (int i = 0; i < P.n; ++i)
        for (int c = i; c < P.n; ++c) {
            double a = A[P.a_off + (e++) * PIECE + lane];
            acc += c == i ? a * w[i] * u[i] : a * (w[i] * u[c] + w[c] * u[i]);
        }
    g[slot_cell[P.slot + lane]] = acc;
}

// ---- assembled matrix (comparator of the matrix-free apply): CSR values of
// [A, -W^T, L; W, 0, 0; L^T, 0, 0] in the reference sign, masked rows and columns zeroed and a unit
// diagonal on masked rows (constrained), every slot receiving at most two addends onto zero
__device__ __forceinline__ long long csr_find(const long long* rp, const int* ci, long long r, int c) {
    long long lo = rp[r], hi = rp[r + 1] - 1;
    while (lo <= hi) {
        long long mid = (lo + hi) >> 1;
        int v = ci[mid];
        if (v == c) return mid;
        if (v < c)
            lo = mid + 1;
        else
            hi = mid - 1;
    }
    return -1;
}

__global__ void k_assemble(const double* A, const double* W, const int* map, const int* slot_cell, const int* mask,
                           const double* L, const Piece* pieces, int npieces, int k, long long nf, long long N,
                           int constrained, int mult, const long long* rp, const int* ci, double* val, int* bad) {
    Piece P;
    int lane;
    if (!slot_of(pieces, npieces, P, lane)) return;
    const int q = (k + 1) * (k + 2) / 2, n = P.n;
    const int cell = slot_cell[P.slot + lane];
    auto add = [&](long long r, long long c, double v) {
        long long s = csr_find(rp, ci, r, int(c));
        if (s < 0)
            atomicExch(bad, 1);
        else
            atomicAdd(val + s, v);
    };
    auto gdof = [&](int i, double& sg) {
        int g = map[P.map_off + (long long)i * PIECE + lane];
        sg = g < 0 ? -1.0 : 1.0;
        return g < 0 ? ~g : g;
    };
    auto masked = [&](long long g) { return constrained && mask[g] != 0; };
    long long e = 0;
    for (int i = 0; i < n; ++i) {
        double si;
        const long long gi = gdof(i, si);
        for (int j = i; j < n; ++j, ++e) {
            double sj;
            const long long gj = gdof(j, sj);
            if (masked(gi) || masked(gj)) continue;
            const double a = A[P.a_off + e * PIECE + lane] * si * sj;
            add(gi, gj, a);
            if (j != i) add(gj, gi, a);
        }
    }
    for (int r = 0; r < q; ++r) {
        const long long pr = nf + (long long)cell * q + r;
        for (int i = 0; i < n; ++i) {
            double si;
            const long long gi = gdof(i, si);
            if (masked(gi)) continue;
            const double w = (k == 0 ? 1.0 : W[P.w_off + (long long)(r * n + i) * PIECE + lane]) * si;
            add(gi, pr, -w);
            add(pr, gi, w);
        }
        if (mult) {
            const double l = L[(long long)cell * q + r];
            add(pr, N - 1, l);
            add(N - 1, pr, l);
        }
    }
}

__global__ void k_assemble_mask(const int* mask, long long N, const long long* rp, const int* ci, double* val,
                                int* bad) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < N; g += (long long)gridDim.x * blockDim.x)
        if (mask[g]) {
            long long s = csr_find(rp, ci, g, int(g));
            if (s < 0)
                atomicExch(bad, 1);
            else
                val[s] = 1.0;
        }
}

// values of the pressure Schur block S = B diag(A)^{-1} B^T on its stored pattern (rows and columns
// in the solver's internal pressure order): row (E, r) sums over the flux dofs g of E, over the cells
// F around g and the moments r2 of F: W_E[r, i] s_Ei dinv[g] W_F[r2, j] s_Fj (k = 0: W = 1)
__global__ void k_schur_values(const int* sptr, const int* scol, int nrows, int q, int k, const int* rank_cell,
                               const int* cell_rank, const int* cell_slot, const Piece* pieces, const int* map,
                               const double* W, const double* dinv, const int* inc_ptr, const int* inc_cell,
                               const int* inc_i, const signed char* inc_s, double* sval) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    const int c = rank_cell[t / q], r = t % q;
    const int lo = sptr[t], hi = sptr[t + 1];
    for (int j = lo; j < hi; ++j) sval[j] = 0.0;
    const int slot = cell_slot[c];
    const Piece P = pieces[slot / PIECE];
    const int lane = slot % PIECE;
    for (int i = 0; i < P.n; ++i) {
        const int g0 = map[P.map_off + (long long)i * PIECE + lane], g = g0 < 0 ? ~g0 : g0;
        const double wi = k == 0 ? 1.0 : W[P.w_off + (long long)(r * P.n + i) * PIECE + lane];
        const double coef = wi * (g0 < 0 ? -1.0 : 1.0) * dinv[g];
        if (coef == 0.0) continue;
        for (int b = inc_ptr[g]; b < inc_ptr[g + 1]; ++b) {
            const int F = inc_cell[b], jf = inc_i[b];
            const int fslot = cell_slot[F];
            const Piece Q = pieces[fslot / PIECE];
            const int flane = fslot % PIECE;
            for (int r2 = 0; r2 < q; ++r2) {
                const int colv = cell_rank[F] * q + r2;
                const double wf = k == 0 ? 1.0 : W[Q.w_off + (long long)(r2 * Q.n + jf) * PIECE + flane];
                int a = lo, z = hi;
                while (a < z) {
                    int mid = (a + z) >> 1;
                    if (scol[mid] < colv)
                        a = mid + 1;
                    else
                        z = mid;
                }
                if (a < hi && scol[a] == colv) sval[a] += coef * wf * double(inc_s[b]);
            }
        }
    }
}

// out[j] = in[idx[j + off] - off]: a permutation of a vector (off = 0) or of its part from off on
template <typename T>
__global__ void k_gather(const T* in, const int* idx, long long off, T* out, long long n) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x)
        out[j] = in[idx[j + off] - off];
}

__global__ void k_axpy64(double* x, const double* d, double a, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] += a * d[i];
}

// smallest index of a non-finite entry (atomicMin into *first, which starts at n)
__global__ void k_first_nonfinite(const double* v, long long n, unsigned long long* first) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (!isfinite(v[i])) atomicMin(first, (unsigned long long)i);
}

inline int blocks_for(long long n) { return int((n + 255) / 256); }

}  // namespace

void diag_flux(const double* A, const int* map, const Piece* pieces, int npieces, double* d, cudaStream_t s) {
    k_diag_flux<<<blocks_for((long long)npieces * PIECE), 256, 0, s>>>(A, map, pieces, npieces, d);
    VG_CUDA(cudaGetLastError());
}

void diag_finish(const double* W, const int* map, const int* slot_cell, const int* mask, const double* L,
                 const Piece* pieces, int npieces, int k, long long nf, double* d, double* contrib, cudaStream_t s) {
    k_diag_finish<<<blocks_for((long long)npieces * PIECE), 256, 0, s>>>(W, map, slot_cell, mask, L, pieces, npieces,
                                                                         k, nf, d, contrib);
    VG_CUDA(cudaGetLastError());
}

void diag_invert(double* d, const int* mask, const double* contrib, int nc, long long nf, long long np, int mult,
                 long long N, cudaStream_t s) {
    DevBuf<double> msum(1);
    if (mult) {
        k_sum<<<1, 256, 0, s>>>(contrib, nc, msum.data());
        VG_CUDA(cudaGetLastError());
    }
    k_invert<<<148 * 4, 256, 0, s>>>(d, mask, nf + np, mult, N, msum.data());
    VG_CUDA(cudaGetLastError());
    VG_CUDA(cudaStreamSynchronize(s));
}

void lift_rhs(const int* mask, const double* g, const double* y, double* b, long long N, cudaStream_t s) {
    k_lift<<<148 * 4, 256, 0, s>>>(mask, g, y, b, N);
    VG_CUDA(cudaGetLastError());
}

void rescale_ops(const double* theta, const int* slot_cell, const Piece* pieces, int npieces, const double* A0,
                 double* A64, float* A32, cudaStream_t s) {
    k_rescale<<<blocks_for((long long)npieces * PIECE), 256, 0, s>>>(theta, slot_cell, pieces, npieces, A0, A64, A32);
    VG_CUDA(cudaGetLastError());
}

void contract_adjoint(const double* A, const int* map, const int* slot_cell, const int* mask, const Piece* pieces,
                      int npieces, int k, const double* x, const double* mu, int constrained, double* g,
                      cudaStream_t s) {
    k_contract<<<blocks_for((long long)npieces * PIECE), 256, 0, s>>>(A, map, slot_cell, mask, pieces, npieces, k, x, mu,
                                                                      constrained, g);
    VG_CUDA(cudaGetLastError());
}

void assemble_values(const double* A, const double* W, const int* map, const int* slot_cell, const int* mask,
                     const double* L, const Piece* pieces, int npieces, int k, long long nf, long long N,
                     int constrained, int mult, const long long* rp, const int* ci, double* val, int* bad,
                     cudaStream_t s) {
    k_assemble<<<blocks_for((long long)npieces * PIECE), 256, 0, s>>>(A, W, map, slot_cell, mask, L, pieces, npieces, k,
                                                                       nf, N, constrained, mult, rp, ci, val, bad);
    VG_CUDA(cudaGetLastError());
    if (constrained) {
        k_assemble_mask<<<148 * 4, 256, 0, s>>>(mask, N, rp, ci, val, bad);
        VG_CUDA(cudaGetLastError());
    }
}

void schur_values(const int* sptr, const int* scol, int nrows, int q, int k, const int* rank_cell, const int* cell_rank,
                  const int* cell_slot, const Piece* pieces, const int* map, const double* W, const double* dinv,
                  const int* inc_ptr, const int* inc_cell, const int* inc_i, const signed char* inc_s, double* sval) {
    k_schur_values<<<(nrows + 255) / 256, 256>>>(sptr, scol, nrows, q, k, rank_cell, cell_rank, cell_slot, pieces, map, W,
                                                 dinv, inc_ptr, inc_cell, inc_i, inc_s, sval);
    VG_CUDA(cudaGetLastError());
}

template <typename T>
void gather_launch(const T* in, const int* idx, long long off, T* out, long long n, cudaStream_t s) {
    if (n <= 0) return;
    k_gather<T><<<148 * 4, 256, 0, s>>>(in, idx, off, out, n);
    VG_CUDA(cudaGetLastError());
}
template void gather_launch<double>(const double*, const int*, long long, double*, long long, cudaStream_t);
template void gather_launch<float>(const float*, const int*, long long, float*, long long, cudaStream_t);
template void gather_launch<int>(const int*, const int*, long long, int*, long long, cudaStream_t);

long long first_nonfinite(const double* v, long long n) {
    DevBuf<unsigned long long> first(1);
    const unsigned long long init = (unsigned long long)n;
    VG_CUDA(cudaMemcpy(first.data(), &init, sizeof(init), cudaMemcpyHostToDevice));
    k_first_nonfinite<<<148 * 4, 256>>>(v, n, first.data());
    VG_CUDA(cudaGetLastError());
    unsigned long long out = init;
    VG_CUDA(cudaMemcpy(&out, first.data(), sizeof(out), cudaMemcpyDeviceToHost));
    return out < init ? (long long)out : -1;
}

void axpy64_kernel_launch(double* x, const double* d, double a, long long n, cudaStream_t s) {
    k_axpy64<<<148 * 4, 256, 0, s>>>(x, d, a, n);
    VG_CUDA(cudaGetLastError());
}

}  // namespace vg
