// Preconditioned MINRES (Paige-Saunders, in the form with unnormalised Lanczos vectors and a
// symmetric positive definite preconditioner) on the symmetric saddle-point system
//     [A, -W^T; -W, 0] [u; p] = [g; -f],
// replacing the PETSc FGMRES of vem/CurvedVEM_Darcy_gpu/src/krylov.cu:49-175. Per iteration:
//   (a) apply        y = K z_j and delta_j = z_j^T K z_j (fused, vg_apply.cu)
//   (b) update       v_{j+1} = y/g_j - (delta_j/g_j^2) v_j - (g_j/g_{j-1}) v_{j-1},
//                    z_{j+1} = P^{-1} v_{j+1}, gamma_{j+1} = sqrt(z_{j+1}.v_{j+1}), clear y,
//                    Givens rotation, residual estimate (last block, device scalars)
//   (c) step         w_{j+1} = (z_j/g_j - a3 w_{j-1} - a2 w_j)/a1, x += c_{j+1} eta_j w_{j+1}
// All scalars stay on the device; convergence sets a stop flag that turns the remaining kernels
// of a batch into no-ops, so iterations run without host synchronisation. Every reduction is a
// fixed-shape two-level sum (block partials, last block sums them in order): results are
// bitwise reproducible.
#include "vg_krylov.cuh"
#include "vg_pipe.cuh"

namespace vg {

namespace {

// [lo, hi) split into a scalar head up to a multiple of 4, 4-wide body, scalar tail; grid-stride
template <class F4, class F1>
__device__ __forceinline__ void for_range(long long lo, long long hi, F4 body4, F1 body1) {
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, nth = (long long)gridDim.x * blockDim.x;
    long long a = (lo + 3) & ~3LL;
    if (a > hi) a = hi;
    const long long b = a + ((hi - a) & ~3LL);
    for (long long i = lo + tid; i < a; i += nth) body1(i);
    for (long long i = a + 4 * tid; i < b; i += 4 * nth) body4(i);
    for (long long i = b + tid; i < hi; i += nth) body1(i);
}

// block + grid reduction of NV values; the last block to finish calls fin(total)
template <int NV, class F>
__device__ void grid_reduce(double (&v)[NV], double* partials, unsigned* counter, F fin) {
    __shared__ double sh[VEC_THREADS / 32][NV];
    __shared__ double tot[VEC_THREADS][NV];
    __shared__ bool last;
    const int t = threadIdx.x, w = t >> 5, l = t & 31;
#pragma unroll
    for (int i = 0; i < NV; ++i)
        for (int off = 16; off; off >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], off);
    if (l == 0)
#pragma unroll
        for (int i = 0; i < NV; ++i) sh[w][i] = v[i];
    __syncthreads();
    if (t == 0) {
        for (int i = 0; i < NV; ++i) {
            double s = 0;
            for (int k = 0; k < VEC_THREADS / 32; ++k) s += sh[k][i];
            partials[NV * blockIdx.x + i] = s;
        }
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] = 0;
    for (int b = t; b < (int)gridDim.x; b += VEC_THREADS)
#pragma unroll
        for (int i = 0; i < NV; ++i) acc[i] += __ldcg(partials + NV * b + i);
#pragma unroll
    for (int i = 0; i < NV; ++i) tot[t][i] = acc[i];
    __syncthreads();
    for (int s = VEC_THREADS / 2; s; s >>= 1) {
        if (t < s)
#pragma unroll
            for (int i = 0; i < NV; ++i) tot[t][i] += tot[t + s][i];
        __syncthreads();
    }
    if (t == 0) {
        double r[NV];
        for (int i = 0; i < NV; ++i) r[i] = tot[0][i];
        fin(r);
        *counter = 0u;
    }
}

__device__ void init_scalars(Scalars* sc, int* flags, double g2, double tol) {
    double g = sqrt(fmax(g2, 0.0));
    sc->gam = g;
    sc->gam_prev = 1.0;
    sc->c_prev = 1.0;
    sc->c = 1.0;
    sc->s_prev = 0.0;
    sc->s = 0.0;
    sc->eta = g;
    sc->eta0 = g;
    sc->tol = tol;
    flags[0] = (g > 0 && isfinite(g)) ? 0 : 1;
    flags[1] = 0;
    flags[2] = 0;
}

// Givens rotation and residual estimate once gamma_{j+1}^2 is known
__device__ void update_scalars(Scalars* sc, int* flags, double gn2) {
    const double g = sc->gam, dl = sc->delta / (g * g);
    double gn = sqrt(fmax(gn2, 0.0));
    double c = sc->c, cp = sc->c_prev, s = sc->s, sp = sc->s_prev, eta = sc->eta;
    double a0 = c * dl - cp * s * g;
    double a1 = sqrt(a0 * a0 + gn * gn);
    double a2 = s * dl + cp * c * g;
    double a3 = sp * g;
    bool ok = a1 > 0 && isfinite(a1);
    double cn = ok ? a0 / a1 : 1.0, sn = ok ? gn / a1 : 0.0;
    sc->a1 = ok ? a1 : 1.0;
    sc->a2 = a2;
    sc->a3 = a3;
    sc->zscale = 1.0 / g;
    sc->xcoef = ok ? cn * eta : 0.0;
    sc->eta = -sn * eta;
    sc->c_prev = c;
    sc->c = cn;
    sc->s_prev = s;
    sc->s = sn;
    sc->gam_prev = g;
    sc->gam = gn;
    flags[1] = ok ? 1 : 0;
    flags[2] += 1;
    if (!ok || !(gn > 0) || fabs(sc->eta) <= sc->tol * sc->eta0) flags[0] = 1;
}

// entries in [plo, phi) (the pressure block when it is preconditioned by multigrid) are left to
// the V-cycle: z is not written there and the dot product is finished by k_finish
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_init(const T* r, MinresVecs<T> v, long long n, Scalars* sc,
                                                      int* flags, double tol, double* partials, unsigned* counter,
                                                      long long plo, long long phi) {
    double acc[1] = {0};
    auto one = [&](long long i) {
        T ri = r[i];
        v.v_cur[i] = ri;
        v.v_old[i] = T(0);
        v.w_cur[i] = T(0);
        v.w_old[i] = T(0);
        v.y[i] = T(0);
        if (i < plo || i >= phi) {
            T zi = v.dinv[i] * ri;
            v.z_cur[i] = zi;
            acc[0] += double(zi) * double(ri);
        }
    };
    auto four = [&](long long i) {
        T r4[4], z0[4] = {T(0), T(0), T(0), T(0)};
        ld4(r + i, r4);
        st4(v.v_cur + i, r4);
        st4(v.v_old + i, z0);
        st4(v.w_cur + i, z0);
        st4(v.w_old + i, z0);
        st4(v.y + i, z0);
        if (i + 3 < plo || i >= phi) {
            T d4[4], zi[4];
            ld4(v.dinv + i, d4);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                zi[j] = d4[j] * r4[j];
                acc[0] += double(zi[j]) * double(r4[j]);
            }
            st4(v.z_cur + i, zi);
        } else {
            for (int j = 0; j < 4; ++j)
                if (i + j < plo || i + j >= phi) {
                    T zi = v.dinv[i + j] * r4[j];
                    v.z_cur[i + j] = zi;
                    acc[0] += double(zi) * double(r4[j]);
                }
        }
    };
    for_range(0, n, four, one);
    const bool split = phi > plo;
    grid_reduce<1>(acc, partials, counter, [&](double* tot) {
        if (split)
            sc->dot = tot[0];
        else
            init_scalars(sc, flags, tot[0], tol);
    });
}

template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_update(MinresVecs<T> v, long long lo, long long hi, Scalars* sc,
                                                        int* flags, double* partials, unsigned* counter,
                                                        long long plo, long long phi, int reduce) {
    // the first V-cycle kernel after this one (launched with programmatic dependent launch) may
    // start now and copy its matrix rows while the update runs; it waits for the update's results
    pdl_trigger();
    if (flags[0]) {
        if (reduce && blockIdx.x == 0 && threadIdx.x == 0) flags[1] = 0;
        return;
    }
    const double g = sc->gam, gp = sc->gam_prev, dl = sc->delta / (g * g);
    const T f1 = T(1.0 / g), f2 = T(dl / g), f3 = T(g / gp);
    double acc[1] = {0};
    auto one = [&](long long i) {
        T vn = v.y[i] * f1 - f2 * v.v_cur[i] - f3 * v.v_old[i];
        v.v_old[i] = vn;
        v.y[i] = T(0);
        if (i < plo || i >= phi) {
            T zn = v.dinv[i] * vn;
            v.z_new[i] = zn;
            acc[0] += double(zn) * double(vn);
        }
    };
    auto four = [&](long long i) {
        T y4[4], vc[4], vo[4], vn[4], z0[4] = {T(0), T(0), T(0), T(0)};
        ld4(v.y + i, y4);
        ld4(v.v_cur + i, vc);
        ld4(v.v_old + i, vo);
#pragma unroll
        for (int j = 0; j < 4; ++j) vn[j] = y4[j] * f1 - f2 * vc[j] - f3 * vo[j];
        st4(v.v_old + i, vn);
        st4(v.y + i, z0);
        if (i + 3 < plo || i >= phi) {
            T d4[4], zn[4];
            ld4(v.dinv + i, d4);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                zn[j] = d4[j] * vn[j];
                acc[0] += double(zn[j]) * double(vn[j]);
            }
            st4(v.z_new + i, zn);
        } else {
            for (int j = 0; j < 4; ++j)
                if (i + j < plo || i + j >= phi) {
                    T zn = v.dinv[i + j] * vn[j];
                    v.z_new[i + j] = zn;
                    acc[0] += double(zn) * double(vn[j]);
                }
        }
    };
    for_range(lo, hi, four, one);
    if (!reduce) return;
    const bool split = phi > plo;
    grid_reduce<1>(acc, partials, counter, [&](double* tot) {
        if (split)
            sc->dot = tot[0];
        else
            update_scalars(sc, flags, tot[0]);
    });
}

// pressure part of gamma^2 = z . v after the V-cycle, then the scalar update (init or iteration)
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_finish(const T* z, const T* vv, long long plo, long long phi,
                                                        Scalars* sc, int* flags, double* partials, unsigned* counter,
                                                        int init, double tol) {
    if (!init && flags[0]) return;
    double acc[1] = {0};
    for_range(
        plo, phi,
        [&](long long i) {
            T z4[4], v4[4];
            ld4(z + i, z4);
            ld4(vv + i, v4);
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[0] += double(z4[j]) * double(v4[j]);
        },
        [&](long long i) { acc[0] += double(z[i]) * double(vv[i]); });
    grid_reduce<1>(acc, partials, counter, [&](double* tot) {
        double g2 = tot[0] + sc->dot;
        if (init)
            init_scalars(sc, flags, g2, tol);
        else
            update_scalars(sc, flags, g2);
    });
}

template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_step(MinresVecs<T> v, long long n, Scalars* sc, int* flags) {
    if (!flags[1]) return;
    const T zs = T(sc->zscale), a2 = T(sc->a2), a3 = T(sc->a3), ia1 = T(1.0 / sc->a1), xc = T(sc->xcoef);
    for_range(
        0, n,
        [&](long long i) {
            T z4[4], wo[4], wc[4], x4[4], wn[4];
            ld4(v.z_cur + i, z4);
            ld4(v.w_old + i, wo);
            ld4(v.w_cur + i, wc);
            ld4(v.x + i, x4);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                wn[j] = (z4[j] * zs - a3 * wo[j] - a2 * wc[j]) * ia1;
                x4[j] += xc * wn[j];
            }
            st4(v.w_old + i, wn);
            st4(v.x + i, x4);
        },
        [&](long long i) {
            T wn = (v.z_cur[i] * zs - a3 * v.w_old[i] - a2 * v.w_cur[i]) * ia1;
            v.w_old[i] = wn;
            v.x[i] += xc * wn;
        });
}

// end of one body of the graph's while loop: continue while not converged and below the cap
__global__ void k_loop_check(cudaGraphConditionalHandle h, const int* flags, int* loop) {
    int c = ++loop[0];
    cudaGraphSetConditional(h, (flags[0] == 0 && c < loop[1]) ? 1u : 0u);
}

__global__ void __launch_bounds__(VEC_THREADS) k_residual64(const double* b, const double* y, double* r, long long n,
                                                            double* red, double* partials, unsigned* counter) {
    double acc[2] = {0, 0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double bi = b[i], ri = bi - y[i];
        r[i] = ri;
        acc[0] += ri * ri;
        acc[1] += bi * bi;
    }
    grid_reduce<2>(acc, partials, counter, [&](double* tot) {
        red[0] = tot[0];
        red[1] = tot[1];
    });
}

__global__ void k_to_float(const double* in, float* out, double scale, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = float(scale * in[i]);
}

__global__ void k_axpy_from_float(double* x, const float* d, double scale, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] += scale * double(d[i]);
}

__global__ void k_flip(const double* in, double* out, long long nf, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = i < nf ? in[i] : -in[i];
}

__global__ void k_to_float_plain(const double* in, float* out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = float(in[i]);
}

}  // namespace

// the 4-wide kernels need every vector on a 16-byte boundary (cudaMalloc gives 256)
template <typename T>
void check_aligned(const MinresVecs<T>& v, const T* extra = nullptr) {
    const void* ps[] = {v.v_cur, v.v_old, v.z_cur, v.z_new, v.w_cur, v.w_old, v.y, v.x, v.dinv, extra};
    for (const void* p : ps)
        if (reinterpret_cast<uintptr_t>(p) % 16) throw Error(VG_EINVAL, "Krylov vectors must be 16-byte aligned");
}

template <typename T>
void minres_init(const T* r, MinresVecs<T> v, long long n, Scalars* sc, int* flags, double tol, double* partials,
                 unsigned* counter, cudaStream_t s, long long plo, long long phi) {
    check_aligned(v, r);
    k_init<T><<<VEC_BLOCKS, VEC_THREADS, 0, s>>>(r, v, n, sc, flags, tol, partials, counter, plo, phi);
    VG_CUDA(cudaGetLastError());
}

template <typename T>
void minres_update(MinresVecs<T> v, long long n, Scalars* sc, int* flags, double* partials, unsigned* counter,
                   cudaStream_t s, long long plo, long long phi) {
    minres_update_rows<T>(v, 0, n, 1, sc, flags, partials, counter, s, plo, phi);
}

template <typename T>
void minres_update_rows(MinresVecs<T> v, long long lo, long long hi, int reduce, Scalars* sc, int* flags,
                        double* partials, unsigned* counter, cudaStream_t s, long long plo, long long phi) {
    check_aligned(v);
    const int nb = reduce ? VEC_BLOCKS : int(std::min<long long>(VEC_BLOCKS, (hi - lo + 4 * VEC_THREADS - 1) / (4 * VEC_THREADS)));
    k_update<T><<<std::max(nb, 1), VEC_THREADS, 0, s>>>(v, lo, hi, sc, flags, partials, counter, plo, phi, reduce);
    VG_CUDA(cudaGetLastError());
}

template <typename T>
void minres_finish(const T* z, const T* v, long long plo, long long phi, Scalars* sc, int* flags, double* partials,
                   unsigned* counter, int init, double tol, cudaStream_t s) {
    if (reinterpret_cast<uintptr_t>(z) % 16 || reinterpret_cast<uintptr_t>(v) % 16)
        throw Error(VG_EINVAL, "Krylov vectors must be 16-byte aligned");
    k_finish<T><<<VEC_BLOCKS, VEC_THREADS, 0, s>>>(z, v, plo, phi, sc, flags, partials, counter, init, tol);
    VG_CUDA(cudaGetLastError());
}

template <typename T>
void minres_step(MinresVecs<T> v, long long n, Scalars* sc, int* flags, cudaStream_t s) {
    check_aligned(v);
    k_step<T><<<VEC_BLOCKS, VEC_THREADS, 0, s>>>(v, n, sc, flags);
    VG_CUDA(cudaGetLastError());
}

template void minres_init<double>(const double*, MinresVecs<double>, long long, Scalars*, int*, double, double*,
                                  unsigned*, cudaStream_t, long long, long long);
template void minres_init<float>(const float*, MinresVecs<float>, long long, Scalars*, int*, double, double*,
                                 unsigned*, cudaStream_t, long long, long long);
template void minres_update_rows<double>(MinresVecs<double>, long long, long long, int, Scalars*, int*, double*,
                                         unsigned*, cudaStream_t, long long, long long);
template void minres_update_rows<float>(MinresVecs<float>, long long, long long, int, Scalars*, int*, double*,
                                        unsigned*, cudaStream_t, long long, long long);
template void minres_update<double>(MinresVecs<double>, long long, Scalars*, int*, double*, unsigned*, cudaStream_t,
                                    long long, long long);
template void minres_update<float>(MinresVecs<float>, long long, Scalars*, int*, double*, unsigned*, cudaStream_t,
                                   long long, long long);
template void minres_finish<double>(const double*, const double*, long long, long long, Scalars*, int*, double*,
                                    unsigned*, int, double, cudaStream_t);
template void minres_finish<float>(const float*, const float*, long long, long long, Scalars*, int*, double*,
                                   unsigned*, int, double, cudaStream_t);
template void minres_step<double>(MinresVecs<double>, long long, Scalars*, int*, cudaStream_t);
template void minres_step<float>(MinresVecs<float>, long long, Scalars*, int*, cudaStream_t);

void loop_check(cudaGraphConditionalHandle h, const int* flags, int* loop, cudaStream_t s) {
    k_loop_check<<<1, 1, 0, s>>>(h, flags, loop);
    VG_CUDA(cudaGetLastError());
}

void residual64(const double* b, const double* y, double* r, long long n, double* red, double* partials,
                unsigned* counter, cudaStream_t s) {
    k_residual64<<<VEC_BLOCKS, VEC_THREADS, 0, s>>>(b, y, r, n, red, partials, counter);
    VG_CUDA(cudaGetLastError());
}

void to_float(const double* in, float* out, double scale, long long n, cudaStream_t s) {
    k_to_float<<<VEC_BLOCKS, VEC_THREADS, 0, s>>>(in, out, scale, n);
    VG_CUDA(cudaGetLastError());
}

void axpy_from_float(double* x, const float* d, double scale, long long n, cudaStream_t s) {
    k_axpy_from_float<<<VEC_BLOCKS, VEC_THREADS, 0, s>>>(x, d, scale, n);
    VG_CUDA(cudaGetLastError());
}

void flip_pressure(const double* in, double* out, long long nf, long long n, cudaStream_t s) {
    k_flip<<<VEC_BLOCKS, VEC_THREADS, 0, s>>>(in, out, nf, n);
    VG_CUDA(cudaGetLastError());
}

void to_float_plain(const double* in, float* out, long long n, cudaStream_t s) {
    k_to_float_plain<<<VEC_BLOCKS, VEC_THREADS, 0, s>>>(in, out, n);
    VG_CUDA(cudaGetLastError());
}

}  // namespace vg
