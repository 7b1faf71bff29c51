// Krylov kernels: preconditioned MINRES on the symmetric saddle-point form, FP64 residuals for
// iterative refinement, the adjoint contraction.
#pragma once
#include "vg_common.cuh"

namespace vg {

// MINRES scalars, device resident (double precision for both FP64 and FP32 inner solves)
struct Scalars {
    double gam_prev, gam, delta;   // gamma_{j-1}, gamma_j, raw z_j^T K z_j (from the apply)
    double c_prev, c, s_prev, s;   // Givens c_{j-1}, c_j, s_{j-1}, s_j
    double eta, eta0, tol;         // residual estimate |eta| (preconditioner norm), stop at tol * eta0
    double a1, a2, a3, xcoef, zscale;
    double dot;                    // scratch
};
// flags[0] = stop (converged or breakdown), flags[1] = current iteration valid, flags[2] = iterations
constexpr int NFLAGS = 4;

constexpr int VEC_BLOCKS = 148 * 4;  // grid of the vector kernels (fixed: deterministic reductions)
constexpr int VEC_THREADS = 256;

template <typename T>
struct MinresVecs {
    T *v_cur, *v_old, *z_cur, *z_new, *w_cur, *w_old, *y, *x;
    const T* dinv;
};

// z = dinv .* r ; v_cur = r ; v_old = w_cur = w_old = y = 0 ; gamma_1 = sqrt(z.r)
template <typename T>
void minres_init(const T* r, MinresVecs<T> v, long long n, Scalars* sc, int* flags, double tol, double* partials,
                 unsigned* counter, cudaStream_t s, long long plo = 0, long long phi = 0);
// v_new = y/g - (d/g) v_cur - (g/g_prev) v_old (into v_old), z_new = dinv .* v_new, y = 0, scalars
template <typename T>
void minres_update(MinresVecs<T> v, long long n, Scalars* sc, int* flags, double* partials, unsigned* counter,
                   cudaStream_t s, long long plo = 0, long long phi = 0);
// the same on rows [lo, hi) only; reduce = 0: no dot product and no scalar update (a part of the
// rows processed beside another launch that reduces)
template <typename T>
void minres_update_rows(MinresVecs<T> v, long long lo, long long hi, int reduce, Scalars* sc, int* flags,
                        double* partials, unsigned* counter, cudaStream_t s, long long plo, long long phi);
// gamma^2 over [plo, phi) + the partial of init / update, then the scalar recurrences
template <typename T>
void minres_finish(const T* z, const T* v, long long plo, long long phi, Scalars* sc, int* flags, double* partials,
                   unsigned* counter, int init, double tol, cudaStream_t s);
// w_new = (z_cur/g - a3 w_old - a2 w_cur)/a1 (into w_old), x += xcoef w_new
template <typename T>
void minres_step(MinresVecs<T> v, long long n, Scalars* sc, int* flags, cudaStream_t s);

// graph while-loop condition: loop[0] = bodies run (incremented here), loop[1] = cap on bodies
void loop_check(cudaGraphConditionalHandle h, const int* flags, int* loop, cudaStream_t s);
// r = b - y (FP64), red[0] = ||r||^2, red[1] = ||b||^2 (deterministic)
void residual64(const double* b, const double* y, double* r, long long n, double* red, double* partials,
                unsigned* counter, cudaStream_t s);
// out32 = float(scale * in64)
void to_float(const double* in, float* out, double scale, long long n, cudaStream_t s);
// x64 += scale * double(d32)
void axpy_from_float(double* x, const float* d, double scale, long long n, cudaStream_t s);
// out = sign-flip of the pressure / multiplier block: out[i] = (i < nf ? 1 : -1) * in[i]
void flip_pressure(const double* in, double* out, long long nf, long long n, cudaStream_t s);
// dinv (float copy)
void to_float_plain(const double* in, float* out, long long n, cudaStream_t s);
// x += a d (FP64)
void axpy64_kernel_launch(double* x, const double* d, double a, long long n, cudaStream_t s);

}  // namespace vg
