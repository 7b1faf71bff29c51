// Shared device/host definitions of the vemgpu library: error type, device buffers, the scaled
// monomial / H(div) basis, quadrature tables, geometry maps and built-in PDE data.
//
// Mathematics follows the reference GPU project (vem/CurvedVEM_Darcy_gpu/include/device.cuh:151-222,
// include/problem_device.cuh:166-233) and its CPU modules (lib/polynomial_basis.cpp:95-293,
// core/gauss_quadrature.cpp:74-305, examples/darcy_problem.h:70-121). The basis helpers below
// (multi_index, mono, hdiv, binomial, edge_coeff, moment) are a deliberate restatement of the
// reference's exponent / mono / basis / binom / edge_coeff / moment (device.cuh:159-222): they fix
// the ordering and scaling of the monomial and H(div) degrees of freedom, which must be the same
// for the discrete operator and the solution vectors to match the reference entry for entry.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <stdexcept>
#include <string>
#include <vector>

#include "vemgpu.h"

namespace vg {

// ---------------------------------------------------------------------------------------------
// errors and device memory
// ---------------------------------------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(e == cudaErrorMemoryAllocation ? VG_ENOMEM : VG_ECUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
    }
}
#define VG_CUDA(call) ::vg::cuda_check((call), #call)

template <class T>
class DevBuf {
    T* p_ = nullptr;
    size_t n_ = 0;

public:
    DevBuf() = default;
    explicit DevBuf(size_t n) { resize(n); }
    ~DevBuf() {
        if (p_) cudaFree(p_);
    }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            if (p_) cudaFree(p_);
            p_ = o.p_;
            n_ = o.n_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    void resize(size_t n) {
        if (n == n_) return;
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
        if (n) VG_CUDA(cudaMalloc(&p_, n * sizeof(T)));
        n_ = n;
    }
    void upload(const std::vector<T>& v) {
        resize(v.size());
        if (n_) VG_CUDA(cudaMemcpy(p_, v.data(), n_ * sizeof(T), cudaMemcpyHostToDevice));
    }
    std::vector<T> download() const {
        std::vector<T> v(n_);
        if (n_) VG_CUDA(cudaMemcpy(v.data(), p_, n_ * sizeof(T), cudaMemcpyDeviceToHost));
        return v;
    }
    void zero(cudaStream_t s = nullptr) {
        if (n_) VG_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
    }
    T* data() { return p_; }
    const T* data() const { return p_; }
    size_t size() const { return n_; }
};

// diagnostics: wall time of setup phases on stderr when the environment sets VG_STATS=1
struct PhaseTimer {
    bool on;
    double t;
    static double now() {
        timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        return ts.tv_sec + 1e-9 * ts.tv_nsec;
    }
    PhaseTimer() : on(stats_enabled()), t(now()) {}
    static bool stats_enabled() {
        const char* e = std::getenv("VG_STATS");
        return e && *e == '1';
    }
    void mark(const char* what) {
        if (!on) return;
        const double n = now();
        std::fprintf(stderr, "vg setup %-28s %8.3f s\n", what, n - t);
        t = n;
    }
};

// ---------------------------------------------------------------------------------------------
// polynomial spaces
// ---------------------------------------------------------------------------------------------
__host__ __device__ inline int dimP(int k) { return k < 0 ? 0 : (k + 1) * (k + 2) / 2; }
__host__ __device__ inline int ngrad_of(int k) { return dimP(k + 1) - 1; }
__host__ __device__ inline int p_of(int k) { return ngrad_of(k) + dimP(k - 1); }
__host__ __device__ inline int internal_of(int k) { return dimP(k) - 1 + k * (k + 1) / 2; }

constexpr int MAX_NE = 16;    // largest polygon handled by the device kernels
constexpr int MAX_K = 4;
constexpr int MAX_QP = 36;    // points of one triangle rule
constexpr int MAX_GL = 10;

// status word written by kernels (first failure wins): code in the high bits, cell in the low
constexpr unsigned long long ST_SINGULAR = 1ull, ST_JACOBIAN = 2ull;

#ifdef __CUDACC__
// 16-byte vector access of 4 consecutive entries (the index is a multiple of 4 and every vector
// starts on a cudaMalloc boundary): 4 floats in one load, 4 doubles in two
__device__ __forceinline__ void ld4(const float* p, float (&o)[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = t.z;
    o[3] = t.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&o)[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    o[0] = a.x;
    o[1] = a.y;
    o[2] = b.x;
    o[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, const float (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&v)[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

__device__ __forceinline__ void set_status(unsigned long long* st, unsigned long long code, int cell) {
    atomicCAS(st, 0ull, (code << 40) | (unsigned long long)(unsigned)cell);
}

__host__ __device__ inline void multi_index(int i, int& a, int& b) {
    int d = 0;
    while (i > d) {
        i -= d + 1;
        ++d;
    }
    b = i;
    a = d - i;
}

__host__ __device__ inline double ipow(double x, int n) {
    double r = 1.0;
    for (int j = 0; j < n; ++j) r *= x;
    return r;
}

struct Frame {
    double cx, cy, h;
};

__host__ __device__ inline double mono(int i, const Frame& f, double x, double y) {
    int a, b;
    multi_index(i, a, b);
    return ipow((x - f.cx) / f.h, a) * ipow((y - f.cy) / f.h, b);
}

// gradients of P_{k+1} \ R first, then the complement (-(b+1)/a X^{a-1} Y^{b+1}, X^a Y^b)
__host__ __device__ inline void hdiv(int i, int k, const Frame& f, double x, double y, double& vx, double& vy) {
    double X = (x - f.cx) / f.h, Y = (y - f.cy) / f.h;
    int ng = dimP(k + 1) - 1;
    if (i < ng) {
        int a, b;
        multi_index(i + 1, a, b);
        vx = a ? a * ipow(X, a - 1) * ipow(Y, b) / f.h : 0.0;
        vy = b ? b * ipow(X, a) * ipow(Y, b - 1) / f.h : 0.0;
        return;
    }
    int z = i - ng, d = 1;
    while (z >= d) {
        z -= d;
        ++d;
    }
    int b = z, a = d - b;
    vx = -double(b + 1) / a * ipow(X, a - 1) * ipow(Y, b + 1);
    vy = ipow(X, a) * ipow(Y, b);
}

__host__ __device__ inline double binomial(int n, int k) {
    double r = 1;
    for (int j = 1; j <= k; ++j) r *= double(n - j + 1) / j;
    return r;
}

// coefficient of t^r of m_i restricted to the straight edge p0->p1, t = ((x-mid).tau)/L
__host__ __device__ inline double edge_coeff(int i, int r, const Frame& f, double x0, double y0, double x1, double y1) {
    double ex = x1 - x0, ey = y1 - y0;
    double X = (0.5 * (x0 + x1) - f.cx) / f.h, Y = (0.5 * (y0 + y1) - f.cy) / f.h;
    double dx = ex / f.h, dy = ey / f.h;
    int a, b;
    multi_index(i, a, b);
    double s = 0;
    for (int u = 0; u <= a; ++u) {
        int v = r - u;
        if (v >= 0 && v <= b) s += binomial(a, u) * binomial(b, v) * ipow(X, a - u) * ipow(Y, b - v) * ipow(dx, u) * ipow(dy, v);
    }
    return s;
}

// int_{-1/2}^{1/2} t^r dt
__host__ __device__ inline double moment(int r) { return (r & 1) ? 0.0 : ipow(0.5, r) / (r + 1); }

// ---------------------------------------------------------------------------------------------
// geometry maps
// ---------------------------------------------------------------------------------------------
struct Pt {
    double x, y, w;            // computational point and weight
    double X, Y;               // physical point
    double j00, j01, j10, j11, det;
};

__host__ __device__ inline void map_identity(Pt& s) {
    s.X = s.x;
    s.Y = s.y;
    s.j00 = 1;
    s.j01 = 0;
    s.j10 = 0;
    s.j11 = 1;
    s.det = 1;
}

__host__ __device__ inline void map_sine(Pt& s, double eps) {
    const double tp = 6.283185307179586476925286766559;
    s.X = s.x + eps * sin(tp * s.y);
    s.Y = s.y + eps * sin(tp * s.x);
    s.j00 = 1;
    s.j01 = eps * tp * cos(tp * s.y);
    s.j10 = eps * tp * cos(tp * s.x);
    s.j11 = 1;
    s.det = 1.0 - s.j01 * s.j10;
}

// triangle (c, a, b) whose side a->b is the chord of a circular arc of circle (ox, oy, r):
// x = c + lam (a - c + t e), F(x) = c + lam (gamma(t) - c), J = [gamma - c, gamma'] [a - c + t e, e]^{-1}
__host__ __device__ inline void map_arc(Pt& s, double cx, double cy, double ax, double ay, double bx, double by, double ox,
                                        double oy, double r) {
    const double pi = 3.14159265358979323846;
    double ex = bx - ax, ey = by - ay, dx = ax - cx, dy = ay - cy;
    double d0 = dx * ey - dy * ex;
    double rx = s.x - cx, ry = s.y - cy;
    double lam = (rx * ey - ry * ex) / d0, sl = (dx * ry - dy * rx) / d0;
    double t = lam > 0 ? sl / lam : 0.5;
    double ta = atan2(ay - oy, ax - ox), tb = atan2(by - oy, bx - ox);
    double dth = tb - ta;
    while (dth > pi) dth -= 2 * pi;
    while (dth < -pi) dth += 2 * pi;
    double th = ta + t * dth;
    double gx = ox + r * cos(th), gy = oy + r * sin(th);
    double gpx = -r * dth * sin(th), gpy = r * dth * cos(th);
    s.X = cx + lam * (gx - cx);
    s.Y = cy + lam * (gy - cy);
    double m00 = dx + t * ex, m01 = ex, m10 = dy + t * ey, m11 = ey;
    double md = m00 * m11 - m01 * m10;
    double i00 = m11 / md, i01 = -m01 / md, i10 = -m10 / md, i11 = m00 / md;
    double f00 = gx - cx, f01 = gpx, f10 = gy - cy, f11 = gpy;
    s.j00 = f00 * i00 + f01 * i10;
    s.j01 = f00 * i01 + f01 * i11;
    s.j10 = f10 * i00 + f11 * i10;
    s.j11 = f10 * i01 + f11 * i11;
    s.det = s.j00 * s.j11 - s.j01 * s.j10;
}

// ---------------------------------------------------------------------------------------------
// built-in PDE data (u = -grad p, K = I for the exact solutions)
// ---------------------------------------------------------------------------------------------
__host__ __device__ inline double prob_p(int kind, double X, double Y) {
    const double pi = 3.14159265358979323846;
    if (kind == VG_PROBLEM_SINCOS) return sin(pi * X) * cos(pi * Y);
    if (kind == VG_PROBLEM_SINSIN) return sin(pi * X) * sin(pi * Y);
    return log(sqrt(X * X + Y * Y)) / log(0.3);
}

__host__ __device__ inline void prob_u(int kind, double X, double Y, double& ux, double& uy) {
    const double pi = 3.14159265358979323846;
    if (kind == VG_PROBLEM_SINCOS) {
        ux = -pi * cos(pi * X) * cos(pi * Y);
        uy = pi * sin(pi * X) * sin(pi * Y);
    } else if (kind == VG_PROBLEM_SINSIN) {
        ux = -pi * cos(pi * X) * sin(pi * Y);
        uy = -pi * sin(pi * X) * cos(pi * Y);
    } else {
        double r2 = X * X + Y * Y, c = 1.0 / log(0.3);
        ux = -c * X / r2;
        uy = -c * Y / r2;
    }
}

__host__ __device__ inline double prob_f(int kind, double X, double Y) {
    const double pi = 3.14159265358979323846;
    if (kind == VG_PROBLEM_ANNULUS) return 0.0;
    return 2.0 * pi * pi * prob_p(kind, X, Y);
}

__host__ __device__ inline double prob_dirichlet(int kind, double X, double Y) {
    if (kind == VG_PROBLEM_ANNULUS) return sqrt(X * X + Y * Y) < 0.65 ? 1.0 : 0.0;
    return prob_p(kind, X, Y);
}
#endif  // __CUDACC__

// ---------------------------------------------------------------------------------------------
// packed cell triangle: local vertex ids (APEX = fan apex at the vertex average), arc edge or NO_ARC
// ---------------------------------------------------------------------------------------------
constexpr uint8_t APEX = 255, NO_ARC = 255;
struct TriIdx {
    uint8_t a, b, c, arc;
};

// Operator layout. Cells (in mesh order, which the generators make a Hilbert order) are cut into
// chunks of CHUNK cells; inside a chunk the cells are grouped by edge count and every group is
// split into pieces of at most PIECE cells. One piece = one warp in the apply kernel: its cells
// share the edge count (warp-uniform control flow) and live in one compact region of the mesh
// (gathers of x and scatters into y stay local). Per-cell arrays are stored piece-major with the
// lane innermost: entry e of lane l of a piece lives at off + e * PIECE + l, so every entry load of
// a warp is one coalesced 128-byte (FP32) or 256-byte (FP64) transaction.
constexpr int PIECE = 32;
constexpr int CHUNK = 4096;
struct Piece {
    int ne;            // edges per cell
    int n;             // local flux dofs
    int count;         // cells in the piece (<= PIECE); lanes >= count are padding
    int pad_;
    long long slot;    // first slot (PIECE per piece); slot = PIECE * piece + lane
    long long a_off;   // packed A_E, n(n+1)/2 entries per cell
    long long w_off;   // W_E (k >= 1), q n entries per cell
    long long map_off; // signed flux dof map, n entries per cell
    long long p_off;   // projector P, p n entries per cell
    long long hw_off;  // H^{-1} W, q n entries per cell
};

// cells with the same edge count (setup and error kernels are launched per class)
struct CellClass {
    int ne, n, count;
    const int* cells;  // device list
};

}  // namespace vg
