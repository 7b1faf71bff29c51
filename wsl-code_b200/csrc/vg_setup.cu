// FP64 per-polygon setup on the device: one warp per cell.
//
// For each cell the warp generates and maps its quadrature points, integrates the projector
// blocks and the equation factors, inverts the small Gram matrices and writes the packed local
// flux operator
//     A_E = P^T AG P + alpha (I - D P)^T (I - D P)        (K = exp(theta) I factored out)
// together with W_E, P, H^{-1} W, the multiplier vector L, the pressure right-hand side and the
// boundary data. The mathematics is that of the reference:
//   D, G, H, H*, W          vem/CurvedVEM_Darcy_gpu/src/hdiv_gpu.cu:10-78   (integrate_base)
//   H^{-1}, edge mass^{-1}, B = [B_grad; B_comp], P = G^{-1} B
//                           vem/CurvedVEM_Darcy_gpu/src/hdiv_gpu.cu:81-136  (projection)
//   AG = int g^T T g, T = J^T K^{-1} J / det J, alpha = ||int T||_F / area, M
//                           vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:148-195 (integrate_equation)
//   K_ac + K_as             vem/CurvedVEM_Darcy/solver/DarcySolver.cpp:1228-1269, 1476-1509
//   boundary moments        vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:317-337 (boundary_kernel)
//   pressure rhs            vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:340-373 (rhs_kernel)
// Differences of form: quadrature points are generated on the device from the cell's
// triangulation instead of being uploaded (no per-point host arrays), the whole chain runs in one
// kernel, and the local flux operator is formed explicitly (it is what the hot apply streams).
#include <algorithm>
#include <cmath>

#include "vg_setup.cuh"

namespace vg {

__constant__ double c_tri[3 * MAX_QP];   // (xi, eta, w) of the reference triangle rule
__constant__ double c_gl[2 * MAX_GL];    // (x, w) of the Gauss-Legendre rule on [-1, 1]

void upload_rules(const std::vector<double>& tri, const std::vector<double>& gl) {
    VG_CUDA(cudaMemcpyToSymbol(c_tri, tri.data(), tri.size() * sizeof(double)));
    VG_CUDA(cudaMemcpyToSymbol(c_gl, gl.data(), gl.size() * sizeof(double)));
}

namespace {

// warp-cooperative Gauss-Jordan inversion with partial pivoting; a is destroyed.
// A pivot that is not finite or below 1e-28 in magnitude marks the cell singular
// (the rule of vem/CurvedVEM_Darcy_gpu/include/device.cuh:226-274).
__device__ bool warp_inverse(double* a, double* inv, int n, int lane) {
    bool ok = true;
    for (int z = lane; z < n * n; z += 32) inv[z] = (z / n == z % n) ? 1.0 : 0.0;
    __syncwarp();
    for (int col = 0; col < n; ++col) {
        double best = -1.0;
        int bi = n;
        for (int i = col + lane; i < n; i += 32) {
            double v = fabs(a[i * n + col]);
            if (v > best) {
                best = v;
                bi = i;
            }
        }
        for (int off = 16; off; off >>= 1) {
            double ob = __shfl_down_sync(0xffffffffu, best, off);
            int oi = __shfl_down_sync(0xffffffffu, bi, off);
            if (ob > best || (ob == best && oi < bi)) {
                best = ob;
                bi = oi;
            }
        }
        int piv = __shfl_sync(0xffffffffu, bi, 0);
        double d = a[piv * n + col];
        if (!isfinite(d) || fabs(d) < 1e-28) ok = false;
        if (piv != col)
            for (int c = lane; c < n; c += 32) {
                double t = a[col * n + c];
                a[col * n + c] = a[piv * n + c];
                a[piv * n + c] = t;
                t = inv[col * n + c];
                inv[col * n + c] = inv[piv * n + c];
                inv[piv * n + c] = t;
            }
        __syncwarp();
        for (int c = lane; c < n; c += 32) {
            a[col * n + c] /= d;
            inv[col * n + c] /= d;
        }
        __syncwarp();
        for (int i = lane; i < n; i += 32)
            if (i != col) {
                double fct = a[i * n + col];
                for (int c = 0; c < n; ++c) {
                    a[i * n + c] -= fct * a[col * n + c];
                    inv[i * n + c] -= fct * inv[col * n + c];
                }
            }
        __syncwarp();
    }
    return ok;
}

// C = A (r x m) B (m x c), row-major, lanes over outputs
__device__ void warp_matmul(const double* A, const double* B, double* C, int r, int m, int c, int lane) {
    for (int z = lane; z < r * c; z += 32) {
        int i = z / c, j = z % c;
        double s = 0;
        for (int l = 0; l < m; ++l) s += A[i * m + l] * B[l * c + j];
        C[z] = s;
    }
    __syncwarp();
}

__device__ __forceinline__ void vertex(const double* V, int idx, double ax, double ay, double& x, double& y) {
    if (idx == APEX) {
        x = ax;
        y = ay;
    } else {
        x = V[2 * idx];
        y = V[2 * idx + 1];
    }
}

}  // namespace

// map a computational point of triangle T of a cell (shared by setup and error kernels)
__device__ static void map_cell_point(const CellGeo& g, Pt& s, int arc_local, double ax, double ay, double bx, double by,
                               double cx, double cy) {
    if (g.geom == VG_GEOM_SINE) {
        map_sine(s, g.eps);
    } else if (g.geom == VG_GEOM_ARCS && arc_local != NO_ARC) {
        const double* C = g.arc + 3 * g.gedge_base[arc_local];
        map_arc(s, cx, cy, ax, ay, bx, by, C[0], C[1], C[2]);
    } else {
        map_identity(s);
    }
}

// generate the volume points of one cell into VP (VPS doubles per point:
// x, y, w, t00, t01, t11, det, det * f, X, Y, j00, j01, j10, j11); returns the number of points
constexpr int VPS = 14;
__device__ static int cell_volume_points(const SetupArgs& a, int cell, const double* V, int ne, double apx, double apy,
                                  double* VP, int lane, bool with_data) {
    const int t0 = a.triptr[cell], nt = a.triptr[cell + 1] - t0, npt = nt * a.nqp;
    CellGeo g{a.geom, a.eps, a.arc, a.gedges + a.cptr[cell]};
    for (int i = lane; i < npt; i += 32) {
        int t = i / a.nqp, r = i % a.nqp;
        TriIdx T = a.tris[t0 + t];
        double x0, y0, x1, y1, x2, y2;
        vertex(V, T.a, apx, apy, x0, y0);
        vertex(V, T.b, apx, apy, x1, y1);
        vertex(V, T.c, apx, apy, x2, y2);
        double J = fabs((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0));
        Pt s;
        s.x = x0 + (x1 - x0) * c_tri[3 * r] + (x2 - x0) * c_tri[3 * r + 1];
        s.y = y0 + (y1 - y0) * c_tri[3 * r] + (y2 - y0) * c_tri[3 * r + 1];
        s.w = c_tri[3 * r + 2] * J;
        // the arc triangle is (apex, a, b) with the chord a->b
        map_cell_point(g, s, T.arc, x1, y1, x2, y2, x0, y0);
        if (!(s.det > 0) || !isfinite(s.det)) set_status(a.status, ST_JACOBIAN, cell);
        double* o = VP + VPS * i;
        o[0] = s.x;
        o[1] = s.y;
        o[2] = s.w;
        o[3] = (s.j00 * s.j00 + s.j10 * s.j10) / s.det;
        o[4] = (s.j00 * s.j01 + s.j10 * s.j11) / s.det;
        o[5] = (s.j01 * s.j01 + s.j11 * s.j11) / s.det;
        o[6] = s.det;
        o[7] = with_data ? s.det * prob_f(a.problem, s.X, s.Y) : 0.0;
        o[8] = s.X;
        o[9] = s.Y;
        o[10] = s.j00;
        o[11] = s.j01;
        o[12] = s.j10;
        o[13] = s.j11;
    }
    return npt;
}

__global__ void setup_kernel(SetupArgs a, CellClass cls, SmemLayout L) {
    extern __shared__ double sm[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int jc = blockIdx.x * wpb + wid;
    if (jc >= cls.count) return;
    double* S = sm + size_t(wid) * L.per_warp;
    const int cell = cls.cells[jc];
    const int slot = a.cell_slot[cell];
    const Piece b = a.pieces[slot / PIECE];
    const int j = slot % PIECE;
    const int ne = cls.ne, n = cls.n, k = a.k, q = a.q, p = a.p, ng = a.ng, ngr = a.ngrad, ed = (k + 1) * ne;
    const int m = PIECE;
    const Frame f{a.cx[cell], a.cy[cell], a.diam[cell]};
    const int vb = a.cptr[cell];
    double* V = S + L.vert;
    if (lane < ne) {
        int g = a.cnodes[vb + lane];
        V[2 * lane] = a.xy[2 * g];
        V[2 * lane + 1] = a.xy[2 * g + 1];
    }
    __syncwarp();
    double apx = 0, apy = 0;
    for (int i = 0; i < ne; ++i) {
        apx += V[2 * i];
        apy += V[2 * i + 1];
    }
    apx /= ne;
    apy /= ne;
    double area = 0;
    {
        const int t0 = a.triptr[cell], nt = a.triptr[cell + 1] - t0;
        for (int t = 0; t < nt; ++t) {
            TriIdx T = a.tris[t0 + t];
            double x0, y0, x1, y1, x2, y2;
            vertex(V, T.a, apx, apy, x0, y0);
            vertex(V, T.b, apx, apy, x1, y1);
            vertex(V, T.c, apx, apy, x2, y2);
            area += 0.5 * fabs((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0));
        }
    }
    // ---- quadrature points
    double* VP = S + L.vol;
    const int npt = cell_volume_points(a, cell, V, ne, apx, apy, VP, lane, true);
    double* EP = S + L.edge;  // x, y, w, p_D, u.n per edge point
    CellGeo geo{a.geom, a.eps, a.arc, a.gedges + vb};
    for (int i = lane; i < ne * ng; i += 32) {
        int e = i / ng, l = i % ng;
        double x0 = V[2 * e], y0 = V[2 * e + 1], x1 = V[2 * ((e + 1) % ne)], y1 = V[2 * ((e + 1) % ne) + 1];
        double dx = x1 - x0, dy = y1 - y0, len = sqrt(dx * dx + dy * dy);
        Pt s;
        s.x = x0 + dx * (c_gl[2 * l] + 1.0) / 2.0;
        s.y = y0 + dy * (c_gl[2 * l] + 1.0) / 2.0;
        s.w = c_gl[2 * l + 1] * len / 2.0;
        bool is_arc = a.geom == VG_GEOM_ARCS && a.arc[3 * a.gedges[vb + e] + 2] > 0;
        map_cell_point(geo, s, is_arc ? e : NO_ARC, x0, y0, x1, y1, apx, apy);
        if (!(s.det > 0) || !isfinite(s.det)) set_status(a.status, ST_JACOBIAN, cell);
        double ux, uy;
        prob_u(a.problem, s.X, s.Y, ux, uy);
        double hx = s.j11 * ux - s.j01 * uy, hy = -s.j10 * ux + s.j00 * uy;
        double* o = EP + 5 * i;
        o[0] = s.x;
        o[1] = s.y;
        o[2] = s.w;
        o[3] = prob_dirichlet(a.problem, s.X, s.Y);
        o[4] = (hx * dy - hy * dx) / len;  // outward normal (dy, -dx) / len
    }
    __syncwarp();
    // ---- integrals: G, AG, H, H*, L, rhs, int T, D
    double* G = S + L.G;
    double* AG = S + L.AG;
    double* H = S + L.H;
    double* Hs = S + L.Hs;
    double* Lm = S + L.Lm;
    double* Rh = S + L.Rh;
    double* Ts = S + L.Ts;
    double* D = S + L.D;
    const int nG = p * p, nH = q * q, nHs = ngr * q, nD = n * p;
    const int total = 2 * nG + nH + nHs + 2 * q + 4 + nD;
    for (int z = lane; z < total; z += 32) {
        int y = z;
        double s = 0;
        if (y < nG) {
            int i = y / p, jj = y % p;
            for (int l = 0; l < npt; ++l) {
                const double* P = VP + VPS * l;
                double ax, ay, bx, by;
                hdiv(i, k, f, P[0], P[1], ax, ay);
                hdiv(jj, k, f, P[0], P[1], bx, by);
                s += P[2] * (ax * bx + ay * by);
            }
            G[y] = s;
            continue;
        }
        y -= nG;
        if (y < nG) {
            int i = y / p, jj = y % p;
            for (int l = 0; l < npt; ++l) {
                const double* P = VP + VPS * l;
                double ax, ay, bx, by;
                hdiv(i, k, f, P[0], P[1], ax, ay);
                hdiv(jj, k, f, P[0], P[1], bx, by);
                s += P[2] * (ax * (P[3] * bx + P[4] * by) + ay * (P[4] * bx + P[5] * by));
            }
            AG[y] = s;
            continue;
        }
        y -= nG;
        if (y < nH) {
            int i = y / q, jj = y % q;
            for (int l = 0; l < npt; ++l) {
                const double* P = VP + VPS * l;
                s += P[2] * mono(i, f, P[0], P[1]) * mono(jj, f, P[0], P[1]);
            }
            H[y] = s;
            continue;
        }
        y -= nH;
        if (y < nHs) {
            int i = y / q, jj = y % q;
            for (int l = 0; l < npt; ++l) {
                const double* P = VP + VPS * l;
                s += P[2] * mono(i + 1, f, P[0], P[1]) * mono(jj, f, P[0], P[1]);
            }
            Hs[y] = s;
            continue;
        }
        y -= nHs;
        if (y < q) {
            for (int l = 0; l < npt; ++l) {
                const double* P = VP + VPS * l;
                s += P[2] * P[6] * mono(y, f, P[0], P[1]);
            }
            Lm[y] = s;
            continue;
        }
        y -= q;
        if (y < q) {
            for (int l = 0; l < npt; ++l) {
                const double* P = VP + VPS * l;
                s += P[2] * P[7] * mono(y, f, P[0], P[1]);
            }
            Rh[y] = s;
            continue;
        }
        y -= q;
        if (y < 4) {
            int c = y == 0 ? 3 : y == 3 ? 5 : 4;
            for (int l = 0; l < npt; ++l) s += VP[VPS * l + 2] * VP[VPS * l + c];
            Ts[y] = s;
            continue;
        }
        y -= 4;
        {
            int i = y / p, jj = y % p;
            if (i < ed) {
                int e = i % ne, r = i / ne;
                double x0 = V[2 * e], y0 = V[2 * e + 1], x1 = V[2 * ((e + 1) % ne)], y1 = V[2 * ((e + 1) % ne) + 1];
                double ex = x1 - x0, ey = y1 - y0, len = sqrt(ex * ex + ey * ey);
                double nx = ey / len, ny = -ex / len, mx = 0.5 * (x0 + x1), my = 0.5 * (y0 + y1);
                for (int l = 0; l < ng; ++l) {
                    const double* P = EP + 5 * (e * ng + l);
                    double vx, vy;
                    hdiv(jj, k, f, P[0], P[1], vx, vy);
                    double t = ((P[0] - mx) * ex / len + (P[1] - my) * ey / len) / len;
                    s += P[2] * (vx * nx + vy * ny) * ipow(t, r);
                }
            } else {
                int aa = i - ed;
                int idx = aa < q - 1 ? aa : aa - (q - 1) + ngr;
                for (int l = 0; l < npt; ++l) {
                    const double* P = VP + VPS * l;
                    double vx, vy, gx, gy;
                    hdiv(jj, k, f, P[0], P[1], vx, vy);
                    hdiv(idx, k, f, P[0], P[1], gx, gy);
                    s += P[2] * (vx * gx + vy * gy);
                }
            }
            D[y] = s;
        }
    }
    // ---- W (q x n): edge restriction coefficients, -1 on the gradient interior moments
    double* W = S + L.W;
    for (int z = lane; z < q * n; z += 32) {
        int r = z / n, col = z % n;
        double w = 0;
        if (col < ed) {
            int e = col % ne;
            w = edge_coeff(r, col / ne, f, V[2 * e], V[2 * e + 1], V[2 * ((e + 1) % ne)], V[2 * ((e + 1) % ne) + 1]);
        } else if (col - ed == r - 1 && r > 0) {
            w = -1.0;
        }
        W[z] = w;
    }
    // normalised edge mass int_{-1/2}^{1/2} t^{r+s} dt
    double* Me = S + L.Me;
    const int kk = k + 1;
    for (int z = lane; z < kk * kk; z += 32) Me[z] = moment(z / kk + z % kk);
    __syncwarp();
    // ---- inverses
    double* Hi = S + L.Hi;
    double* Gi = S + L.Gi;
    double* Mi = S + L.Mi;
    bool ok = warp_inverse(H, Hi, q, lane);
    ok = warp_inverse(Me, Mi, kk, lane) && ok;
    ok = warp_inverse(G, Gi, p, lane) && ok;
    if (!ok && lane == 0) set_status(a.status, ST_SINGULAR, cell);
    // ---- H^{-1} W, B, P
    double* HW = S + L.HW;
    warp_matmul(Hi, W, HW, q, q, n, lane);
    double* B = S + L.B;
    for (int z = lane; z < p * n; z += 32) {
        int i = z / n, col = z % n;
        double v = 0;
        if (i < ngr) {
            for (int r = 0; r < q; ++r) v -= Hs[i * q + r] * HW[r * n + col];
            if (col < ed) {
                int deg = col / ne, e = col % ne;
                double x0 = V[2 * e], y0 = V[2 * e + 1], x1 = V[2 * ((e + 1) % ne)], y1 = V[2 * ((e + 1) % ne) + 1];
                for (int s2 = 0; s2 <= k + 1; ++s2) {
                    double coef = edge_coeff(i + 1, s2, f, x0, y0, x1, y1);
                    for (int t = 0; t < kk; ++t) v += coef * moment(s2 + t) * Mi[t * kk + deg];
                }
            }
        } else if (col == ed + (q - 1) + (i - ngr)) {
            v = 1.0;
        }
        B[z] = v;
    }
    __syncwarp();
    double* P = S + L.P;
    warp_matmul(Gi, B, P, p, p, n, lane);
    // C = I - D P (n x n), AGP = AG P (p x n)
    double* C = S + L.C;
    for (int z = lane; z < n * n; z += 32) {
        int i = z / n, c = z % n;
        double v = (i == c) ? 1.0 : 0.0;
        for (int aa = 0; aa < p; ++aa) v -= D[i * p + aa] * P[aa * n + c];
        C[z] = v;
    }
    double* AGP = S + L.AGP;
    warp_matmul(AG, P, AGP, p, p, n, lane);
    const double alpha = sqrt(Ts[0] * Ts[0] + Ts[1] * Ts[1] + Ts[2] * Ts[2] + Ts[3] * Ts[3]) / area;
    const double et = exp(-a.theta[cell]);
    // ---- packed upper-triangular A (row-major over i <= j), slot-major in the bucket
    const int npk = n * (n + 1) / 2;
    for (int z = lane; z < npk; z += 32) {
        // decode z -> (i, jj) with jj >= i: row i holds n - i entries
        int i = 0, rem = z;
        while (rem >= n - i) {
            rem -= n - i;
            ++i;
        }
        int jj = i + rem;
        double v = 0;
        for (int aa = 0; aa < p; ++aa) v += P[aa * n + i] * AGP[aa * n + jj];
        double st = 0;
        for (int l = 0; l < n; ++l) st += C[l * n + i] * C[l * n + jj];
        v += alpha * st;
        long long o = b.a_off + (long long)z * m + j;
        a.A0[o] = v;
        a.A64[o] = et * v;
        a.A32[o] = float(et * v);
    }
    if (k >= 1)
        for (int z = lane; z < q * n; z += 32) {
            long long o = b.w_off + (long long)z * m + j;
            a.W64[o] = W[z];
            a.W32[o] = float(W[z]);
        }
    for (int z = lane; z < p * n; z += 32) a.P[b.p_off + (long long)z * m + j] = P[z];
    for (int z = lane; z < q * n; z += 32) a.HW[b.hw_off + (long long)z * m + j] = HW[z];
    if (lane < q) {
        a.L[(long long)cell * q + lane] = Lm[lane];
        a.L32[(long long)cell * q + lane] = float(Lm[lane]);
        a.rhs[a.nf + (long long)cell * q + lane] = Rh[lane];
    }
    if (lane == 0) a.alpha[cell] = alpha;
    // ---- boundary moments: essential normal-flux values (BC_FLUX) or Dirichlet loads (BC_PRESSURE)
    for (int i = lane; i < ed; i += 32) {
        int e = i % ne, r = i / ne;
        int ge = a.gedges[vb + e];
        if (a.eocc[ge] != 1) continue;
        int g = a.map[b.map_off + (long long)i * m + j];  // boundary dofs carry the + orientation
        double x0 = V[2 * e], y0 = V[2 * e + 1], x1 = V[2 * ((e + 1) % ne)], y1 = V[2 * ((e + 1) % ne) + 1];
        double ex = x1 - x0, ey = y1 - y0, len = sqrt(ex * ex + ey * ey), mx = 0.5 * (x0 + x1), my = 0.5 * (y0 + y1);
        if (a.bc == VG_BC_FLUX) {
            double s = 0;
            for (int l = 0; l < ng; ++l) {
                const double* Pp = EP + 5 * (e * ng + l);
                double t = ((Pp[0] - mx) * ex / len + (Pp[1] - my) * ey / len) / len;
                s += Pp[2] * Pp[4] * ipow(t, r);
            }
            a.bval[g] = s;
            a.mask[g] = 1;
        } else {
            double s = 0;
            for (int s2 = 0; s2 < kk; ++s2) {
                double mom = 0;
                for (int l = 0; l < ng; ++l) {
                    const double* Pp = EP + 5 * (e * ng + l);
                    double t = ((Pp[0] - mx) * ex / len + (Pp[1] - my) * ey / len) / len;
                    mom += Pp[2] * Pp[3] * ipow(t, s2);
                }
                s += Mi[r * kk + s2] * mom;
            }
            a.rhs[g] = -s / len;
        }
    }
}

SmemLayout make_layout(int k, int ne, int nqp, int ng) {
    SmemLayout L{};
    int q = dimP(k), p = p_of(k), ngr = ngrad_of(k), n = (k + 1) * ne + internal_of(k), kk = k + 1;
    int o = 0;
    auto take = [&](int cnt) {
        int r = o;
        o += cnt;
        return r;
    };
    L.vert = take(2 * MAX_NE);
    L.vol = take(VPS * ne * nqp);
    L.edge = take(5 * ne * ng);
    L.G = take(p * p);
    L.AG = take(p * p);
    L.Gi = take(p * p);
    L.H = take(q * q);
    L.Hi = take(q * q);
    L.Hs = take(ngr * q);
    L.Lm = take(q);
    L.Rh = take(q);
    L.Ts = take(4);
    L.Me = take(kk * kk);
    L.Mi = take(kk * kk);
    L.D = take(n * p);
    L.W = take(q * n);
    L.HW = take(q * n);
    L.B = take(p * n);
    L.P = take(p * n);
    L.AGP = take(p * n);
    L.C = take(n * n);
    L.per_warp = o;
    return L;
}

void launch_setup(const SetupArgs& a, const CellClass& b, int nqp, cudaStream_t s) {
    SmemLayout L = make_layout(a.k, b.ne, nqp, a.ng);
    size_t per = size_t(L.per_warp) * sizeof(double);
    int wpb = int(std::max<size_t>(1, std::min<size_t>(4, (96u << 10) / per)));
    size_t smem = per * wpb;
    if (smem > (227u << 10)) throw Error(VG_EINVAL, "cell too large for the setup kernel's shared memory");
    VG_CUDA(cudaFuncSetAttribute(setup_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int blocks = (b.count + wpb - 1) / wpb;
    setup_kernel<<<blocks, 32 * wpb, smem, s>>>(a, b, L);
    VG_CUDA(cudaGetLastError());
}

// Six error figures per cell (MixedGpu::errors, vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:387-462):
// projected flux P u, divergence H^{-1} W u, errors against the built-in exact solution on the
// computational and the physical domain, and the physical pressure mass. One warp per cell.
__global__ void error_kernel(SetupArgs a, CellClass cls, SmemLayout L, const double* x, double* per_cell) {
    extern __shared__ double sm[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int jc = blockIdx.x * wpb + wid;
    if (jc >= cls.count) return;
    double* S = sm + size_t(wid) * L.per_warp;
    const int cell = cls.cells[jc];
    const int slot = a.cell_slot[cell];
    const Piece b = a.pieces[slot / PIECE];
    const int j = slot % PIECE;
    const int ne = cls.ne, n = cls.n, k = a.k, q = a.q, p = a.p, m = PIECE;
    const Frame f{a.cx[cell], a.cy[cell], a.diam[cell]};
    const int vb = a.cptr[cell];
    double* V = S + L.vert;
    if (lane < ne) {
        int g = a.cnodes[vb + lane];
        V[2 * lane] = a.xy[2 * g];
        V[2 * lane + 1] = a.xy[2 * g + 1];
    }
    double* U = S + L.D;   // local flux dofs (n)
    double* Z = S + L.P;   // projected flux coefficients (p), divergence (q), pressure (q)
    for (int i = lane; i < n; i += 32) {
        int g = a.map[b.map_off + (long long)i * m + j];
        U[i] = g < 0 ? -x[~g] : x[g];
    }
    __syncwarp();
    double apx = 0, apy = 0;
    for (int i = 0; i < ne; ++i) {
        apx += V[2 * i];
        apy += V[2 * i + 1];
    }
    apx /= ne;
    apy /= ne;
    for (int z = lane; z < p + 2 * q; z += 32) {
        double s = 0;
        if (z < p) {
            for (int i = 0; i < n; ++i) s += a.P[b.p_off + (long long)(z * n + i) * m + j] * U[i];
        } else if (z < p + q) {
            for (int i = 0; i < n; ++i) s += a.HW[b.hw_off + (long long)((z - p) * n + i) * m + j] * U[i];
        } else {
            s = x[a.nf + (long long)cell * q + (z - p - q)];
        }
        Z[z] = s;
    }
    double* VP = S + L.vol;
    const int npt = cell_volume_points(a, cell, V, ne, apx, apy, VP, lane, false);
    __syncwarp();
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int l = lane; l < npt; l += 32) {
        const double* P = VP + VPS * l;
        double xx = P[0], yy = P[1], w = P[2], det = P[6], X = P[8], Y = P[9];
        double j00 = P[10], j01 = P[11], j10 = P[12], j11 = P[13];
        double cn = 0, dn = 0, ux = 0, uy = 0;
        for (int r = 0; r < q; ++r) {
            double mv = mono(r, f, xx, yy);
            cn += Z[p + q + r] * mv;
            dn += Z[p + r] * mv;
        }
        for (int aa = 0; aa < p; ++aa) {
            double vx, vy;
            hdiv(aa, k, f, xx, yy, vx, vy);
            ux += Z[aa] * vx;
            uy += Z[aa] * vy;
        }
        double pe = prob_p(a.problem, X, Y), rx, ry;
        prob_u(a.problem, X, Y, rx, ry);
        double dc = cn - pe;
        double dx = ux - (j11 * rx - j01 * ry), dy = uy - (-j10 * rx + j00 * ry);
        acc[0] += w * dc * dc;
        acc[1] += w * (dx * dx + dy * dy);
        acc[2] += w * det * dc * dc;
        double px = (j00 * ux + j01 * uy) / det - rx, py = (j10 * ux + j11 * uy) / det - ry;
        acc[3] += w * det * (px * px + py * py);
        double dd = dn / det - prob_f(a.problem, X, Y);
        acc[4] += w * det * dd * dd;
        acc[5] += w * det * cn;
    }
    for (int c = 0; c < 6; ++c) {
        double v = acc[c];
        for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) per_cell[6LL * cell + c] = v;
    }
}

// fixed-order sum over cells: one block, each thread sums a contiguous chunk, then a tree
__global__ void error_sum_kernel(const double* per_cell, int nc, double* out) {
    __shared__ double sh[6][256];
    int t = threadIdx.x;
    long long chunk = (nc + 255) / 256, lo = t * chunk, hi = min((long long)nc, lo + chunk);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (long long c = lo; c < hi; ++c)
        for (int j = 0; j < 6; ++j) acc[j] += per_cell[6 * c + j];
    for (int j = 0; j < 6; ++j) sh[j][t] = acc[j];
    __syncthreads();
    for (int s = 128; s; s >>= 1) {
        if (t < s)
            for (int j = 0; j < 6; ++j) sh[j][t] += sh[j][t + s];
        __syncthreads();
    }
    if (t < 6) out[t] = t == 5 ? sh[5][0] : sqrt(fmax(sh[t][0], 0.0));
}

void launch_errors(const SetupArgs& a, const CellClass& b, int nqp, const double* x, double* per_cell, cudaStream_t s) {
    SmemLayout L = make_layout(a.k, b.ne, nqp, a.ng);
    size_t per = size_t(L.per_warp) * sizeof(double);
    int wpb = int(std::max<size_t>(1, std::min<size_t>(4, (96u << 10) / per)));
    size_t smem = per * wpb;
    VG_CUDA(cudaFuncSetAttribute(error_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    error_kernel<<<(b.count + wpb - 1) / wpb, 32 * wpb, smem, s>>>(a, b, L, x, per_cell);
    VG_CUDA(cudaGetLastError());
}

void launch_error_sum(const double* per_cell, int nc, double* out, cudaStream_t s) {
    error_sum_kernel<<<1, 256, 0, s>>>(per_cell, nc, out);
    VG_CUDA(cudaGetLastError());
}

}  // namespace vg
