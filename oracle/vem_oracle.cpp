// ORACLE — test infrastructure only. Nothing in the product links, loads or calls this file.
//
// A plain FP64 CPU restatement of the reference's curved mixed-VEM Darcy path, used as the
// checker for the CUDA library and as the timed CPU baseline ("reference algorithm, restated"):
//
//   * mesh post-processing of the reference reader (CCW reorder, centroid / area / diameter with
//     the bounding-box rule for 4-gons, global edges by sorting, edge occurrence):
//       vem/CurvedVEM_Darcy_gpu/mesh/straight_mesh.cpp:467-664
//   * ear-clipping triangulation: vem/CurvedVEM_Darcy_gpu/mesh/polygon_triangulator.cpp:56-150
//     (decisions taken in cell-scaled coordinates, see ear_clip below)
//   * quadrature tables: vem/CurvedVEM_Darcy_gpu/core/gauss_quadrature.cpp:74-305, 36-point Duffy
//     rule of vem/CurvedVEM_Darcy_gpu/src/mesh_pack.cpp:110-124
//   * scaled monomials and the H(div) basis: vem/CurvedVEM_Darcy_gpu/lib/polynomial_basis.cpp:95-293
//   * element matrices D, G, H, H*, W, H_edge, H*_edge, B, Pi: vem/CurvedVEM_Darcy/solver/HdivMatrix.cpp:94-652
//   * G_Kappa, alpha, K_ac, K_as, Lagrange vector, RHS, direction adjustment, local-to-global
//     numbering and assembly: vem/CurvedVEM_Darcy/solver/DarcySolver.cpp:182-500,1133-1509
//   * essential normal-flux boundary values: vem/CurvedVEM_Darcy/solver/DarcySolver.cpp:502-663
//   * L2 errors (computational domain): vem/CurvedVEM_Darcy/solver/DarcySolver.cpp:942-1131, and the
//     physical-domain / divergence / mass figures of vem/CurvedVEM_Darcy_gpu/src/equation_gpu.cu:387-462
//   * GMRES(100) + ILU(0), rtol 1e-10: vem/CurvedVEM_Darcy/core/petsc_utils.cpp:144-211
//
// Extensions that the reference does not have (same mathematics, new data): per-cell log
// permeability theta (T = e^{-theta} J^T J / det J), exact circular-arc boundary edges through a
// per-cell blending map, Dirichlet pressure loads -int p_D v.n on boundary edge moments.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double PI = 3.14159265358979323846;

// ---------------------------------------------------------------------------------------------
// quadrature tables (restated from gauss_quadrature.cpp)
// ---------------------------------------------------------------------------------------------
struct P1 { double x, w; };
struct P2 { double x, y, w; };

std::vector<P1> gauss_legendre(int n) {
    std::vector<P1> p;
    auto sym = [&](std::initializer_list<std::pair<double, double>> half, bool centre, double wc) {
        std::vector<std::pair<double, double>> h(half);
        for (auto& q : h) p.push_back({-q.first, q.second});
        if (centre) p.push_back({0.0, wc});
        for (auto it = h.rbegin(); it != h.rend(); ++it) p.push_back({it->first, it->second});
    };
    switch (n) {
    case 1: p.push_back({0.0, 2.0}); break;
    case 2: sym({{0.5773502691896257645091488, 1.0}}, false, 0); break;
    case 3: sym({{0.7745966692414833770358531, 0.5555555555555556}}, true, 0.8888888888888889); break;
    case 4: sym({{0.8611363115940526, 0.3478548451374539}, {0.3399810435848563, 0.6521451548625461}}, false, 0); break;
    case 5:
        sym({{0.9061798459386640, 0.2369268850561891}, {0.5384693101056831, 0.4786286704993665}}, true,
            0.5688888888888889);
        break;
    case 6:
        sym({{0.9324695142031520, 0.1713244923791703}, {0.6612093864662645, 0.3607615730481386},
             {0.2386191860831969, 0.4679139345726910}},
            false, 0);
        break;
    case 7:
        sym({{0.9491079123427585, 0.1294849661688697}, {0.7415311855993944, 0.2797053914892767},
             {0.4058451513773972, 0.3818300505051190}},
            true, 0.4179591836734694);
        break;
    case 8:
        sym({{0.9602898564975362, 0.1012285362903763}, {0.7966664774136267, 0.2223810344533745},
             {0.5255324099163290, 0.3137066458778873}, {0.1834346424956498, 0.3626837833783620}},
            false, 0);
        break;
    case 9:
        sym({{0.9681602395076261, 0.0812743883615744}, {0.8360311073266358, 0.1806481606948574},
             {0.6133714327005904, 0.2606106964029355}, {0.3242534234038089, 0.3123470770400028}},
            true, 0.3302393550012598);
        break;
    case 10:
        sym({{0.9739065285171717, 0.0666713443086881}, {0.8650633666889845, 0.1494513491505806},
             {0.6794095682990244, 0.2190863625159820}, {0.4333953941292472, 0.2692667193099964},
             {0.1488743389816312, 0.2955242247147529}},
            false, 0);
        break;
    default: throw std::invalid_argument("Gauss-Legendre order must be 1..10");
    }
    return p;
}

std::vector<P2> triangle_rule(int n) {
    std::vector<P2> p;
    switch (n) {
    case 1: p.push_back({1.0 / 3.0, 1.0 / 3.0, 0.5}); break;
    case 3:
        p.push_back({0.5, 0.0, 1.0 / 6.0});
        p.push_back({0.5, 0.5, 1.0 / 6.0});
        p.push_back({0.0, 0.5, 1.0 / 6.0});
        break;
    case 4: {
        double s = 1.0 / std::sqrt(3.0);
        p.push_back({(1 + s) / 2, (1 - s) * (1 + s) / 4, (1 - s) / 8.0});
        p.push_back({(1 + s) / 2, (1 - s) * (1 - s) / 4, (1 - s) / 8.0});
        p.push_back({(1 - s) / 2, (1 + s) * (1 + s) / 4, (1 + s) / 8.0});
        p.push_back({(1 - s) / 2, (1 + s) * (1 - s) / 4, (1 + s) / 8.0});
        break;
    }
    case 7: {
        p.push_back({1.0 / 3.0, 1.0 / 3.0, 0.1125});
        double a = 0.797426985353087, b = 0.101286507323456, w1 = 0.0629695902724135;
        p.push_back({a, b, w1});
        p.push_back({b, a, w1});
        p.push_back({b, b, w1});
        double c = 0.059715871789770, d = 0.470142064105115, w2 = 0.0661970763907399;
        p.push_back({c, d, w2});
        p.push_back({d, c, w2});
        p.push_back({d, d, w2});
        break;
    }
    case 9: {
        double s = std::sqrt(3.0 / 5.0);
        p.push_back({0.5, 0.25, 64.0 / 81.0 * 1.0 / 8.0});
        p.push_back({(1 + s) / 2, (1 - s) * (1 + s) / 4, 100.0 / 324.0 * (1 - s) / 8.0});
        p.push_back({(1 + s) / 2, (1 - s) * (1 - s) / 4, 100.0 / 324.0 * (1 - s) / 8.0});
        p.push_back({(1 - s) / 2, (1 + s) * (1 + s) / 4, 100.0 / 324.0 * (1 + s) / 8.0});
        p.push_back({(1 - s) / 2, (1 + s) * (1 - s) / 4, 100.0 / 324.0 * (1 + s) / 8.0});
        p.push_back({0.5, (1 + s) / 4, 40.0 / 81.0 * 1.0 / 8.0});
        p.push_back({0.5, (1 - s) / 4, 40.0 / 81.0 * 1.0 / 8.0});
        p.push_back({(1 + s) / 2, (1 - s) / 4, 40.0 / 81.0 * (1 - s) / 8.0});
        p.push_back({(1 - s) / 2, (1 + s) / 4, 40.0 / 81.0 * (1 + s) / 8.0});
        break;
    }
    case 12: {
        const double a = 0.5611400349004341, b = 0.2194299825497830, wa = 0.1713331241529811 * 0.5;
        const double c = 0.0397240717755698, d = 0.4801379641122151, wc = 0.0807310895930309 * 0.5;
        const double e = 0.0193717243612408, f = 0.1416190159239682, g = 0.8390092597147911,
                     we = 0.0406345597936607 * 0.5;
        p.push_back({a, b, wa});
        p.push_back({b, b, wa});
        p.push_back({b, a, wa});
        p.push_back({c, d, wc});
        p.push_back({d, d, wc});
        p.push_back({d, c, wc});
        p.push_back({e, f, we});
        p.push_back({f, g, we});
        p.push_back({g, e, we});
        p.push_back({f, e, we});
        p.push_back({e, g, we});
        p.push_back({g, f, we});
        break;
    }
    default: throw std::invalid_argument("triangle rule must be 1, 3, 4, 7, 9, 12 or 36");
    }
    return p;
}

// ---------------------------------------------------------------------------------------------
// scaled monomials, H(div) basis, edge restriction coefficients (polynomial_basis.cpp)
// ---------------------------------------------------------------------------------------------
inline int dimP(int k) { return k < 0 ? 0 : (k + 1) * (k + 2) / 2; }

inline void multi_index(int index, int& a, int& b) {
    int degree = 0, preceding = 0;
    while (index >= preceding + degree + 1) {
        preceding += degree + 1;
        ++degree;
    }
    int offset = index - preceding;
    a = degree - offset;
    b = offset;
}

inline double ipow(double x, int n) {
    double r = 1.0;
    for (int i = 0; i < n; ++i) r *= x;
    return r;
}

struct Frame { double cx, cy, h; };

inline double mono(int i, const Frame& f, double x, double y) {
    int a, b;
    multi_index(i, a, b);
    return ipow((x - f.cx) / f.h, a) * ipow((y - f.cy) / f.h, b);
}

inline void hdiv(int i, int k, const Frame& f, double x, double y, double& vx, double& vy) {
    double X = (x - f.cx) / f.h, Y = (y - f.cy) / f.h;
    int ngrad = dimP(k + 1) - 1;
    if (i < ngrad) {
        int a, b;
        multi_index(i + 1, a, b);
        vx = a > 0 ? a * ipow(X, a - 1) * ipow(Y, b) / f.h : 0.0;
        vy = b > 0 ? b * ipow(X, a) * ipow(Y, b - 1) / f.h : 0.0;
        return;
    }
    int c = i - ngrad, degree = 1;
    while (c >= degree) {
        c -= degree;
        ++degree;
    }
    int yb = c, xa = degree - yb;
    double factor = double(yb + 1) / xa;
    vx = -factor * ipow(X, xa - 1) * ipow(Y, yb + 1);
    vy = ipow(X, xa) * ipow(Y, yb);
}

double binom(int n, int k) {
    double r = 1;
    for (int j = 1; j <= k; ++j) r = r * (n - k + j) / j;
    return r;
}

// coefficients c_d of m_i restricted to the straight edge p0->p1 as a polynomial in
// t = ((x - mid).tau)/L in [-1/2, 1/2]  (getEdgeBasisCoeffs)
std::vector<double> edge_coeffs(int i, int kmax, const Frame& f, double x0, double y0, double x1, double y1) {
    double ex = x1 - x0, ey = y1 - y0, L = std::sqrt(ex * ex + ey * ey);
    int a, b;
    multi_index(i, a, b);
    std::vector<double> c(std::max(kmax + 1, a + b + 1), 0.0);
    double mx = 0.5 * (x0 + x1), my = 0.5 * (y0 + y1), tx = ex / L, ty = ey / L, ox = mx - f.cx, oy = my - f.cy;
    for (int u = 0; u <= a; ++u)
        for (int v = 0; v <= b; ++v)
            c[u + v] += binom(a, u) * binom(b, v) * ipow(ox, a - u) * ipow(oy, b - v) * ipow(tx, u) * ipow(ty, v);
    for (int d = 0; d <= a + b; ++d) c[d] *= ipow(L, d) / ipow(f.h, a + b);
    c.resize(kmax + 1);
    return c;
}

inline double edge_t(double x0, double y0, double x1, double y1, double x, double y) {
    double ex = x1 - x0, ey = y1 - y0, L = std::sqrt(ex * ex + ey * ey);
    double mx = 0.5 * (x0 + x1), my = 0.5 * (y0 + y1);
    return ((x - mx) * ex / L + (y - my) * ey / L) / L;
}

// ---------------------------------------------------------------------------------------------
// small dense linear algebra
// ---------------------------------------------------------------------------------------------
using Mat = std::vector<double>;  // row-major

Mat inverse(Mat a, int n) {
    Mat inv(n * n, 0.0);
    for (int i = 0; i < n; ++i) inv[i * n + i] = 1.0;
    for (int k = 0; k < n; ++k) {
        int piv = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(a[i * n + k]) > std::fabs(a[piv * n + k])) piv = i;
        double d = a[piv * n + k];
        if (!std::isfinite(d) || std::fabs(d) < 1e-300) throw std::runtime_error("singular local matrix");
        if (piv != k)
            for (int j = 0; j < n; ++j) {
                std::swap(a[k * n + j], a[piv * n + j]);
                std::swap(inv[k * n + j], inv[piv * n + j]);
            }
        for (int j = 0; j < n; ++j) {
            a[k * n + j] /= d;
            inv[k * n + j] /= d;
        }
        for (int i = 0; i < n; ++i)
            if (i != k) {
                double f = a[i * n + k];
                if (f == 0.0) continue;
                for (int j = 0; j < n; ++j) {
                    a[i * n + j] -= f * a[k * n + j];
                    inv[i * n + j] -= f * inv[k * n + j];
                }
            }
    }
    return inv;
}

Mat matmul(const Mat& a, const Mat& b, int n, int m, int p) {  // (n x m) (m x p)
    Mat c(n * p, 0.0);
    for (int i = 0; i < n; ++i)
        for (int l = 0; l < m; ++l) {
            double v = a[i * m + l];
            if (v == 0.0) continue;
            for (int j = 0; j < p; ++j) c[i * p + j] += v * b[l * p + j];
        }
    return c;
}

Mat transpose(const Mat& a, int n, int m) {
    Mat t(m * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) t[j * n + i] = a[i * m + j];
    return t;
}

// ---------------------------------------------------------------------------------------------
// mesh (StraightMeshData post-processing of the reference reader)
// ---------------------------------------------------------------------------------------------
struct Mesh {
    int nn = 0, nc = 0, ne = 0;
    std::vector<double> xy;
    std::vector<int> cptr, cnodes, nper;
    std::vector<double> cx, cy, area, diam;
    std::vector<int> gedges, eend, eocc;
};

void build_mesh(Mesh& m, int nn, const double* xy, int nc, const int* ptr, const int* nodes) {
    m.nn = nn;
    m.nc = nc;
    m.xy.assign(xy, xy + 2 * nn);
    m.cptr.assign(ptr, ptr + nc + 1);
    m.cnodes.assign(nodes, nodes + ptr[nc]);
    m.nper.resize(nc);
    for (int c = 0; c < nc; ++c) {
        int n = ptr[c + 1] - ptr[c];
        if (n < 3) throw std::invalid_argument("cell with fewer than 3 vertices");
        m.nper[c] = n;
        double s = 0;  // signed area (polygon_signed_area) -> CCW
        for (int i = 0; i < n; ++i) {
            int a = m.cnodes[ptr[c] + i], b = m.cnodes[ptr[c] + (i + 1) % n];
            if (a < 0 || a >= nn) throw std::invalid_argument("node index out of range");
            s += m.xy[2 * a] * m.xy[2 * b + 1] - m.xy[2 * b] * m.xy[2 * a + 1];
        }
        if (s / 2.0 < 0) std::reverse(m.cnodes.begin() + ptr[c], m.cnodes.begin() + ptr[c + 1]);
    }
    m.cx.assign(nc, 0);
    m.cy.assign(nc, 0);
    m.area.assign(nc, 0);
    m.diam.assign(nc, 0);
    for (int c = 0; c < nc; ++c) {
        int n = m.nper[c];
        std::vector<double> x(n), y(n);
        for (int i = 0; i < n; ++i) {
            int g = m.cnodes[m.cptr[c] + i];
            x[i] = m.xy[2 * g];
            y[i] = m.xy[2 * g + 1];
        }
        if (n == 4) {  // bounding-box centre for quadrilaterals (straight_mesh.cpp:536-547)
            double x0 = *std::min_element(x.begin(), x.end()), x1 = *std::max_element(x.begin(), x.end());
            double y0 = *std::min_element(y.begin(), y.end()), y1 = *std::max_element(y.begin(), y.end());
            m.cx[c] = (x0 + x1) / 2.0;
            m.cy[c] = (y0 + y1) / 2.0;
            m.area[c] = (x1 - x0) * (y1 - y0);
        } else {
            double sx = 0, sy = 0;
            for (int i = 0; i < n; ++i) {
                sx += x[i];
                sy += y[i];
            }
            m.cx[c] = sx / n;
            m.cy[c] = sy / n;
            double a = 0;
            for (int i = 0; i < n; ++i) a += x[i] * y[(i + 1) % n] - x[(i + 1) % n] * y[i];
            m.area[c] = std::fabs(a) / 2.0;
        }
        double d = 0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) d = std::max(d, std::sqrt((x[i] - x[j]) * (x[i] - x[j]) + (y[i] - y[j]) * (y[i] - y[j])));
        m.diam[c] = d;
    }
    // global edges: sort (min,max) pairs, unique in sorted order
    std::vector<std::pair<std::pair<int, int>, int>> all;
    all.reserve(m.cnodes.size());
    for (int c = 0; c < nc; ++c)
        for (int j = 0; j < m.nper[c]; ++j) {
            int a = m.cnodes[m.cptr[c] + j], b = m.cnodes[m.cptr[c] + (j + 1) % m.nper[c]];
            all.push_back({{std::min(a, b), std::max(a, b)}, int(all.size())});
        }
    std::vector<std::pair<std::pair<int, int>, int>> sorted = all;
    std::sort(sorted.begin(), sorted.end());
    m.gedges.assign(all.size(), -1);
    m.eend.clear();
    int count = 0;
    for (size_t i = 0; i < sorted.size(); ++i) {
        if (i == 0 || sorted[i].first != sorted[i - 1].first) {
            m.eend.push_back(sorted[i].first.first);
            m.eend.push_back(sorted[i].first.second);
            ++count;
        }
        m.gedges[sorted[i].second] = count - 1;
    }
    m.ne = count;
    m.eocc.assign(count, 0);
    for (int e : m.gedges) m.eocc[e]++;
}

// ---------------------------------------------------------------------------------------------
// triangulation
// ---------------------------------------------------------------------------------------------
struct Tri {
    double v[6];
    int arc = -1;  // local edge index whose arc blending map acts on this triangle, -1 = unmapped
};

// Ear clipping of polygon_triangulator.cpp:56-150. The ear and inside decisions are taken on
// cell-scaled coordinates ((x - x_D)/h_D): the reference's absolute tolerances (1e-8 on the
// cross product, 1e-6 on triangle areas) then act on O(1) numbers at every mesh size, giving the
// reference's choice on the reference meshes and a valid choice on 1e6-cell meshes, where the
// absolute 1e-6 area tolerance would accept every vertex as "inside".
std::vector<Tri> ear_clip(const std::vector<double>& x, const std::vector<double>& y, const Frame& f) {
    int n = int(x.size());
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::vector<double> u(n), v(n);
    for (int i = 0; i < n; ++i) {
        u[i] = (x[i] - f.cx) / f.h;
        v[i] = (y[i] - f.cy) / f.h;
    }
    auto inside = [&](int p, int a, int b, int c) {
        double px = u[p], py = v[p], ax = u[a], ay = v[a], bx = u[b], by = v[b], cx = u[c], cy = v[c];
        double t = 0.5 * std::fabs((bx - ax) * (cy - ay) - (cx - ax) * (by - ay));
        double a1 = 0.5 * std::fabs((ax - px) * (by - py) - (bx - px) * (ay - py));
        double a2 = 0.5 * std::fabs((bx - px) * (cy - py) - (cx - px) * (by - py));
        double a3 = 0.5 * std::fabs((cx - px) * (ay - py) - (ax - px) * (cy - py));
        return std::fabs((a1 + a2 + a3) - t) < 1e-6;
    };
    std::vector<Tri> out;
    auto push = [&](int a, int b, int c) {
        Tri t;
        t.v[0] = x[a]; t.v[1] = y[a]; t.v[2] = x[b]; t.v[3] = y[b]; t.v[4] = x[c]; t.v[5] = y[c];
        out.push_back(t);
    };
    while (int(idx.size()) > 3) {
        int r = int(idx.size());
        bool found = false;
        for (int i = 0; i < r; ++i) {
            int pv = idx[(i - 1 + r) % r], cu = idx[i], nx = idx[(i + 1) % r];
            double cross = (u[nx] - u[cu]) * (v[pv] - v[cu]) - (u[pv] - u[cu]) * (v[nx] - v[cu]);
            if (cross <= 1e-8) continue;
            bool ear = true;
            for (int j = 0; j < r && ear; ++j) {
                int q = idx[j];
                if (q == pv || q == cu || q == nx) continue;
                if (inside(q, pv, cu, nx)) ear = false;
            }
            if (!ear) continue;
            push(pv, cu, nx);
            idx.erase(idx.begin() + i);
            found = true;
            break;
        }
        if (!found) throw std::runtime_error("no valid ear found for polygon");
    }
    push(idx[0], idx[1], idx[2]);
    return out;
}

// ---------------------------------------------------------------------------------------------
// geometry maps and problem data
// ---------------------------------------------------------------------------------------------
enum { GEOM_IDENTITY = 0, GEOM_SINE = 1, GEOM_ARCS = 2 };
enum { PROB_SINCOS = 1, PROB_SINSIN = 2, PROB_ANNULUS = 3 };
enum { BC_FLUX = 0, BC_PRESSURE = 1 };

struct Sample { double x, y, w, X, Y, j00, j01, j10, j11, det; };

// points of one straight triangle: reference rule (map_triangle) or the 36-point Duffy rule
std::vector<Sample> tri_points(const double* v, int nq, const std::vector<P2>& tr, const std::vector<P1>& g6) {
    std::vector<Sample> out;
    double J = std::fabs((v[2] - v[0]) * (v[5] - v[1]) - (v[4] - v[0]) * (v[3] - v[1]));
    if (nq != 36) {
        for (auto& r : tr) {
            Sample s{};
            s.x = v[0] + (v[2] - v[0]) * r.x + (v[4] - v[0]) * r.y;
            s.y = v[1] + (v[3] - v[1]) * r.x + (v[5] - v[1]) * r.y;
            s.w = r.w * J;
            out.push_back(s);
        }
        return out;
    }
    for (auto& a : g6)
        for (auto& b : g6) {
            double u = (a.x + 1) / 2, wa = a.w / 2, ub = (b.x + 1) / 2, wb = b.w / 2;
            double w = (1 - u) * ub;
            Sample s{};
            s.x = v[0] + u * (v[2] - v[0]) + w * (v[4] - v[0]);
            s.y = v[1] + u * (v[3] - v[1]) + w * (v[5] - v[1]);
            s.w = wa * wb * (1 - u) * J;
            out.push_back(s);
        }
    return out;
}

struct Arc { double cx, cy, r; };

struct Problem {
    int kind;
    double p(double X, double Y) const {
        switch (kind) {
        case PROB_SINCOS: return std::sin(PI * X) * std::cos(PI * Y);
        case PROB_SINSIN: return std::sin(PI * X) * std::sin(PI * Y);
        default: return std::log(std::sqrt(X * X + Y * Y)) / std::log(0.3);
        }
    }
    void u(double X, double Y, double& ux, double& uy) const {  // u = -grad p (K = I)
        switch (kind) {
        case PROB_SINCOS:
            ux = -PI * std::cos(PI * X) * std::cos(PI * Y);
            uy = PI * std::sin(PI * X) * std::sin(PI * Y);
            return;
        case PROB_SINSIN:
            ux = -PI * std::cos(PI * X) * std::sin(PI * Y);
            uy = -PI * std::sin(PI * X) * std::cos(PI * Y);
            return;
        default: {
            double r2 = X * X + Y * Y, c = 1.0 / std::log(0.3);
            ux = -c * X / r2;
            uy = -c * Y / r2;
        }
        }
    }
    double f(double X, double Y) const {
        if (kind == PROB_ANNULUS) return 0.0;
        return 2.0 * PI * PI * p(X, Y);
    }
    double dirichlet(double X, double Y) const {
        if (kind == PROB_ANNULUS) return std::sqrt(X * X + Y * Y) < 0.65 ? 1.0 : 0.0;
        return p(X, Y);
    }
};

// ---------------------------------------------------------------------------------------------
// the oracle state
// ---------------------------------------------------------------------------------------------
struct Oracle {
    Mesh m;
    int k, nq, ng, geom, problem, bc;
    double eps = 0;
    std::vector<Arc> arcs;  // per global edge, r = 0 -> straight
    std::vector<double> theta;
    int q, p, ngrad, internal, nf, np, N;
    // per cell local data
    std::vector<int> n;                    // local flux dofs
    std::vector<std::vector<Sample>> vol;  // volume samples
    std::vector<std::vector<Sample>> edg;  // edge samples, ng per local edge
    std::vector<Mat> D, G, H, Hs, W, B, P, Pd, AG, A, Mm, Hi;
    std::vector<double> alpha, areaT;
    std::vector<std::vector<double>> L, rhs, dir;
    std::vector<std::vector<int>> gdofs;
    std::vector<std::vector<double>> bvals;  // essential flux values per local dof (NaN = not boundary)
    std::vector<std::vector<double>> dload;  // Dirichlet load per local flux dof
    Problem prob;

    Frame frame(int c) const { return {m.cx[c], m.cy[c], m.diam[c]}; }

    void map_point(int c, const Tri* t, Sample& s) const {
        s.X = s.x; s.Y = s.y; s.j00 = 1; s.j01 = 0; s.j10 = 0; s.j11 = 1; s.det = 1;
        if (geom == GEOM_SINE) {
            s.X = s.x + eps * std::sin(2 * PI * s.y);
            s.Y = s.y + eps * std::sin(2 * PI * s.x);
            s.j01 = eps * 2 * PI * std::cos(2 * PI * s.y);
            s.j10 = eps * 2 * PI * std::cos(2 * PI * s.x);
            s.det = 1.0 - s.j01 * s.j10;
        } else if (geom == GEOM_ARCS && t && t->arc >= 0) {
            // triangle (c, a, b) with the chord a->b mapped onto the circular arc:
            // x = c + lam (a - c + t e),  F(x) = c + lam (gamma(t) - c),  e = b - a
            double cx = t->v[0], cy = t->v[1], ax = t->v[2], ay = t->v[3], bx = t->v[4], by = t->v[5];
            int ge = m.gedges[m.cptr[c] + t->arc];
            const Arc& A = arcs[ge];
            arc_map(cx, cy, ax, ay, bx, by, A, s);
        }
    }

    static void arc_map(double cx, double cy, double ax, double ay, double bx, double by, const Arc& A, Sample& s) {
        double ex = bx - ax, ey = by - ay, dx = ax - cx, dy = ay - cy;
        double det0 = dx * ey - dy * ex;
        double rx = s.x - cx, ry = s.y - cy;
        double lam = (rx * ey - ry * ex) / det0, sl = (dx * ry - dy * rx) / det0;
        double t = lam > 0 ? sl / lam : 0.5;
        double ta = std::atan2(ay - A.cy, ax - A.cx), tb = std::atan2(by - A.cy, bx - A.cx);
        double dth = tb - ta;
        while (dth > PI) dth -= 2 * PI;
        while (dth < -PI) dth += 2 * PI;
        double th = ta + t * dth;
        double gx = A.cx + A.r * std::cos(th), gy = A.cy + A.r * std::sin(th);
        double gpx = -A.r * dth * std::sin(th), gpy = A.r * dth * std::cos(th);
        s.X = cx + lam * (gx - cx);
        s.Y = cy + lam * (gy - cy);
        // J = [gamma - c, gamma'] [a - c + t e, e]^{-1}
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

    std::vector<Tri> triangulate(int c) const {
        int ncn = m.nper[c];
        std::vector<double> x(ncn), y(ncn);
        for (int i = 0; i < ncn; ++i) {
            int g = m.cnodes[m.cptr[c] + i];
            x[i] = m.xy[2 * g];
            y[i] = m.xy[2 * g + 1];
        }
        bool curved = false;
        if (geom == GEOM_ARCS)
            for (int j = 0; j < ncn; ++j)
                if (arcs[m.gedges[m.cptr[c] + j]].r > 0) curved = true;
        if (!curved) return ear_clip(x, y, frame(c));
        // cells with an arc edge: fan from the vertex average, one triangle per edge
        double ax = 0, ay = 0;
        for (int i = 0; i < ncn; ++i) {
            ax += x[i];
            ay += y[i];
        }
        ax /= ncn;
        ay /= ncn;
        std::vector<Tri> out;
        for (int j = 0; j < ncn; ++j) {
            Tri t;
            int b = (j + 1) % ncn;
            t.v[0] = ax; t.v[1] = ay; t.v[2] = x[j]; t.v[3] = y[j]; t.v[4] = x[b]; t.v[5] = y[b];
            t.arc = arcs[m.gedges[m.cptr[c] + j]].r > 0 ? j : -1;
            out.push_back(t);
        }
        return out;
    }

    void build() {
        q = dimP(k);
        ngrad = dimP(k + 1) - 1;
        p = ngrad + dimP(k - 1);
        internal = (q - 1) + (q - (k + 1));
        nf = m.ne * (k + 1) + m.nc * internal;
        np = m.nc * q;
        N = nf + np + (bc == BC_FLUX ? 1 : 0);
        prob.kind = problem;
        int nc = m.nc;
        n.resize(nc);
        vol.resize(nc); edg.resize(nc);
        D.resize(nc); G.resize(nc); H.resize(nc); Hs.resize(nc); W.resize(nc); B.resize(nc); P.resize(nc);
        Pd.resize(nc); AG.resize(nc); A.resize(nc); Mm.resize(nc); Hi.resize(nc);
        alpha.resize(nc); areaT.resize(nc); L.resize(nc); rhs.resize(nc); dir.resize(nc); gdofs.resize(nc);
        bvals.resize(nc); dload.resize(nc);
        std::vector<P2> tr;
        if (nq != 36) tr = triangle_rule(nq);
        auto g6 = gauss_legendre(6);
        auto gl = gauss_legendre(ng);
        std::string err;
#pragma omp parallel for schedule(dynamic, 64)
        for (int c = 0; c < nc; ++c) {
            try {
                cell(c, tr, g6, gl);
            } catch (const std::exception& e) {
#pragma omp critical
                err = "cell " + std::to_string(c) + ": " + e.what();
            }
        }
        if (!err.empty()) throw std::runtime_error(err);
    }

    void cell(int c, const std::vector<P2>& tr, const std::vector<P1>& g6, const std::vector<P1>& gl) {
        Frame f = frame(c);
        int ncn = m.nper[c];
        int nn = (k + 1) * ncn + internal;
        int ed = (k + 1) * ncn;
        n[c] = nn;
        // --- volume samples
        auto tris = triangulate(c);
        double at = 0;
        auto& vs = vol[c];
        vs.clear();
        for (auto& t : tris) {
            const double* v = t.v;
            double J = std::fabs((v[2] - v[0]) * (v[5] - v[1]) - (v[4] - v[0]) * (v[3] - v[1]));
            at += 0.5 * J;
            for (auto& s : tri_points(v, nq, tr, g6)) {
                map_point(c, &t, s);
                vs.push_back(s);
            }
        }
        areaT[c] = at;
        for (auto& s : vs)
            if (!(s.det > 0) || !std::isfinite(s.det)) throw std::runtime_error("nonpositive Jacobian");
        // --- edge samples (on the chord, mapped)
        auto& es = edg[c];
        es.clear();
        for (int j = 0; j < ncn; ++j) {
            int a = m.cnodes[m.cptr[c] + j], b = m.cnodes[m.cptr[c] + (j + 1) % ncn];
            double x0 = m.xy[2 * a], y0 = m.xy[2 * a + 1], x1 = m.xy[2 * b], y1 = m.xy[2 * b + 1];
            double dx = x1 - x0, dy = y1 - y0, len = std::sqrt(dx * dx + dy * dy);
            Tri fan;
            const Tri* tp = nullptr;
            if (geom == GEOM_ARCS && arcs[m.gedges[m.cptr[c] + j]].r > 0) {
                for (auto& t : tris)
                    if (t.arc == j) fan = t;
                tp = &fan;
            }
            for (auto& g : gl) {
                Sample s{};
                s.x = x0 + dx * (g.x + 1.0) / 2.0;
                s.y = y0 + dy * (g.x + 1.0) / 2.0;
                s.w = g.w * len / 2.0;
                map_point(c, tp, s);
                if (!(s.det > 0)) throw std::runtime_error("nonpositive boundary Jacobian");
                es.push_back(s);
            }
        }
        // --- D (n x p)
        Mat d(nn * p, 0.0);
        for (int i = 0; i < nn; ++i)
            for (int j = 0; j < p; ++j) {
                double sum = 0;
                if (i < ed) {
                    int e = i % ncn, r = i / ncn;
                    int a = m.cnodes[m.cptr[c] + e], b = m.cnodes[m.cptr[c] + (e + 1) % ncn];
                    double x0 = m.xy[2 * a], y0 = m.xy[2 * a + 1], x1 = m.xy[2 * b], y1 = m.xy[2 * b + 1];
                    double len = std::sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0));
                    double nx = (y1 - y0) / len, ny = -(x1 - x0) / len;
                    for (int l = 0; l < ng; ++l) {
                        const Sample& s = es[e * ng + l];
                        double vx, vy;
                        hdiv(j, k, f, s.x, s.y, vx, vy);
                        sum += s.w * (vx * nx + vy * ny) * ipow(edge_t(x0, y0, x1, y1, s.x, s.y), r);
                    }
                } else {
                    int a = i - ed;
                    int idx = a < q - 1 ? a : a - (q - 1) + ngrad;
                    for (auto& s : vs) {
                        double vx, vy, gx, gy;
                        hdiv(j, k, f, s.x, s.y, vx, vy);
                        hdiv(idx, k, f, s.x, s.y, gx, gy);
                        sum += (vx * gx + vy * gy) * s.w;
                    }
                }
                d[i * p + j] = sum;
            }
        // --- G, H, H*
        Mat g(p * p, 0.0), h(q * q, 0.0), hs(ngrad * q, 0.0);
        for (int i = 0; i < p; ++i)
            for (int j = 0; j < p; ++j) {
                double sum = 0;
                for (auto& s : vs) {
                    double ax, ay, bx, by;
                    hdiv(i, k, f, s.x, s.y, ax, ay);
                    hdiv(j, k, f, s.x, s.y, bx, by);
                    sum += (ax * bx + ay * by) * s.w;
                }
                g[i * p + j] = sum;
            }
        for (int i = 0; i < q; ++i)
            for (int j = 0; j < q; ++j) {
                double sum = 0;
                for (auto& s : vs) sum += mono(i, f, s.x, s.y) * mono(j, f, s.x, s.y) * s.w;
                h[i * q + j] = sum;
            }
        for (int i = 0; i < ngrad; ++i)
            for (int j = 0; j < q; ++j) {
                double sum = 0;
                for (auto& s : vs) sum += mono(i + 1, f, s.x, s.y) * mono(j, f, s.x, s.y) * s.w;
                hs[i * q + j] = sum;
            }
        // --- W (q x n): edge restriction coefficients, -1 on the gradient interior moments
        Mat w(q * nn, 0.0);
        for (int r = 0; r < q; ++r)
            for (int col = 0; col < nn; ++col) {
                double val = 0;
                int gd = col - ed;
                if (gd >= 0 && gd == r - 1) val = -1.0;
                if (col < ed) {
                    int e = col % ncn;
                    int a = m.cnodes[m.cptr[c] + e], b = m.cnodes[m.cptr[c] + (e + 1) % ncn];
                    auto co = edge_coeffs(r, k, f, m.xy[2 * a], m.xy[2 * a + 1], m.xy[2 * b], m.xy[2 * b + 1]);
                    val += co[col / ncn];
                }
                w[r * nn + col] = val;
            }
        // --- B = [B_grad; B_curl],  B_grad = -H* H^{-1} W + sum_e H*_e H_e^{-1} W_e
        Mat hi = inverse(h, q);
        Mat b1 = matmul(hs, matmul(hi, w, q, q, nn), ngrad, q, nn);
        Mat bb(p * nn, 0.0);
        for (int i = 0; i < ngrad * nn; ++i) bb[i] = -b1[i];
        int kk = k + 1;
        for (int e = 0; e < ncn; ++e) {
            int a = m.cnodes[m.cptr[c] + e], b = m.cnodes[m.cptr[c] + (e + 1) % ncn];
            double x0 = m.xy[2 * a], y0 = m.xy[2 * a + 1], x1 = m.xy[2 * b], y1 = m.xy[2 * b + 1];
            Mat he(kk * kk, 0.0), hes(ngrad * kk, 0.0);
            for (int l = 0; l < ng; ++l) {
                const Sample& s = es[e * ng + l];
                double t = edge_t(x0, y0, x1, y1, s.x, s.y);
                for (int r = 0; r < kk; ++r)
                    for (int r2 = 0; r2 < kk; ++r2) he[r * kk + r2] += ipow(t, r) * ipow(t, r2) * s.w;
                for (int i = 0; i < ngrad; ++i)
                    for (int r = 0; r < kk; ++r) hes[i * kk + r] += mono(i + 1, f, s.x, s.y) * ipow(t, r) * s.w;
            }
            // W_edge is the identity on the k+1 edge moments (equals Delta(col % n_e, row) whenever k < n_e)
            Mat tmp = matmul(hes, inverse(he, kk), ngrad, kk, kk);
            for (int r = 0; r < kk; ++r)
                for (int i = 0; i < ngrad; ++i) bb[i * nn + r * ncn + e] += tmp[i * kk + r];
        }
        int ncurl = q - (k + 1);
        for (int r = 0; r < ncurl; ++r) bb[(ngrad + r) * nn + ed + (q - 1) + r] = 1.0;
        Mat pp = matmul(inverse(g, p), bb, p, p, nn);
        Mat pd = matmul(d, pp, nn, p, nn);
        // --- G_Kappa (T = e^{-theta} J^T J / det), alpha, M, L, rhs
        double et = std::exp(-theta[c]);
        Mat ag(p * p, 0.0);
        double T[4] = {0, 0, 0, 0};
        for (auto& s : vs) {
            double t00 = et * (s.j00 * s.j00 + s.j10 * s.j10) / s.det;
            double t01 = et * (s.j00 * s.j01 + s.j10 * s.j11) / s.det;
            double t11 = et * (s.j01 * s.j01 + s.j11 * s.j11) / s.det;
            T[0] += t00 * s.w; T[1] += t01 * s.w; T[2] += t01 * s.w; T[3] += t11 * s.w;
        }
        for (int i = 0; i < p; ++i)
            for (int j = 0; j < p; ++j) {
                double sum = 0;
                for (auto& s : vs) {
                    double t00 = et * (s.j00 * s.j00 + s.j10 * s.j10) / s.det;
                    double t01 = et * (s.j00 * s.j01 + s.j10 * s.j11) / s.det;
                    double t11 = et * (s.j01 * s.j01 + s.j11 * s.j11) / s.det;
                    double ax, ay, bx, by;
                    hdiv(i, k, f, s.x, s.y, ax, ay);
                    hdiv(j, k, f, s.x, s.y, bx, by);
                    sum += (ax * (t00 * bx + t01 * by) + ay * (t01 * bx + t11 * by)) * s.w;
                }
                ag[i * p + j] = sum;
            }
        double al = 0;
        for (int j = 0; j < 4; ++j) al += (T[j] / at) * (T[j] / at);
        al = std::sqrt(al);
        // A = P^T AG P + alpha (I - D P)^T (I - D P)
        Mat kac = matmul(transpose(pp, p, nn), matmul(ag, pp, p, p, nn), nn, p, nn);
        Mat cmp(nn * nn);
        for (int i = 0; i < nn; ++i)
            for (int j = 0; j < nn; ++j) cmp[i * nn + j] = (i == j ? 1.0 : 0.0) - pd[i * nn + j];
        Mat kas = matmul(transpose(cmp, nn, nn), cmp, nn, nn, nn);
        Mat aa(nn * nn);
        for (int i = 0; i < nn * nn; ++i) aa[i] = kac[i] + al * kas[i];
        Mat mm(q * q, 0.0);
        std::vector<double> lv(q, 0.0), rv(q, 0.0);
        for (auto& s : vs)
            for (int r = 0; r < q; ++r) {
                double mr = mono(r, f, s.x, s.y);
                lv[r] += mr * s.det * s.w;
                rv[r] += s.det * prob.f(s.X, s.Y) * mr * s.w;
                for (int r2 = 0; r2 < q; ++r2) mm[r * q + r2] += s.w * s.det * mr * mono(r2, f, s.x, s.y);
            }
        // --- numbering and directions
        std::vector<int> gd(nn + q + (bc == BC_FLUX ? 1 : 0));
        std::vector<double> dr(nn, 1.0);
        for (int r = 0; r <= k; ++r)
            for (int e = 0; e < ncn; ++e) {
                int ge = m.gedges[m.cptr[c] + e];
                gd[r * ncn + e] = r * m.ne + ge;
                if (m.eocc[ge] == 1) continue;
                int a = m.cnodes[m.cptr[c] + e];
                bool rev = a == m.eend[2 * ge + 1];
                if (rev && r % 2 == 0) dr[r * ncn + e] = -1.0;
            }
        for (int j = 0; j < internal; ++j) gd[ed + j] = m.ne * (k + 1) + c * internal + j;
        for (int j = 0; j < q; ++j) gd[nn + j] = nf + c * q + j;
        if (bc == BC_FLUX) gd[nn + q] = nf + np;
        // --- boundary data: essential flux values and Dirichlet loads
        std::vector<double> bv(nn, std::nan("")), dl(nn, 0.0);
        for (int e = 0; e < ncn; ++e) {
            int ge = m.gedges[m.cptr[c] + e];
            if (m.eocc[ge] != 1) continue;
            int a = m.cnodes[m.cptr[c] + e], b = m.cnodes[m.cptr[c] + (e + 1) % ncn];
            double x0 = m.xy[2 * a], y0 = m.xy[2 * a + 1], x1 = m.xy[2 * b], y1 = m.xy[2 * b + 1];
            double len = std::sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0));
            double nx = (y1 - y0) / len, ny = -(x1 - x0) / len;
            Mat he(kk * kk, 0.0);
            std::vector<double> mom(kk, 0.0);
            for (int r = 0; r <= k; ++r) {
                double sum = 0;
                for (int l = 0; l < ng; ++l) {
                    const Sample& s = es[e * ng + l];
                    double ux, uy;
                    prob.u(s.X, s.Y, ux, uy);
                    // computational flux det J * J^{-1} u = adj(J) u
                    double hx = s.j11 * ux - s.j01 * uy, hy = -s.j10 * ux + s.j00 * uy;
                    double t = edge_t(x0, y0, x1, y1, s.x, s.y);
                    sum += (hx * nx + hy * ny) * ipow(t, r) * s.w;
                    mom[r] += prob.dirichlet(s.X, s.Y) * ipow(t, r) * s.w;
                    for (int r2 = 0; r2 <= k; ++r2) he[r * kk + r2] += ipow(t, r) * ipow(t, r2) * s.w;
                }
                bv[r * ncn + e] = sum;
            }
            Mat hei = inverse(he, kk);
            for (int r = 0; r <= k; ++r) {
                double s = 0;
                for (int r2 = 0; r2 <= k; ++r2) s += hei[r * kk + r2] * mom[r2];
                dl[r * ncn + e] = -s;
            }
        }
        D[c] = d; G[c] = g; H[c] = h; Hs[c] = hs; W[c] = w; B[c] = bb; P[c] = pp; Pd[c] = pd;
        AG[c] = ag; A[c] = aa; Mm[c] = mm; Hi[c] = hi;
        alpha[c] = al; L[c] = lv; rhs[c] = rv; dir[c] = dr; gdofs[c] = gd; bvals[c] = bv; dload[c] = dl;
    }

    // global system in the reference sign [A, -W^T, 0; W, 0, L; 0, L^T, 0] (L only for flux BC)
    void assemble(std::vector<int>& rows, std::vector<int>& cols, std::vector<double>& vals, std::vector<double>& b) const {
        rows.clear(); cols.clear(); vals.clear();
        b.assign(N, 0.0);
        for (int c = 0; c < m.nc; ++c) {
            int nn = n[c];
            const auto& gd = gdofs[c];
            const auto& dr = dir[c];
            for (int i = 0; i < nn; ++i)
                for (int j = 0; j < nn; ++j) {
                    rows.push_back(gd[i]); cols.push_back(gd[j]); vals.push_back(dr[i] * dr[j] * A[c][i * nn + j]);
                }
            for (int r = 0; r < q; ++r)
                for (int j = 0; j < nn; ++j) {
                    double v = dr[j] * W[c][r * nn + j];
                    rows.push_back(gd[nn + r]); cols.push_back(gd[j]); vals.push_back(v);
                    rows.push_back(gd[j]); cols.push_back(gd[nn + r]); vals.push_back(-v);
                }
            if (bc == BC_FLUX)
                for (int r = 0; r < q; ++r) {
                    rows.push_back(gd[nn + r]); cols.push_back(N - 1); vals.push_back(L[c][r]);
                    rows.push_back(N - 1); cols.push_back(gd[nn + r]); vals.push_back(L[c][r]);
                }
            for (int r = 0; r < q; ++r) b[gd[nn + r]] += rhs[c][r];
            if (bc == BC_PRESSURE)
                for (int i = 0; i < nn; ++i) b[gd[i]] += dr[i] * dload[c][i];
        }
    }

    // six figures of equation_gpu.cu:387-462 (+ computational errors of DarcySolver.cpp:942-1131)
    void errors(const double* x, double* out) const {
        for (int i = 0; i < 6; ++i) out[i] = 0;
        for (int c = 0; c < m.nc; ++c) {
            Frame f = frame(c);
            int nn = n[c];
            std::vector<double> u(nn);
            for (int i = 0; i < nn; ++i) u[i] = dir[c][i] * x[gdofs[c][i]];
            std::vector<double> z(p, 0.0), dv(q, 0.0), wu(q, 0.0);
            for (int a = 0; a < p; ++a)
                for (int i = 0; i < nn; ++i) z[a] += P[c][a * nn + i] * u[i];
            for (int r = 0; r < q; ++r)
                for (int i = 0; i < nn; ++i) wu[r] += W[c][r * nn + i] * u[i];
            for (int a = 0; a < q; ++a)
                for (int r = 0; r < q; ++r) dv[a] += Hi[c][a * q + r] * wu[r];
            for (auto& s : vol[c]) {
                double cn = 0, dn = 0, ux = 0, uy = 0;
                for (int a = 0; a < q; ++a) {
                    double mv = mono(a, f, s.x, s.y);
                    cn += x[gdofs[c][nn + a]] * mv;
                    dn += dv[a] * mv;
                }
                for (int a = 0; a < p; ++a) {
                    double vx, vy;
                    hdiv(a, k, f, s.x, s.y, vx, vy);
                    ux += z[a] * vx;
                    uy += z[a] * vy;
                }
                double pe = prob.p(s.X, s.Y), rx, ry;
                prob.u(s.X, s.Y, rx, ry);
                double dc = cn - pe;
                double dx = ux - (s.j11 * rx - s.j01 * ry), dy = uy - (-s.j10 * rx + s.j00 * ry);
                out[0] += s.w * dc * dc;
                out[1] += s.w * (dx * dx + dy * dy);
                out[2] += s.w * s.det * dc * dc;
                double px = (s.j00 * ux + s.j01 * uy) / s.det - rx, py = (s.j10 * ux + s.j11 * uy) / s.det - ry;
                out[3] += s.w * s.det * (px * px + py * py);
                double dd = dn / s.det - prob.f(s.X, s.Y);
                out[4] += s.w * s.det * dd * dd;
                out[5] += s.w * s.det * cn;
            }
        }
        for (int i = 0; i < 5; ++i) out[i] = std::sqrt(std::max(out[i], 0.0));
    }
};

// ---------------------------------------------------------------------------------------------
// CSR + ILU(0) + left-preconditioned GMRES(m) with classical Gram-Schmidt (PETSc defaults used by
// solve_linear_system: KSPGMRES, restart 100, PCILU levels 0 natural ordering, preconditioned norm)
// ---------------------------------------------------------------------------------------------
struct Csr {
    int n;
    std::vector<int> ptr, col;
    std::vector<double> val;
};

Csr coo_to_csr(int n, const std::vector<int>& r, const std::vector<int>& c, const std::vector<double>& v, bool diag) {
    std::vector<int64_t> key(r.size());
    std::vector<size_t> order(r.size());
    for (size_t i = 0; i < r.size(); ++i) {
        key[i] = int64_t(r[i]) * n + c[i];
        order[i] = i;
    }
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return key[a] < key[b]; });
    Csr m;
    m.n = n;
    m.ptr.assign(n + 1, 0);
    std::vector<int> rr;
    int64_t last = -1;
    for (size_t t = 0; t < order.size(); ++t) {
        size_t i = order[t];
        if (key[i] != last) {
            rr.push_back(r[i]);
            m.col.push_back(c[i]);
            m.val.push_back(v[i]);
            last = key[i];
        } else
            m.val.back() += v[i];
    }
    if (diag) {  // explicit diagonal slots (DarcySolver::initialize inserts them)
        std::vector<int> r2, c2;
        std::vector<double> v2;
        std::vector<char> has(n, 0);
        for (size_t i = 0; i < rr.size(); ++i)
            if (rr[i] == m.col[i]) has[rr[i]] = 1;
        size_t i = 0;
        for (int row = 0; row < n; ++row) {
            bool done = has[row];
            while (i < rr.size() && rr[i] == row) {
                if (!done && m.col[i] > row) {
                    r2.push_back(row); c2.push_back(row); v2.push_back(0.0);
                    done = true;
                }
                r2.push_back(rr[i]); c2.push_back(m.col[i]); v2.push_back(m.val[i]);
                ++i;
            }
            if (!done) {
                r2.push_back(row); c2.push_back(row); v2.push_back(0.0);
            }
        }
        rr.swap(r2);
        m.col.swap(c2);
        m.val.swap(v2);
    }
    for (int x : rr) m.ptr[x + 1]++;
    for (int i = 0; i < n; ++i) m.ptr[i + 1] += m.ptr[i];
    return m;
}

void spmv(const Csr& a, const double* x, double* y) {
    for (int i = 0; i < a.n; ++i) {
        double s = 0;
        for (int j = a.ptr[i]; j < a.ptr[i + 1]; ++j) s += a.val[j] * x[a.col[j]];
        y[i] = s;
    }
}

struct Ilu0 {
    Csr lu;
    std::vector<int> diag;
    void factor(const Csr& a) {
        lu = a;
        int n = a.n;
        diag.assign(n, -1);
        for (int i = 0; i < n; ++i)
            for (int j = a.ptr[i]; j < a.ptr[i + 1]; ++j)
                if (a.col[j] == i) diag[i] = j;
        std::vector<int> pos(n, -1);
        for (int i = 0; i < n; ++i) {
            for (int j = lu.ptr[i]; j < lu.ptr[i + 1]; ++j) pos[lu.col[j]] = j;
            for (int j = lu.ptr[i]; j < lu.ptr[i + 1]; ++j) {
                int kc = lu.col[j];
                if (kc >= i) break;
                double piv = lu.val[diag[kc]];
                if (piv == 0.0) throw std::runtime_error("zero pivot in ILU(0)");
                double l = lu.val[j] / piv;
                lu.val[j] = l;
                for (int t = diag[kc] + 1; t < lu.ptr[kc + 1]; ++t) {
                    int cc = lu.col[t];
                    if (pos[cc] >= 0) lu.val[pos[cc]] -= l * lu.val[t];
                }
            }
            for (int j = lu.ptr[i]; j < lu.ptr[i + 1]; ++j) pos[lu.col[j]] = -1;
            if (diag[i] < 0 || lu.val[diag[i]] == 0.0) throw std::runtime_error("zero pivot in ILU(0)");
        }
    }
    void solve(const double* b, double* x) const {
        int n = lu.n;
        for (int i = 0; i < n; ++i) {
            double s = b[i];
            for (int j = lu.ptr[i]; j < diag[i]; ++j) s -= lu.val[j] * x[lu.col[j]];
            x[i] = s;
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = x[i];
            for (int j = diag[i] + 1; j < lu.ptr[i + 1]; ++j) s -= lu.val[j] * x[lu.col[j]];
            x[i] = s / lu.val[diag[i]];
        }
    }
};

int gmres_ilu(const Csr& a, const Ilu0& pc, const double* b, double* x, double rtol, double atol, int restart,
              int maxit, double* rnorm_out) {
    int n = a.n;
    std::vector<double> r(n), t(n), w(n);
    std::vector<std::vector<double>> V(restart + 1, std::vector<double>(n));
    std::vector<double> H((restart + 1) * restart), cs(restart), sn(restart), g(restart + 1);
    auto dot = [&](const std::vector<double>& u, const std::vector<double>& v) {
        double s = 0;
        for (int i = 0; i < n; ++i) s += u[i] * v[i];
        return s;
    };
    int it = 0;
    double r0 = -1, rn = 0;
    while (true) {
        spmv(a, x, t.data());
        for (int i = 0; i < n; ++i) w[i] = b[i] - t[i];
        pc.solve(w.data(), r.data());
        double beta = std::sqrt(dot(r, r));
        if (r0 < 0) r0 = beta;
        rn = beta;
        if (beta <= std::max(rtol * r0, atol) || it >= maxit) break;
        for (int i = 0; i < n; ++i) V[0][i] = r[i] / beta;
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        for (; j < restart && it < maxit; ++j, ++it) {
            spmv(a, V[j].data(), t.data());
            pc.solve(t.data(), w.data());
            for (int i = 0; i <= j; ++i) H[i * restart + j] = dot(w, V[i]);  // classical Gram-Schmidt
            for (int i = 0; i <= j; ++i)
                for (int l = 0; l < n; ++l) w[l] -= H[i * restart + j] * V[i][l];
            double hn = std::sqrt(dot(w, w));
            H[(j + 1) * restart + j] = hn;
            for (int i = 0; i < j; ++i) {
                double h1 = H[i * restart + j], h2 = H[(i + 1) * restart + j];
                H[i * restart + j] = cs[i] * h1 + sn[i] * h2;
                H[(i + 1) * restart + j] = -sn[i] * h1 + cs[i] * h2;
            }
            double h1 = H[j * restart + j], h2 = H[(j + 1) * restart + j];
            double den = std::sqrt(h1 * h1 + h2 * h2);
            cs[j] = den > 0 ? h1 / den : 1.0;
            sn[j] = den > 0 ? h2 / den : 0.0;
            H[j * restart + j] = den;
            H[(j + 1) * restart + j] = 0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            if (hn > 0)
                for (int l = 0; l < n; ++l) V[j + 1][l] = w[l] / hn;
            rn = std::fabs(g[j + 1]);
            if (rn <= std::max(rtol * r0, atol)) {
                ++j;
                ++it;
                break;
            }
        }
        std::vector<double> y(j);
        for (int i = j - 1; i >= 0; --i) {
            double s = g[i];
            for (int l = i + 1; l < j; ++l) s -= H[i * restart + l] * y[l];
            y[i] = s / H[i * restart + i];
        }
        for (int i = 0; i < j; ++i)
            for (int l = 0; l < n; ++l) x[l] += y[i] * V[i][l];
        if (rn <= std::max(rtol * r0, atol) || it >= maxit) break;
    }
    if (rnorm_out) *rnorm_out = r0 > 0 ? rn / r0 : 0;
    return it;
}

thread_local std::string g_error;

}  // namespace

extern "C" {

const char* orc_last_error() { return g_error.c_str(); }

// Build the oracle state. cell_ptr/cell_nodes: raw polygons (any orientation, reordered CCW here).
// edge_arc: optional (cx, cy, r) per *raw boundary chord*, given as a lookup by node pair through
// arc_nodes (2 per arc) and arc_data (3 per arc); geometry GEOM_ARCS uses them.
void* orc_create(int nn, const double* xy, int nc, const int* cell_ptr, const int* cell_nodes, int k, int nq, int ng,
                 int geom, double eps, int narcs, const int* arc_nodes, const double* arc_data, int problem, int bc,
                 const double* theta, int threads) {
    try {
        auto* o = new Oracle();
        build_mesh(o->m, nn, xy, nc, cell_ptr, cell_nodes);
        o->k = k; o->nq = nq; o->ng = ng; o->geom = geom; o->eps = eps; o->problem = problem; o->bc = bc;
        o->arcs.assign(o->m.ne, Arc{0, 0, 0});
        if (narcs > 0) {
            std::map<std::pair<int, int>, int> look;
            for (int e = 0; e < o->m.ne; ++e) look[{o->m.eend[2 * e], o->m.eend[2 * e + 1]}] = e;
            for (int a = 0; a < narcs; ++a) {
                int u = arc_nodes[2 * a], v = arc_nodes[2 * a + 1];
                auto it = look.find({std::min(u, v), std::max(u, v)});
                if (it == look.end()) throw std::invalid_argument("arc chord is not a mesh edge");
                o->arcs[it->second] = Arc{arc_data[3 * a], arc_data[3 * a + 1], arc_data[3 * a + 2]};
            }
        }
        o->theta.assign(nc, 0.0);
        if (theta) o->theta.assign(theta, theta + nc);
#ifdef _OPENMP
        if (threads > 0) omp_set_num_threads(threads);
#else
        (void)threads;
#endif
        o->build();
        return o;
    } catch (const std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}

void orc_free(void* h) { delete static_cast<Oracle*>(h); }

// sizes: nc, ne, nf, np, N, q, p, internal, nnodes
void orc_info(void* h, long* out) {
    auto* o = static_cast<Oracle*>(h);
    out[0] = o->m.nc; out[1] = o->m.ne; out[2] = o->nf; out[3] = o->np; out[4] = o->N;
    out[5] = o->q; out[6] = o->p; out[7] = o->internal; out[8] = o->m.nn;
}

// processed mesh arrays (the StraightMeshData of the reference reader)
void orc_mesh(void* h, int* cell_nodes, int* global_edges, int* edge_endpoints, int* edge_occurrence, double* cx,
              double* cy, double* diam, double* area) {
    auto* o = static_cast<Oracle*>(h);
    std::copy(o->m.cnodes.begin(), o->m.cnodes.end(), cell_nodes);
    std::copy(o->m.gedges.begin(), o->m.gedges.end(), global_edges);
    std::copy(o->m.eend.begin(), o->m.eend.end(), edge_endpoints);
    std::copy(o->m.eocc.begin(), o->m.eocc.end(), edge_occurrence);
    std::copy(o->m.cx.begin(), o->m.cx.end(), cx);
    std::copy(o->m.cy.begin(), o->m.cy.end(), cy);
    std::copy(o->m.diam.begin(), o->m.diam.end(), diam);
    std::copy(o->m.area.begin(), o->m.area.end(), area);
}

// assembled full system: returns nnz after coalescing; call with null arrays to query
long orc_csr(void* h, int* ptr, int* col, double* val, double* b) {
    auto* o = static_cast<Oracle*>(h);
    std::vector<int> r, c;
    std::vector<double> v, bb;
    o->assemble(r, c, v, bb);
    Csr m = coo_to_csr(o->N, r, c, v, true);
    if (ptr) {
        std::copy(m.ptr.begin(), m.ptr.end(), ptr);
        std::copy(m.col.begin(), m.col.end(), col);
        std::copy(m.val.begin(), m.val.end(), val);
        std::copy(bb.begin(), bb.end(), b);
    }
    return long(m.val.size());
}

// essential boundary data: mask[N] (1 on boundary flux dofs) and values g[N]
void orc_boundary(void* h, int* mask, double* g) {
    auto* o = static_cast<Oracle*>(h);
    std::fill(mask, mask + o->N, 0);
    std::fill(g, g + o->N, 0.0);
    for (int c = 0; c < o->m.nc; ++c)
        for (int i = 0; i < o->n[c]; ++i)
            if (!std::isnan(o->bvals[c][i])) {
                mask[o->gdofs[c][i]] = 1;
                g[o->gdofs[c][i]] = o->bvals[c][i];
            }
}

// local matrices of one cell: which = 0 A (n x n), 1 W (q x n), 2 P (p x n), 3 D (n x p), 4 G (p x p),
// 5 B (p x n), 6 AG (p x p), 7 M (q x q), 8 alpha (1), 9 L (q), 10 rhs (q), 11 dir (n), 12 gdofs (n+q[+1]),
// 13 dirichlet load (n), 14 area (1), 15 H (q x q), 16 H* (grad x q)
long orc_local(void* h, int c, int which, double* out) {
    auto* o = static_cast<Oracle*>(h);
    auto cp = [&](const std::vector<double>& v) {
        if (out) std::copy(v.begin(), v.end(), out);
        return long(v.size());
    };
    switch (which) {
    case 0: return cp(o->A[c]);
    case 1: return cp(o->W[c]);
    case 2: return cp(o->P[c]);
    case 3: return cp(o->D[c]);
    case 4: return cp(o->G[c]);
    case 5: return cp(o->B[c]);
    case 6: return cp(o->AG[c]);
    case 7: return cp(o->Mm[c]);
    case 8: return cp(std::vector<double>{o->alpha[c]});
    case 9: return cp(o->L[c]);
    case 10: return cp(o->rhs[c]);
    case 11: return cp(o->dir[c]);
    case 12: {
        std::vector<double> g(o->gdofs[c].begin(), o->gdofs[c].end());
        return cp(g);
    }
    case 13: return cp(o->dload[c]);
    case 14: return cp(std::vector<double>{o->areaT[c]});
    case 15: return cp(o->H[c]);
    case 16: return cp(o->Hs[c]);
    }
    return -1;
}

// number of volume / edge samples of a cell and the samples themselves (10 doubles each)
long orc_samples(void* h, int c, int edge, double* out) {
    auto* o = static_cast<Oracle*>(h);
    const auto& v = edge ? o->edg[c] : o->vol[c];
    if (out)
        for (size_t i = 0; i < v.size(); ++i) std::memcpy(out + 10 * i, &v[i], sizeof(Sample));
    return long(v.size());
}

void orc_errors(void* h, const double* x, double* out6) { static_cast<Oracle*>(h)->errors(x, out6); }

// Adjoint contraction per cell, g_E = (S_E lam_E)^T A_E (S_E x_E) over the local flux dofs, S_E the
// orientation signs and lam zero on masked (essential) rows (mask may be null): the CPU FP64
// counterpart of the GPU gradient dJ/dtheta_E = lambda_E^T A_E(theta) u_E (A_E = e^{-theta_E} A_E(0)).
void orc_adjoint_contract(void* h, const double* x, const double* lam, const int* mask, double* g) {
    auto* o = static_cast<Oracle*>(h);
    for (int c = 0; c < o->m.nc; ++c) {
        const int nn = o->n[c];
        const auto& gd = o->gdofs[c];
        const auto& dr = o->dir[c];
        double acc = 0;
        for (int i = 0; i < nn; ++i) {
            const double li = (mask && mask[gd[i]]) ? 0.0 : dr[i] * lam[gd[i]];
            double row = 0;
            for (int j = 0; j < nn; ++j) row += o->A[c][i * nn + j] * dr[j] * x[gd[j]];
            acc += li * row;
        }
        g[c] = acc;
    }
}

// GMRES(restart) + ILU(0) on a CSR matrix (left preconditioning, preconditioned residual norm)
int orc_gmres_ilu(int n, const int* ptr, const int* col, const double* val, const double* b, double* x, double rtol,
                  int restart, int maxit, double* rel_out) {
    try {
        Csr a;
        a.n = n;
        a.ptr.assign(ptr, ptr + n + 1);
        a.col.assign(col, col + ptr[n]);
        a.val.assign(val, val + ptr[n]);
        Ilu0 pc;
        pc.factor(a);
        return gmres_ilu(a, pc, b, x, rtol, 1e-50, restart, maxit, rel_out);
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// The reference CPU solve restated end to end (DarcySolver::solve): element matrices and global
// assembly (timed), essential-BC reduction for BC_FLUX, GMRES(100)+ILU(0) rtol 1e-10 (timed).
// times[0] = element + assembly seconds, times[1] = solve seconds; returns iterations or -1.
int orc_reference_solve(int nn, const double* xy, int nc, const int* cell_ptr, const int* cell_nodes, int k, int nq,
                        int ng, int geom, double eps, int narcs, const int* arc_nodes, const double* arc_data,
                        int problem, int bc, const double* theta, int threads, double rtol, int maxit, double* x,
                        double* times, double* rel_out) {
    try {
        auto t0 = std::chrono::steady_clock::now();
        auto* o = static_cast<Oracle*>(orc_create(nn, xy, nc, cell_ptr, cell_nodes, k, nq, ng, geom, eps, narcs,
                                                  arc_nodes, arc_data, problem, bc, theta, threads));
        if (!o) return -1;
        std::unique_ptr<Oracle> guard(o);
        std::vector<int> r, c;
        std::vector<double> v, b;
        o->assemble(r, c, v, b);
        Csr full = coo_to_csr(o->N, r, c, v, true);
        auto t1 = std::chrono::steady_clock::now();
        int N = o->N;
        std::vector<int> mask(N, 0);
        std::vector<double> g(N, 0.0);
        // essential flux rows only for the flux condition (DarcySolver::solveWithDirichletBC,
        // C/solver/DarcySolver.cpp:665-788); the pressure condition enters as a load on the flux
        // rows and keeps every row
        if (o->bc == BC_FLUX) orc_boundary(o, mask.data(), g.data());
        std::vector<double> kg(N);
        spmv(full, g.data(), kg.data());
        std::vector<int> fidx, inv(N, -1);
        for (int i = 0; i < N; ++i)
            if (!mask[i]) {
                inv[i] = int(fidx.size());
                fidx.push_back(i);
            }
        Csr red;
        red.n = int(fidx.size());
        red.ptr.assign(red.n + 1, 0);
        for (int a = 0; a < red.n; ++a) {
            int i = fidx[a];
            for (int j = full.ptr[i]; j < full.ptr[i + 1]; ++j)
                if (inv[full.col[j]] >= 0) {
                    red.col.push_back(inv[full.col[j]]);
                    red.val.push_back(full.val[j]);
                }
            red.ptr[a + 1] = int(red.col.size());
        }
        std::vector<double> rb(red.n), rx(red.n, 0.0);
        for (int a = 0; a < red.n; ++a) rb[a] = b[fidx[a]] - kg[fidx[a]];
        Ilu0 pc;
        pc.factor(red);
        int it = gmres_ilu(red, pc, rb.data(), rx.data(), rtol, 1e-50, 100, maxit, rel_out);
        auto t2 = std::chrono::steady_clock::now();
        for (int i = 0; i < N; ++i) x[i] = g[i];
        for (int a = 0; a < red.n; ++a) x[fidx[a]] = rx[a];
        times[0] = std::chrono::duration<double>(t1 - t0).count();
        times[1] = std::chrono::duration<double>(t2 - t1).count();
        return it;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// ---- building blocks, for pinning against the reference's compiled modules
long orc_triangles(void* h, int c, double* out) {
    auto* o = static_cast<Oracle*>(h);
    auto t = o->triangulate(c);
    if (out)
        for (size_t i = 0; i < t.size(); ++i) std::memcpy(out + 6 * i, t[i].v, 6 * sizeof(double));
    return long(t.size());
}

int orc_tri_points(const double* v, int nq, double* out) {
    try {
        std::vector<P2> tr;
        if (nq != 36) tr = triangle_rule(nq);
        auto pts = tri_points(v, nq, tr, gauss_legendre(6));
        for (size_t i = 0; i < pts.size(); ++i) {
            out[3 * i] = pts[i].x;
            out[3 * i + 1] = pts[i].y;
            out[3 * i + 2] = pts[i].w;
        }
        return int(pts.size());
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

int orc_line_points(int order, double x1, double y1, double x2, double y2, double* out) {
    auto g = gauss_legendre(order);
    double dx = x2 - x1, dy = y2 - y1, len = std::sqrt(dx * dx + dy * dy);
    for (size_t i = 0; i < g.size(); ++i) {
        out[3 * i] = x1 + dx * (g[i].x + 1.0) / 2.0;
        out[3 * i + 1] = y1 + dy * (g[i].x + 1.0) / 2.0;
        out[3 * i + 2] = g[i].w * len / 2.0;
    }
    return int(g.size());
}

double orc_mono(int idx, double cx, double cy, double h, double x, double y) { return mono(idx, Frame{cx, cy, h}, x, y); }

void orc_hdiv(int k, int idx, double cx, double cy, double h, double x, double y, double* out) {
    hdiv(idx, k, Frame{cx, cy, h}, x, y, out[0], out[1]);
}

void orc_edge_coeffs(int k, int idx, double cx, double cy, double h, double x0, double y0, double x1, double y1,
                     double* out) {
    auto c = edge_coeffs(idx, k, Frame{cx, cy, h}, x0, y0, x1, y1);
    std::copy(c.begin(), c.end(), out);
}

// problem data at a computational point under the sine map: p, u_hat (2), g_hat, X, Y, J (4), det
void orc_problem(int kind, double eps, double xi, double eta, double* out) {
    Oracle o;
    o.geom = GEOM_SINE;
    o.eps = eps;
    Problem pr{kind};
    Sample s{};
    s.x = xi;
    s.y = eta;
    o.map_point(0, nullptr, s);
    double ux, uy;
    pr.u(s.X, s.Y, ux, uy);
    out[0] = pr.p(s.X, s.Y);
    out[1] = s.j11 * ux - s.j01 * uy;
    out[2] = -s.j10 * ux + s.j00 * uy;
    out[3] = s.det * pr.f(s.X, s.Y);
    out[4] = s.X; out[5] = s.Y; out[6] = s.j00; out[7] = s.j01; out[8] = s.j10; out[9] = s.j11; out[10] = s.det;
}

}  // extern "C"
