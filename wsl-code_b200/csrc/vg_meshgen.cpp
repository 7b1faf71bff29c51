// Lloyd relaxation of generator points in a disk or an annulus (host, OpenMP).
//
// The reference builds its CVT polygon meshes with scipy's Voronoi and gmsh
// (vem/gmesh_py/get_gmesh.py:15-77 LloydRelaxation, 487-556 generate_cvt_polygon_mesh). This is
// the same iteration — every generator moves to the centroid of its Voronoi cell clipped to the
// domain — computed cell by cell: the cell of generator i is a box around i clipped by the
// bisectors of its neighbours taken from a uniform bucket grid in order of distance, until no
// remaining neighbour can cut it (security radius twice the farthest vertex), then clipped by the
// domain (tangent half-planes of the circles near the cell, an O(h^2 / r) approximation that only
// affects point placement, not the final mesh topology).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int MAXV = 96;

struct Poly {
    int n = 0;
    double x[MAXV], y[MAXV];
};

// keep the part with a*x + b*y <= c
void clip(Poly& p, double a, double b, double c) {
    Poly o;
    for (int i = 0; i < p.n; ++i) {
        int j = (i + 1) % p.n;
        double si = a * p.x[i] + b * p.y[i] - c, sj = a * p.x[j] + b * p.y[j] - c;
        bool ii = si <= 0, jj = sj <= 0;
        if (ii && o.n < MAXV) {
            o.x[o.n] = p.x[i];
            o.y[o.n++] = p.y[i];
        }
        if (ii != jj && o.n < MAXV) {
            double t = si / (si - sj);
            o.x[o.n] = p.x[i] + t * (p.x[j] - p.x[i]);
            o.y[o.n++] = p.y[i] + t * (p.y[j] - p.y[i]);
        }
    }
    p = o;
}

void centroid(const Poly& p, double& cx, double& cy, double& area) {
    double a = 0, sx = 0, sy = 0;
    for (int i = 0; i < p.n; ++i) {
        int j = (i + 1) % p.n;
        double c = p.x[i] * p.y[j] - p.x[j] * p.y[i];
        a += c;
        sx += (p.x[i] + p.x[j]) * c;
        sy += (p.y[i] + p.y[j]) * c;
    }
    area = 0.5 * a;
    if (std::fabs(a) < 1e-300) {
        cx = cy = 0;
        return;
    }
    cx = sx / (3 * a);
    cy = sy / (3 * a);
}

}  // namespace

extern "C" {

// xy: 2n doubles, updated in place; r_in = 0 for a disk. Returns 0, or -1 on invalid input.
int vg_lloyd(int n, double* xy, double r_in, double r_out, int iterations, int threads) {
    if (n < 4 || !xy || !(r_out > r_in) || r_in < 0) return -1;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    const double pi = 3.14159265358979323846;
    const double area = pi * (r_out * r_out - r_in * r_in);
    const double h = std::sqrt(area / n);
    const double cs = h;  // grid cell size
    const int G = int(std::ceil(2 * r_out / cs)) + 1;
    std::vector<double> nxt(2 * size_t(n));
    std::vector<int> head(size_t(G) * G + 1), idx(n);
    for (int it = 0; it < iterations; ++it) {
        // counting sort into grid cells
        std::fill(head.begin(), head.end(), 0);
        std::vector<int> cell(n);
        for (int i = 0; i < n; ++i) {
            int gx = std::min(G - 1, std::max(0, int((xy[2 * i] + r_out) / cs)));
            int gy = std::min(G - 1, std::max(0, int((xy[2 * i + 1] + r_out) / cs)));
            cell[i] = gy * G + gx;
            head[cell[i] + 1]++;
        }
        for (int c = 0; c < G * G; ++c) head[c + 1] += head[c];
        {
            std::vector<int> fill(head.begin(), head.end() - 1);
            for (int i = 0; i < n; ++i) idx[fill[cell[i]]++] = i;
        }
#pragma omp parallel for schedule(dynamic, 1024)
        for (int i = 0; i < n; ++i) {
            const double px = xy[2 * i], py = xy[2 * i + 1];
            const int gx = cell[i] % G, gy = cell[i] / G;
            Poly P;
            double B = 6 * h;
            P.n = 4;
            P.x[0] = px - B; P.y[0] = py - B;
            P.x[1] = px + B; P.y[1] = py - B;
            P.x[2] = px + B; P.y[2] = py + B;
            P.x[3] = px - B; P.y[3] = py + B;
            std::vector<std::pair<double, int>> cand;
            cand.reserve(64);
            int ring = 2;
            size_t used = 0;
            while (true) {
                cand.clear();
                for (int yy = std::max(0, gy - ring); yy <= std::min(G - 1, gy + ring); ++yy)
                    for (int xx = std::max(0, gx - ring); xx <= std::min(G - 1, gx + ring); ++xx)
                        for (int t = head[yy * G + xx]; t < head[yy * G + xx + 1]; ++t) {
                            int jdx = idx[t];
                            if (jdx == i) continue;
                            double dx = xy[2 * jdx] - px, dy = xy[2 * jdx + 1] - py;
                            cand.push_back({dx * dx + dy * dy, jdx});
                        }
                std::sort(cand.begin(), cand.end());
                bool closed = false;
                for (used = 0; used < cand.size(); ++used) {
                    double rmax = 0;
                    for (int v = 0; v < P.n; ++v)
                        rmax = std::max(rmax, (P.x[v] - px) * (P.x[v] - px) + (P.y[v] - py) * (P.y[v] - py));
                    if (cand[used].first > 4 * rmax) {
                        closed = true;
                        break;
                    }
                    int jdx = cand[used].second;
                    double qx = xy[2 * jdx], qy = xy[2 * jdx + 1];
                    double a = qx - px, b = qy - py;
                    clip(P, a, b, a * 0.5 * (px + qx) + b * 0.5 * (py + qy));
                }
                // the candidate disk of radius ring*cs covers the security radius
                double rmax = 0;
                for (int v = 0; v < P.n; ++v)
                    rmax = std::max(rmax, (P.x[v] - px) * (P.x[v] - px) + (P.y[v] - py) * (P.y[v] - py));
                if (closed || 4 * rmax <= (ring * cs) * (ring * cs) || ring > G) break;
                ring *= 2;
            }
            // domain: tangent half-planes of the outer circle (and the inner one for an annulus)
            double r = std::sqrt(px * px + py * py);
            double th = std::atan2(py, px);
            if (r > r_out - 4 * h)
                for (int s = -3; s <= 3; ++s) {
                    double a = th + s * (h / r_out);
                    clip(P, std::cos(a), std::sin(a), r_out);
                }
            if (r_in > 0 && r < r_in + 4 * h) clip(P, -std::cos(th), -std::sin(th), -r_in);
            double cx, cy, ar;
            centroid(P, cx, cy, ar);
            if (P.n >= 3 && ar > 0 && std::isfinite(cx) && std::isfinite(cy)) {
                nxt[2 * i] = cx;
                nxt[2 * i + 1] = cy;
            } else {
                nxt[2 * i] = px;
                nxt[2 * i + 1] = py;
            }
        }
        std::memcpy(xy, nxt.data(), sizeof(double) * 2 * size_t(n));
    }
    return 0;
}

}  // extern "C"
