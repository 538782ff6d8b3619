// hp_overset_common.h -- the part of the overset table build shared by the
// host builder (hp_overset.cpp) and the device builder (hp_overset_gpu.cu):
// argument checks, fringe marking, the field cells of each block and the
// parameters of the uniform grid over each block's field tets.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/hydraphase.h"

namespace hp_ov {

struct GridParams {
    double lo[3] = {0, 0, 0}, h = 1.0;
    int n[3] = {1, 1, 1};
};

// Grid cell index along axis d of coordinate v (clamped to the grid).
#ifdef __CUDACC__
__host__ __device__
#endif
inline int grid_index(const GridParams& g, int d, double v) {
    double t = floor((v - g.lo[d]) / g.h);
    if (!(t >= 0.0)) return 0;
    return t >= g.n[d] - 1 ? g.n[d] - 1 : (int)t;
}

#ifdef __CUDACC__
#define HP_OV_HD __host__ __device__
#else
#define HP_OV_HD
#endif

HP_OV_HD inline double det3(double A11, double A21, double A31, double A12, double A22, double A32, double A13,
                            double A23, double A33) {
    return A11 * (A22 * A33 - A23 * A32) - A21 * (A12 * A33 - A13 * A32) + A31 * (A12 * A23 - A13 * A22);
}
// Fortran MIN of finite values
HP_OV_HD inline double mn2(double a, double b) { return (b < a || a != a) ? b : a; }

// Barycentric coordinates of x in the tet p0..p3; returns the (scaled)
// volume, 0 for a degenerate tet (lam untouched).  Both builders compile
// this without contraction, so they agree bit for bit.
HP_OV_HD inline double bary(const double p0[3], const double p1[3], const double p2[3], const double p3[3],
                            const double x[3], double lam[4]) {
    double a[3], b[3], c[3], d[3];
    for (int k = 0; k < 3; k++) {
        a[k] = p1[k] - p0[k]; b[k] = p2[k] - p0[k]; c[k] = p3[k] - p0[k]; d[k] = x[k] - p0[k];
    }
    double v = det3(a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]);
    if (v == 0.0) return 0.0;
    double l1 = det3(d[0], d[1], d[2], b[0], b[1], b[2], c[0], c[1], c[2]) / v;
    double l2 = det3(a[0], a[1], a[2], d[0], d[1], d[2], c[0], c[1], c[2]) / v;
    double l3 = det3(a[0], a[1], a[2], b[0], b[1], b[2], d[0], d[1], d[2]) / v;
    lam[0] = 1.0 - l1 - l2 - l3; lam[1] = l1; lam[2] = l2; lam[3] = l3;
    return v;
}

// --- hole cut ---------------------------------------------------------------
// Squared distance from p to the segment u-v and to the triangle a, b, c, and
// whether the ray from p towards +x crosses the triangle (projected edge
// functions taken from the lexicographically lower end of each edge, zeros
// resolved as if p moved by (0, eps, eps^2)).  Compiled without contraction
// on the host and the device, so both builders decide every cell alike.
HP_OV_HD inline double hc_dot(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

HP_OV_HD inline void hc_cross3(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

HP_OV_HD inline double seg_dist2(const double p[3], const double u[3], const double v[3]) {
    double w[3], d[3];
    for (int k = 0; k < 3; k++) { w[k] = v[k] - u[k]; d[k] = p[k] - u[k]; }
    const double ww = hc_dot(w, w), t = hc_dot(d, w);
    if (t <= 0.0 || ww == 0.0) return hc_dot(d, d);
    if (t >= ww) {
        const double q[3] = {p[0] - v[0], p[1] - v[1], p[2] - v[2]};
        return hc_dot(q, q);
    }
    const double s = t / ww;
    double q[3];
    for (int k = 0; k < 3; k++) q[k] = d[k] - s * w[k];
    return hc_dot(q, q);
}

HP_OV_HD inline double tri_dist2(const double p[3], const double a[3], const double b[3], const double c[3]) {
    double ab[3], ac[3], n[3];
    for (int k = 0; k < 3; k++) { ab[k] = b[k] - a[k]; ac[k] = c[k] - a[k]; }
    hc_cross3(ab, ac, n);
    const double nn = hc_dot(n, n);
    if (nn > 0.0) {
        const double* V[3] = {a, b, c};
        bool in = true;
        for (int q = 0; q < 3 && in; q++) {
            const double *u = V[q], *v = V[(q + 1) % 3];
            double e[3], d[3], x[3];
            for (int k = 0; k < 3; k++) { e[k] = v[k] - u[k]; d[k] = p[k] - u[k]; }
            hc_cross3(e, d, x);
            in = hc_dot(n, x) >= 0.0;
        }
        if (in) {
            const double ap[3] = {p[0] - a[0], p[1] - a[1], p[2] - a[2]};
            const double h = hc_dot(ap, n);
            return h * h / nn;
        }
    }
    const double d0 = seg_dist2(p, a, b), d1 = seg_dist2(p, b, c), d2 = seg_dist2(p, c, a);
    return d0 < d1 ? (d0 < d2 ? d0 : d2) : (d1 < d2 ? d1 : d2);
}

HP_OV_HD inline int edge_sign(const double u[3], const double v[3], const double p[3], double* val) {
    const bool swap = u[1] > v[1] || (u[1] == v[1] && u[2] > v[2]);
    const double *s = swap ? v : u, *t = swap ? u : v;
    const double dy = t[1] - s[1], dz = t[2] - s[2];
    if (dy == 0.0 && dz == 0.0) { *val = 0.0; return 0; }
    const double e = dy * (p[2] - s[2]) - dz * (p[1] - s[1]);
    const int sg = e > 0.0 ? 1 : e < 0.0 ? -1 : (dz != 0.0 ? (dz > 0.0 ? -1 : 1) : 1);
    *val = swap ? -e : e;
    return swap ? -sg : sg;
}

HP_OV_HD inline int ray_crosses(const double p[3], const double a[3], const double b[3], const double c[3]) {
    double ea, eb, ec;
    const int sa = edge_sign(b, c, p, &ea), sb = edge_sign(c, a, p, &eb), sc = edge_sign(a, b, p, &ec);
    if (sa == 0 || sb == 0 || sc == 0 || sa != sb || sb != sc) return 0;
    const double den = ea + eb + ec;
    const double xh = den != 0.0 ? (ea * a[0] + eb * b[0] + ec * c[0]) / den : a[0];
    return xh > p[0];
}

// Wall triangles and their two search grids: g3 bins each triangle by its
// bounding box grown by r3 (distance test), g2 by its (y, z) box grown by a
// rounding allowance (ray test; g2.n[0] = 1).  A point outside lo/hi of a
// grid cannot pass that grid's test.  Plain pointers, so kernels take it by
// value.
struct HoleView {
    const double* tri;      // [ntri][9]: a, b, c
    GridParams g3, g2;
    double lo3[3], hi3[3], lo2[3], hi2[3];
    const int *start3, *items3, *start2, *items2;
    double m2;              // margin^2
};

HP_OV_HD inline size_t hole_cell(const GridParams& g, const double p[3]) {
    return ((size_t)grid_index(g, 0, p[0]) * g.n[1] + grid_index(g, 1, p[1])) * g.n[2] + grid_index(g, 2, p[2]);
}

// 1 if a background cell with centroid p is a hole: within the margin of a
// wall triangle, or enclosed by the wall (odd number of crossings).
HP_OV_HD inline int hole_test(const HoleView& H, const double p[3]) {
    if (p[0] >= H.lo3[0] && p[0] <= H.hi3[0] && p[1] >= H.lo3[1] && p[1] <= H.hi3[1] && p[2] >= H.lo3[2] &&
        p[2] <= H.hi3[2]) {
        const size_t c = hole_cell(H.g3, p);
        for (int it = H.start3[c]; it < H.start3[c + 1]; it++) {
            const double* T = H.tri + 9 * (size_t)H.items3[it];
            if (tri_dist2(p, T, T + 3, T + 6) <= H.m2) return 1;
        }
    }
    int par = 0;
    if (p[1] >= H.lo2[1] && p[1] <= H.hi2[1] && p[2] >= H.lo2[2] && p[2] <= H.hi2[2]) {
        const size_t c = hole_cell(H.g2, p);
        for (int it = H.start2[c]; it < H.start2[c + 1]; it++) {
            const double* T = H.tri + 9 * (size_t)H.items2[it];
            par ^= ray_crosses(p, T, T + 3, T + 6);
        }
    }
    return par;
}

struct HolePrep {
    std::vector<double> tri;
    std::vector<int> start3, items3, start2, items2;
    HoleView v;             // points into the vectors above
};

// Checks the arguments, collects the wall triangles and bins them; HP_OK, or
// HP_E_ARG (also when the component has no face of type wall_type).
int prepare_hole(const hp_mesh* mesh, const int32_t* block, int32_t wall_type, double margin, HolePrep& H);

struct Prep {
    std::vector<int> fr;          // fringe cells, 1-based, ascending
    std::vector<int> field[2];    // field cells of each block, 1-based, ascending
    GridParams grid[2];
};

// Checks the arguments, marks the fringe (iblank_out) and fills P; HP_OK or
// HP_E_ARG.
int prepare(const hp_mesh* mesh, const int32_t* block, int32_t layers, int32_t outer_type, int32_t* iblank_out,
            Prep& P);

}  // namespace hp_ov
