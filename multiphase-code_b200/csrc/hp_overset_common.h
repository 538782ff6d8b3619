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
