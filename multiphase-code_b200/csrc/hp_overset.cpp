// hp_overset.cpp -- overset fringe cells and donor tables of a two-block mesh.
//
// New work: the reference only freezes cells with iblank != 1
// (src/sr_RK.F90:31); its hole cutting and donor search come from the TIOGA
// library outside the solver.  Here the two blocks of an overset mesh
// (block 0 background, block 1 component) are one element list, the caller's
// hole cut marks background cells inside the component's body with
// iblank = 0, and this file builds, once per mesh:
//
//   fringe  background field cells next to a hole cell and component field
//           cells next to a ghost of the component's outer boundary type,
//           plus layers - 1 further layers inward; they get iblank = -1 (no
//           RK update of their own);
//   donors  for each fringe cell with centroid x, the lowest-id field cell D
//           of the other block whose tet contains x (barycentric coordinates
//           >= -1e-10), or, if none does, the field cell of that block with
//           the nearest centroid;
//   weights the barycentric coordinates of x in a tet of four centroids
//           among D, its field neighbours and theirs (two rings, face
//           order): of the tets containing x, the one whose vertices are
//           closest to x (least sum of squared distances); if none contains
//           x, the one whose smallest coordinate is largest; or D alone.
//
// Every RK stage then sets a fringe cell's conserved state to
// sum_k w_k cn(donor_k) (k_overset in hp_kernels.cuh).  A uniform grid over
// the donor block's field tets limits the containment tests; it does not
// change the result (every tet containing x is registered in x's grid cell,
// and the lowest id among them is taken).  The arithmetic is the oracle's
// (oracle/hydra_oracle.c), so the tables agree bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/hydraphase.h"
#include "hp_overset_common.h"

namespace {

using hp_ov::bary;
using hp_ov::mn2;

struct Mesh {
    const hp_mesh* m;
    const int32_t* row(int e) const { return m->elem + 9 * (size_t)(e - 1); }
    void node(int n, double p[3]) const { p[0] = m->x[n - 1]; p[1] = m->y[n - 1]; p[2] = m->z[n - 1]; }
    void centroid(int e, double c[3]) const {
        const int32_t* r = row(e);
        const double* x = m->x; const double* y = m->y; const double* z = m->z;
        c[0] = 0.25 * (x[r[0] - 1] + x[r[1] - 1] + x[r[2] - 1] + x[r[3] - 1]);
        c[1] = 0.25 * (y[r[0] - 1] + y[r[1] - 1] + y[r[2] - 1] + y[r[3] - 1]);
        c[2] = 0.25 * (z[r[0] - 1] + z[r[1] - 1] + z[r[2] - 1] + z[r[3] - 1]);
    }
};

// Field tets of one block binned by bounding box (CSR lists, ascending ids).
struct Grid : hp_ov::GridParams {
    std::vector<int> start, items;
    int idx(int d, double v) const { return hp_ov::grid_index(*this, d, v); }
    size_t cell(int i, int j, int k) const { return ((size_t)i * n[1] + j) * n[2] + k; }
};

void build_grid(const Mesh& M, const std::vector<int>& field, const hp_ov::GridParams& gp, Grid& G) {
    static_cast<hp_ov::GridParams&>(G) = gp;
    const size_t ncell = (size_t)G.n[0] * G.n[1] * G.n[2];
    std::vector<int> cnt(ncell + 1, 0);
    auto span = [&](int t, int a[3], int b[3]) {
        double bl[3] = {1e300, 1e300, 1e300}, bh[3] = {-1e300, -1e300, -1e300};
        for (int q = 0; q < 4; q++) {
            double p[3];
            M.node(M.row(t)[q], p);
            for (int d = 0; d < 3; d++) { bl[d] = std::min(bl[d], p[d]); bh[d] = std::max(bh[d], p[d]); }
        }
        for (int d = 0; d < 3; d++) { a[d] = G.idx(d, bl[d]); b[d] = G.idx(d, bh[d]); }
    };
    for (int t : field) {
        int a[3], b[3];
        span(t, a, b);
        for (int i = a[0]; i <= b[0]; i++)
            for (int j = a[1]; j <= b[1]; j++)
                for (int k = a[2]; k <= b[2]; k++) cnt[G.cell(i, j, k) + 1]++;
    }
    for (size_t c = 0; c < ncell; c++) cnt[c + 1] += cnt[c];
    G.start = cnt;
    G.items.assign(cnt[ncell], 0);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int t : field) {
        int a[3], b[3];
        span(t, a, b);
        for (int i = a[0]; i <= b[0]; i++)
            for (int j = a[1]; j <= b[1]; j++)
                for (int k = a[2]; k <= b[2]; k++) G.items[fill[G.cell(i, j, k)]++] = t;
    }
}

}  // namespace

namespace hp_ov {

int prepare(const hp_mesh* mesh, const int32_t* block, int32_t layers, int32_t outer_type, int32_t* iblank_out,
            Prep& P) {
    if (!mesh || !block || !iblank_out || layers < 1 || mesh->neles <= 0 || mesh->nghosts < 0 || !mesh->elem ||
        (mesh->nghosts && !mesh->ghost) || !mesh->x || !mesh->y || !mesh->z)
        return HP_E_ARG;
    const int neles = mesh->neles, nghosts = mesh->nghosts, ntot = neles + nghosts;
    Mesh M{mesh};
    for (int e = 1; e <= neles; e++) {
        const int32_t* r = M.row(e);
        for (int k = 0; k < 4; k++)
            if (r[k] < 1 || r[k] > mesh->nodes || r[4 + k] < 1 || r[4 + k] > ntot) return HP_E_ARG;
        if (block[e - 1] != 0 && block[e - 1] != 1) return HP_E_ARG;
    }
    std::vector<int> gtype(ntot + 2, 0), mark(neles + 1, 0);
    for (int g = 0; g < nghosts; g++) {
        int id = mesh->ghost[4 * g + 1];
        if (id >= 1 && id <= ntot) gtype[id] = mesh->ghost[4 * g + 2];
    }
    for (int e = 1; e <= neles; e++) {
        const int32_t* r = M.row(e);
        if (r[8] != 1) continue;
        for (int k = 0; k < 4; k++) {
            int n = r[4 + k];
            if ((block[e - 1] == 0 && n <= neles && M.row(n)[8] == 0) ||
                (block[e - 1] == 1 && n > neles && gtype[n] == outer_type)) { mark[e] = 1; break; }
        }
    }
    for (int l = 2; l <= layers; l++)
        for (int e = 1; e <= neles; e++) {
            const int32_t* r = M.row(e);
            if (r[8] != 1 || mark[e]) continue;
            for (int k = 0; k < 4; k++) {
                int n = r[4 + k];
                if (n <= neles && mark[n] == l - 1 && block[n - 1] == block[e - 1]) { mark[e] = l; break; }
            }
        }
    P.fr.clear();
    for (int e = 1; e <= neles; e++) {
        iblank_out[e - 1] = mark[e] ? -1 : M.row(e)[8];
        if (mark[e]) P.fr.push_back(e);
    }
    for (int b = 0; b < 2; b++) P.field[b].clear();
    for (int e = 1; e <= neles; e++)
        if (iblank_out[e - 1] == 1) P.field[block[e - 1]].push_back(e);
    // grid over each block's field tets: bounding box, cell size 1.5x the
    // mean tet size, at most 512 cells per axis
    for (int b = 0; b < 2; b++) {
        GridParams& G = P.grid[b];
        G = GridParams{};
        if (P.field[b].empty()) continue;
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int t : P.field[b])
            for (int q = 0; q < 4; q++) {
                double p[3];
                M.node(M.row(t)[q], p);
                for (int d = 0; d < 3; d++) { lo[d] = std::min(lo[d], p[d]); hi[d] = std::max(hi[d], p[d]); }
            }
        double ext[3], vol = 1.0;
        for (int d = 0; d < 3; d++) { ext[d] = std::max(hi[d] - lo[d], 1e-300); vol *= ext[d]; G.lo[d] = lo[d]; }
        G.h = std::cbrt(vol / std::max<size_t>(P.field[b].size(), 1)) * 1.5;
        if (!(G.h > 0.0)) G.h = 1.0;
        for (int d = 0; d < 3; d++) G.n[d] = std::max(1, std::min(512, (int)(ext[d] / G.h) + 1));
    }
    return HP_OK;
}

// Wall triangles of the component (block 1): face k of an element (the nodes
// other than node k, in the order of src/sr_geometry.F90:149-158) whose
// neighbour is a ghost of type wall_type, in (element, face) order; then the
// two search grids of HoleView.  r3 exceeds the margin by a relative 1e-6
// and both grids add 1e-9 of the surface's extent, so every triangle that can
// pass a test at p sits in p's grid cell and the result equals a test of all
// triangles.
int prepare_hole(const hp_mesh* mesh, const int32_t* block, int32_t wall_type, double margin, HolePrep& H) {
    static const int FACE[4][3] = {{2, 3, 4}, {4, 3, 1}, {2, 4, 1}, {3, 2, 1}};
    if (!mesh || !block || !(margin >= 0.0) || !(margin < 1e300) || mesh->neles <= 0 || mesh->nghosts < 0 ||
        !mesh->elem || (mesh->nghosts && !mesh->ghost) || !mesh->x || !mesh->y || !mesh->z)
        return HP_E_ARG;
    const int neles = mesh->neles, ntot = neles + mesh->nghosts;
    Mesh M{mesh};
    std::vector<int> gtype(ntot + 2, 0);
    for (int g = 0; g < mesh->nghosts; g++) {
        const int id = mesh->ghost[4 * g + 1];
        if (id >= 1 && id <= ntot) gtype[id] = mesh->ghost[4 * g + 2];
    }
    H.tri.clear();
    for (int e = 1; e <= neles; e++) {
        const int32_t* r = M.row(e);
        for (int k = 0; k < 4; k++)
            if (r[k] < 1 || r[k] > mesh->nodes || r[4 + k] < 1 || r[4 + k] > ntot) return HP_E_ARG;
        if (block[e - 1] != 0 && block[e - 1] != 1) return HP_E_ARG;
        if (block[e - 1] != 1) continue;
        for (int k = 0; k < 4; k++) {
            const int n = r[4 + k];
            if (n <= neles || gtype[n] != wall_type) continue;
            for (int v = 0; v < 3; v++) {
                double q[3];
                M.node(r[FACE[k][v] - 1], q);
                H.tri.insert(H.tri.end(), q, q + 3);
            }
        }
    }
    const int ntri = (int)(H.tri.size() / 9);
    if (ntri == 0) return HP_E_ARG;
    double blo[3] = {1e300, 1e300, 1e300}, bhi[3] = {-1e300, -1e300, -1e300}, mean_ext = 0.0;
    std::vector<double> tlo(3 * (size_t)ntri), thi(3 * (size_t)ntri);
    for (int t = 0; t < ntri; t++) {
        const double* T = &H.tri[9 * (size_t)t];
        double te = 0.0;
        for (int d = 0; d < 3; d++) {
            const double lo = std::min(std::min(T[d], T[3 + d]), T[6 + d]);
            const double hi = std::max(std::max(T[d], T[3 + d]), T[6 + d]);
            tlo[3 * t + d] = lo; thi[3 * t + d] = hi;
            blo[d] = std::min(blo[d], lo); bhi[d] = std::max(bhi[d], hi);
            te = std::max(te, hi - lo);
        }
        mean_ext += te;
    }
    mean_ext /= ntri;
    const double L = std::max(std::max(bhi[0] - blo[0], bhi[1] - blo[1]), bhi[2] - blo[2]);
    const double tol = 1e-9 * L + 1e-300;
    const double r3 = margin * (1.0 + 1e-6) + tol;
    HoleView& V = H.v;
    V.m2 = margin * margin;
    // grid cells: g3 at least r3 / 2 and the mean triangle size, at most 64
    // per axis; g2 square cells of 1/256 of the projected extent
    auto setup = [&](GridParams& g, const double lo[3], const double hi[3], double h, bool yz, int cap) {
        g = GridParams{};
        g.h = h > 0.0 ? h : 1.0;
        for (int d = 0; d < 3; d++) {
            g.lo[d] = yz && d == 0 ? 0.0 : lo[d];
            g.n[d] = yz && d == 0 ? 1 : std::max(1, std::min(cap, (int)((hi[d] - lo[d]) / g.h) + 1));
        }
    };
    auto bin = [&](const GridParams& g, double grow, bool yz, std::vector<int>& start, std::vector<int>& items) {
        const size_t ncell = (size_t)g.n[0] * g.n[1] * g.n[2];
        start.assign(ncell + 1, 0);
        for (int pass = 0; pass < 2; pass++) {
            std::vector<int> fill;
            if (pass) { fill.assign(start.begin(), start.end() - 1); items.assign(start[ncell], 0); }
            for (int t = 0; t < ntri; t++) {
                int a[3], b[3];
                for (int d = 0; d < 3; d++) {
                    if (yz && d == 0) { a[d] = b[d] = 0; continue; }
                    a[d] = grid_index(g, d, tlo[3 * t + d] - grow);
                    b[d] = grid_index(g, d, thi[3 * t + d] + grow);
                }
                for (int i = a[0]; i <= b[0]; i++)
                    for (int j = a[1]; j <= b[1]; j++)
                        for (int k = a[2]; k <= b[2]; k++) {
                            const size_t c = ((size_t)i * g.n[1] + j) * g.n[2] + k;
                            if (pass) items[fill[c]++] = t; else start[c + 1]++;
                        }
            }
            if (!pass)
                for (size_t c = 0; c < ncell; c++) start[c + 1] += start[c];
        }
    };
    for (int d = 0; d < 3; d++) {
        V.lo3[d] = blo[d] - r3; V.hi3[d] = bhi[d] + r3;
        V.lo2[d] = blo[d] - tol; V.hi2[d] = bhi[d] + tol;
    }
    const double L3 = L + 2.0 * r3;
    setup(V.g3, V.lo3, V.hi3, std::max(std::max(L3 / 64.0, 0.5 * r3), mean_ext), false, 64);
    const double L2 = std::max(V.hi2[1] - V.lo2[1], V.hi2[2] - V.lo2[2]);
    setup(V.g2, V.lo2, V.hi2, L2 / 256.0, true, 256);
    bin(V.g3, r3, false, H.start3, H.items3);
    bin(V.g2, tol, true, H.start2, H.items2);
    V.tri = H.tri.data();
    V.start3 = H.start3.data(); V.items3 = H.items3.data();
    V.start2 = H.start2.data(); V.items2 = H.items2.data();
    return HP_OK;
}

}  // namespace hp_ov

// See include/hydraphase.h.
extern "C" int hp_overset_hole_cut(const hp_mesh* mesh, const int32_t* block, int32_t wall_type, double margin,
                                   int32_t* iblank_out, int32_t* nholes) {
    if (!iblank_out) return HP_E_ARG;
    hp_ov::HolePrep H;
    const int rc = hp_ov::prepare_hole(mesh, block, wall_type, margin, H);
    if (rc != HP_OK) return rc;
    Mesh M{mesh};
    const hp_ov::HoleView V = H.v;
    int nh = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : nh)
    for (int e = 1; e <= mesh->neles; e++) {
        int ib = M.row(e)[8];
        if (block[e - 1] == 0 && ib == 1) {
            double p[3];
            M.centroid(e, p);
            if (hp_ov::hole_test(V, p)) { ib = 0; nh++; }
        }
        iblank_out[e - 1] = ib;
    }
    if (nholes) *nholes = nh;
    return HP_OK;
}

// See include/hydraphase.h.
extern "C" int hp_overset_build(const hp_mesh* mesh, const int32_t* block, int32_t layers, int32_t outer_type,
                                int32_t* iblank_out, hp_overset* out) {
    if (!out) return HP_E_ARG;
    std::memset(out, 0, sizeof *out);
    hp_ov::Prep P;
    const int rc = hp_ov::prepare(mesh, block, layers, outer_type, iblank_out, P);
    if (rc != HP_OK) return rc;
    const int neles = mesh->neles;
    Mesh M{mesh};
    const std::vector<int>& fr = P.fr;
    const int nf = (int)fr.size();
    const std::vector<int>* field = P.field;
    Grid G[2];
    for (int b = 0; b < 2; b++)
        if (!field[b].empty()) build_grid(M, field[b], P.grid[b], G[b]);
    out->nfringe = nf;
    out->fringe = (int32_t*)std::malloc(sizeof(int32_t) * (size_t)(nf + 1));
    out->donor = (int32_t*)std::malloc(sizeof(int32_t) * 4 * (size_t)(nf + 1));
    out->weight = (double*)std::malloc(sizeof(double) * 4 * (size_t)(nf + 1));
    if (!out->fringe || !out->donor || !out->weight) { hp_free_overset(out); return HP_E_NOMEM; }
    std::vector<char> fell(nf, 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int f = 0; f < nf; f++) {
        const int e = fr[f], B = 1 - block[e - 1];
        int32_t* dn = out->donor + 4 * (size_t)f;
        double* w = out->weight + 4 * (size_t)f;
        out->fringe[f] = e;
        double xp[3];
        M.centroid(e, xp);
        int D = 0;
        if (!field[B].empty()) {
            const Grid& g = G[B];
            const size_t c = g.cell(g.idx(0, xp[0]), g.idx(1, xp[1]), g.idx(2, xp[2]));
            for (int it = g.start[c]; it < g.start[c + 1]; it++) {
                const int t = g.items[it];
                if (D && t > D) break;                 // lists are ascending
                const int32_t* r = M.row(t);
                double p[4][3], lam[4];
                for (int q = 0; q < 4; q++) M.node(r[q], p[q]);
                if (bary(p[0], p[1], p[2], p[3], xp, lam) == 0.0) continue;
                if (lam[0] >= -1e-10 && lam[1] >= -1e-10 && lam[2] >= -1e-10 && lam[3] >= -1e-10) D = t;
            }
            if (!D) {   // nearest field centroid of the donor block
                double best = 0.0;
                for (int t : field[B]) {
                    double cc[3];
                    M.centroid(t, cc);
                    double d2 = (cc[0] - xp[0]) * (cc[0] - xp[0]) + (cc[1] - xp[1]) * (cc[1] - xp[1]) +
                                (cc[2] - xp[2]) * (cc[2] - xp[2]);
                    if (!D || d2 < best) { best = d2; D = t; }
                }
                fell[f] = 1;
            }
        }
        if (!D) {   // the other block has no field cell at all
            dn[0] = dn[1] = dn[2] = dn[3] = e;
            w[0] = 1.0; w[1] = w[2] = w[3] = 0.0;
            fell[f] = 1;
            continue;
        }
        dn[0] = dn[1] = dn[2] = dn[3] = D;
        w[0] = 1.0; w[1] = w[2] = w[3] = 0.0;
        int cand[17], m = 0;
        cand[m++] = D;
        for (int ring = 0, lo = 0; ring < 2; ring++) {
            int hi = m;
            for (int a = lo; a < hi; a++)
                for (int k = 0; k < 4 && m < 17; k++) {
                    int n = M.row(cand[a])[4 + k];
                    if (n > neles || iblank_out[n - 1] != 1 || block[n - 1] != B) continue;
                    bool seen = false;
                    for (int q = 0; q < m; q++) seen |= (cand[q] == n);
                    if (!seen) cand[m++] = n;
                }
            lo = hi;
        }
        double cc[17][3];
        for (int a = 0; a < m; a++) M.centroid(cand[a], cc[a]);
        double best_in = 0.0, best_out = -1.0e300;
        bool have_in = false;
        for (int i = 0; i < m; i++)
            for (int j = i + 1; j < m; j++)
                for (int k = j + 1; k < m; k++)
                    for (int l = k + 1; l < m; l++) {
                        double lam[4];
                        if (bary(cc[i], cc[j], cc[k], cc[l], xp, lam) == 0.0) continue;
                        const double sc = mn2(mn2(mn2(lam[0], lam[1]), lam[2]), lam[3]);
                        const int id[4] = {i, j, k, l};
                        if (sc >= -1e-12) {
                            double s2 = 0.0;
                            for (int q = 0; q < 4; q++)
                                s2 = s2 + ((cc[id[q]][0] - xp[0]) * (cc[id[q]][0] - xp[0]) +
                                           (cc[id[q]][1] - xp[1]) * (cc[id[q]][1] - xp[1]) +
                                           (cc[id[q]][2] - xp[2]) * (cc[id[q]][2] - xp[2]));
                            if (!have_in || s2 < best_in) {
                                have_in = true; best_in = s2;
                                for (int q = 0; q < 4; q++) { dn[q] = cand[id[q]]; w[q] = lam[q]; }
                            }
                        } else if (!have_in && sc > best_out) {
                            best_out = sc;
                            for (int q = 0; q < 4; q++) { dn[q] = cand[id[q]]; w[q] = lam[q]; }
                        }
                    }
    }
    out->nfallback = 0;
    for (int f = 0; f < nf; f++) out->nfallback += fell[f];
    return HP_OK;
}

extern "C" void hp_free_overset(hp_overset* ov) {
    if (!ov) return;
    std::free(ov->fringe);
    std::free(ov->donor);
    std::free(ov->weight);
    ov->fringe = nullptr; ov->donor = nullptr; ov->weight = nullptr;
    ov->nfringe = 0;
}
