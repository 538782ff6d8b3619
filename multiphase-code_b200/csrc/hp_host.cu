// hp_host.cu -- C ABI of the engine (include/hydraphase.h): mesh setup,
// geometry, device layout, state transfer and the step loop.
//
// Geometry is set-up work the reference also does on the host
// (src/sr_geometry.F90 has no device regions); it is restated here with the
// reference's operand order so face vectors, volumes, centroids and dl are
// bit-identical.  The time step itself runs only on the device.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>
#include <omp.h>

#include "../../include/hydraphase.h"
#include "hp_device.h"

using namespace hp;

namespace {

thread_local std::string g_create_error;

struct Arena {
    char* base = nullptr;
    size_t size = 0, used = 0;
    void* take(size_t bytes) {
        size_t off = (used + 255) & ~size_t(255);
        used = off + bytes;
        return base ? base + off : nullptr;
    }
};

inline double mn2(double a, double b) { return (b < a || a != a) ? b : a; }
inline double mx2(double a, double b) { return (b > a || a != a) ? b : a; }
inline double sq(double a) { return a * a; }
inline double det3(double A11, double A21, double A31, double A12, double A22, double A32,
                   double A13, double A23, double A33) {
    return A11 * (A22 * A33 - A23 * A32) - A21 * (A12 * A33 - A13 * A32) +
           A31 * (A12 * A23 - A13 * A22);
}

const int GEO_FACE[4][3] = {{2, 3, 4}, {4, 3, 1}, {2, 4, 1}, {3, 2, 1}};
const int HLL_FACE[4][3] = {{2, 4, 3}, {3, 4, 1}, {4, 2, 1}, {2, 3, 1}};
const int VIS_FACE[4][3] = {{2, 3, 4}, {1, 3, 4}, {1, 2, 4}, {1, 2, 3}};

}  // namespace

// Element and ghost ranges of one case of a handle (see DevMesh).
struct CaseRange {
    int e0 = 0, ne = 0;     // elements [e0, e0 + ne)
    int g0 = 0, ng = 0;     // ghost list entries [g0, g0 + ng), slots neles + g0 ...
    int cell1 = 0;          // slot of the case's reference cell 1
    int aliased = 0;
};

// One asynchronous output request (hp_output_async): the device staging of
// the snapshot, its pinned host copy, and the thread that writes the files.
struct OutSlot {
    double* d_buf = nullptr;
    double* h_buf = nullptr;
    size_t cap = 0;            // doubles in each buffer
    cudaEvent_t ready = nullptr, copied = nullptr;
    std::thread writer;
    int ticket = 0;            // 0: idle
    int rc = HP_OK;
};

struct hp_handle {
    hp_params prm{};
    DevParams dp{};
    DevMesh dm{};
    DevState<double> ds{};
    const Variant* var = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    GridSync* d_sync = nullptr;  // fused step (use_graph = 2): its grid barrier
    int fused = 0;               // blocks of the fused step; 0: not this handle
    Arena arena;
    int device = 0;
    int neles = 0, nghosts = 0, ntot = 0;
    long long ld = 0;
    int ncase = 1;
    std::vector<CaseRange> cases;
    std::vector<int> perm;      // [neles] case c's reference element i -> slot, at cases[c].e0 + i
    std::vector<int> ghost_id;  // [nghosts] case c's ghost g -> slot, at cases[c].g0 + g
    void* d_overset = nullptr;  // overset fringe table (hp_set_overset)
    int* d_halo = nullptr;      // partition halo table (hp_set_halo): dst, then src
    hp_exchange_fn xfn = nullptr;   // exchange callback of a part on several GPUs
    void* xuser = nullptr;
    int* d_xlist = nullptr;     // send cells, then receive cells (hp_set_halo_lists)
    int nsend = 0, nrecv = 0;
    int* d_perm = nullptr;      // the two maps above, on the device
    int* d_gid = nullptr;
    double* d_gstage = nullptr; // 6 x nghosts staging of ghost primitives
    bool started = false, have_state = false;
    std::vector<char> state_set;   // per case: state uploaded
    int aliased = 0;
    int neq = 10;               // conserved variables: 10, or 22 with the five-phase model
    int nwall = 0, ngwall = 0;  // FP64 wall-layer cells and their gradient cells
    int wprefix = 0;            // 1: those lists are the first cells of the order
    int max_diag = 4096;
    std::string err;
    double* h_diag = nullptr;   // pinned
    DevScalars* h_scal = nullptr;
    GridSync* h_sync = nullptr;     // pinned copy of d_sync (its error flag)
    OutSlot out[2];             // asynchronous output, two requests in flight
    cudaStream_t ostream = nullptr;
    int next_ticket = 1;
};

static int fail(hp_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    else g_create_error = msg;
    return code;
}

#define CUDA_OK(h, call)                                                                  \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(h, HP_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------
// 30-bit Hilbert index of a point with 10-bit integer coordinates
// (Skilling's transpose algorithm, "Programming the Hilbert curve", AIP
// Conf. Proc. 707, 2004): undo the excess work per level, Gray-encode, then
// interleave the transposed bits.  Consecutive indices are face-adjacent
// cells of the 1024^3 grid, so neighbours stay closer in the sorted order
// than along a Morton curve.
static inline uint32_t hilbert10(uint32_t x0, uint32_t x1, uint32_t x2) {
    uint32_t x[3] = {x0, x1, x2};
    const uint32_t M = 1u << 9;
    for (uint32_t Q = M; Q > 1; Q >>= 1) {
        const uint32_t P = Q - 1;
        for (int i = 0; i < 3; i++) {
            if (x[i] & Q) {
                x[0] ^= P;
            } else {
                const uint32_t t = (x[0] ^ x[i]) & P;
                x[0] ^= t;
                x[i] ^= t;
            }
        }
    }
    x[1] ^= x[0];
    x[2] ^= x[1];
    uint32_t t = 0;
    for (uint32_t Q = M; Q > 1; Q >>= 1)
        if (x[2] & Q) t ^= Q - 1;
    for (int i = 0; i < 3; i++) x[i] ^= t;
    uint32_t key = 0;
    for (int j = 9; j >= 0; j--)
        for (int i = 0; i < 3; i++) key = (key << 1) | ((x[i] >> j) & 1u);
    return key;
}

extern "C" const char* hp_create_error(void) { return g_create_error.c_str(); }

// See include/hydraphase.h.
extern "C" int hp_set_host_threads(int32_t n) {
    if (n < 0) return HP_E_ARG;
    omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
    return HP_OK;
}

extern "C" const char* hp_last_error(const hp_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

// Carves every device array of a handle out of one arena (a probe arena
// with no base only measures).  The same plan sizes hp_estimate_bytes.
static void plan_arena(hp_handle* h, Arena& a, int neles, int nghosts, long long ld, size_t gb, int ncase,
                       int nface) {
    const size_t D = sizeof(double), I = sizeof(int);
    DevMesh& m = h->dm;
    m.nc = (int*)a.take(4 * ld * I); m.snb = (int*)a.take(4 * ld * I);
    m.fk = (unsigned*)a.take(ld * sizeof(unsigned)); m.iblank = (int*)a.take(ld * I);
    m.xc = (double*)a.take(ld * D); m.yc = (double*)a.take(ld * D); m.zc = (double*)a.take(ld * D);
    m.vol = (double*)a.take(ld * D); m.dl = (double*)a.take(ld * D); m.dd = (double*)a.take(ld * D);
    m.eps2 = (double*)a.take(ld * D);
    m.sc = (double*)a.take(12 * ld * D); m.fch = (double*)a.take(12 * ld * D);
    m.fcv = (double*)a.take(12 * ld * D);
    m.dxn = (double*)a.take(12 * ld * D);
    m.lsqa = (double*)a.take(NLSQ * ld * D);
    m.lsqb = (double*)a.take(NLSQ * ld * D);
    m.g_par = (int*)a.take((nghosts + 1) * (size_t)I); m.g_id = (int*)a.take((nghosts + 1) * (size_t)I);
    m.g_type = (int*)a.take((nghosts + 1) * (size_t)I);
    DevState<double>& s = h->ds;
    const long long nq = h->neq;
    s.cn = (double*)a.take(nq * ld * D); s.cu = (double*)a.take(nq * ld * D);
    s.cn1 = (double*)a.take(nq * ld * D); s.pr = (double*)a.take(NPR * ld * D);
    // primitives in the arithmetic of the gradients and fluxes: a float copy
    // for the FP32-arithmetic variants, the FP64 columns themselves otherwise
    s.prr = gb == D ? s.pr : (double*)a.take(NPR * ld * gb);
    s.gr = (double*)a.take(NGR * ld * gb); s.phi = (double*)a.take(ld * D);
    s.anu = (double*)a.take(2 * ld * D); s.d2q = (double*)a.take(nq * ld * D);
    s.d24 = (double*)a.take(nq * ld * D); s.vis = (double*)a.take(8 * ld * D);
    if (h->neq == 22) {
        s.qpr = (double*)a.take(12 * ld * D); s.anuq = (double*)a.take(3 * ld * D);
        s.qdrag = (double*)a.take(9 * ld * D);
    } else {
        s.qpr = s.anuq = s.qdrag = nullptr;
    }
    s.egt = (double*)a.take(2 * ld * D);
    s.s = (DevScalars*)a.take(ncase * sizeof(DevScalars));
    s.diag = (double*)a.take((size_t)ncase * h->max_diag * 8 * D);
    s.max_diag = h->max_diag;
    m.cid = ncase > 1 ? (const int*)a.take((size_t)neles * I) : nullptr;
    m.nwall = h->nwall; m.ngwall = h->ngwall; m.wprefix = h->wprefix;
    if (h->nwall > 0) {
        m.wcells = (const int*)a.take((size_t)h->nwall * I);
        m.gcells = (const int*)a.take((size_t)h->ngwall * I);
        m.wclass = (const unsigned char*)a.take((size_t)ld);
        s.gr64 = (double*)a.take(NGR * ld * D);
    } else {
        m.wcells = m.gcells = nullptr;
        m.wclass = nullptr;
        s.gr64 = nullptr;
    }
    m.nface = nface;
    m.fld = ((long long)nface + 63) / 64 * 64;
    s.racc = nullptr;
    m.fcolor = nullptr;
    if (nface > 0) {
        m.f_i = (const int*)a.take((size_t)nface * I);
        m.f_code = (const int*)a.take((size_t)nface * I);
        m.cface = (const int*)a.take(4 * (size_t)ld * I);
        s.ff = (double*)a.take((size_t)FACE_REC * (size_t)m.fld * gb);
        if (h->prm.face_mode >= 2) {   // colouring or atomics: per-cell face sums
            s.racc = (double*)a.take(10 * (size_t)ld * D);
            m.fcolor = (const int*)a.take((size_t)nface * I);
        }
    } else {
        m.f_i = m.f_code = m.cface = nullptr;
        s.ff = nullptr;
    }
    h->d_sync = (GridSync*)a.take(sizeof(GridSync));
    h->d_perm = (int*)a.take((neles + 1) * (size_t)I);
    h->d_gid = (int*)a.take((nghosts + 1) * (size_t)I);
    h->d_gstage = (double*)a.take(6 * (nghosts + 1) * D);
}

// Host staging of a handle's device layout (columns of leading dimension ld)
// and ghost lists, filled case by case by fill_case.
struct Layout {
    int neles = 0, nghosts = 0;
    long long ld = 0;
    std::vector<int> nc, snb, ib, gpar, gid, gtyp, perm, ghost_id;
    std::vector<unsigned> fk;
    std::vector<double> x, y, z, vol, dl, dd, eps2, sc, fch, fcv, la, lb;
    Layout(int ne, int ng) : neles(ne), nghosts(ng), ld(((long long)ne + ng + 63) / 64 * 64) {
        nc.assign(4 * ld, 0); snb.assign(4 * ld, 0); ib.assign(ld, 0); fk.assign(ld, 0u);
        gpar.assign(ng, 0); gid.assign(ng, 0); gtyp.assign(ng, 0); perm.assign(ne, 0); ghost_id.assign(ng, 0);
        for (auto* v : {&x, &y, &z, &vol, &dl, &dd, &eps2}) v->assign(ld, 0.0);
        for (auto* v : {&sc, &fch, &fcv}) v->assign(12 * ld, 0.0);
        la.assign(NLSQ * ld, 0.0); lb.assign(NLSQ * ld, 0.0);
    }
};

// Cells within `layers` layers of a wall ghost (types 5 and 6), breadth
// first over the interior neighbours: wall (ascending), the same with their
// interior neighbours added (grad, ascending), and the per-slot class (1: a
// layer cell with a neighbour outside the layers, 2: one without).
static void wall_layers(const Layout& L, int neles, int nghosts, long long ld, int layers,
                        std::vector<int>& wall, std::vector<int>& grad, std::vector<unsigned char>& cls) {
    std::vector<int> gtype((size_t)nghosts, 0);
    for (int g = 0; g < nghosts; g++) {
        const int t = L.gid[g];
        if (t >= neles && t < neles + nghosts) gtype[t - neles] = L.gtyp[g];
    }
    std::vector<int> layer((size_t)neles, 0), front;
    for (int t = 0; t < neles; t++)
        for (int f = 0; f < 4; f++) {
            const int j = L.nc[(size_t)f * ld + t];
            if (j >= neles && j < neles + nghosts && (gtype[j - neles] == 5 || gtype[j - neles] == 6)) {
                layer[t] = 1;
                front.push_back(t);
                break;
            }
        }
    for (int k = 2; k <= layers && !front.empty(); k++) {
        std::vector<int> next;
        for (int t : front)
            for (int f = 0; f < 4; f++) {
                const int j = L.nc[(size_t)f * ld + t];
                if (j < neles && layer[j] == 0) { layer[j] = k; next.push_back(j); }
            }
        front.swap(next);
    }
    cls.assign((size_t)ld, 0);
    std::vector<unsigned char> ing((size_t)neles, 0);
    for (int t = 0; t < neles; t++)
        if (layer[t] > 0) {
            wall.push_back(t);
            cls[t] = 1;
            ing[t] = 1;
            for (int f = 0; f < 4; f++) {
                const int j = L.nc[(size_t)f * ld + t];
                if (j < neles) ing[j] = 1;
            }
        }
    for (int t = 0; t < neles; t++)
        if (ing[t]) grad.push_back(t);
    // class 2: every interior neighbour is a layer cell too, so no FP32 face
    // needs the cell's FP32 gradients
    for (int t : wall) {
        bool inner = true;
        for (int f = 0; f < 4 && inner; f++) {
            const int j = L.nc[(size_t)f * ld + t];
            if (j < neles && layer[j] == 0) inner = false;
        }
        if (inner) cls[t] = 2;
    }
}

// One case of a handle: validates its connectivity, computes its geometry
// and static least-squares terms, picks its internal cell order and writes
// everything into the handle's staging layout at the case's offsets
// (elements from cr.e0, ghosts from L.neles + cr.g0).  On error returns an
// HP_E_* code with the message in err.
static int fill_case(const hp_mesh* mesh, const hp_params* params, Layout& L, CaseRange& cr, std::string& err) {
    const int nodes = mesh->nodes, neles = mesh->neles, nghosts = mesh->nghosts;
    const int ntot = neles + nghosts;
    const int E0 = cr.e0, G0 = cr.g0, Etot = L.neles;
    const long long ld = L.ld;
    auto bad = [&](int code, const std::string& m) { err = m; return code; };
    // --- validate connectivity (1-based as read) ---
    for (long long e = 0; e < neles; e++) {
        const int32_t* r = mesh->elem + 9 * e;
        for (int k = 0; k < 4; k++)
            if (r[k] < 1 || r[k] > nodes)
                return bad(HP_E_ARG, "element " + std::to_string(e + 1) + ": node id out of range");
        for (int k = 4; k < 8; k++)
            if (r[k] < 1 || r[k] > ntot)
                return bad(HP_E_ARG, "element " + std::to_string(e + 1) + ": neighbour id out of range");
    }
    for (long long g = 0; g < nghosts; g++) {
        const int32_t* r = mesh->ghost + 4 * g;
        if (r[0] < 1 || r[0] > ntot || r[1] < 1 || r[1] > ntot || r[3] < 1 || r[3] > 4)
            return bad(HP_E_ARG, "ghost " + std::to_string(g + 1) + ": bad parent/id/side");
    }

    // --- geometry, src/sr_geometry.F90:112-347 (1-based work arrays) ---
    std::vector<double> x(nodes + 1), y(nodes + 1), z(nodes + 1);
    for (int n = 1; n <= nodes; n++) { x[n] = mesh->x[n - 1]; y[n] = mesh->y[n - 1]; z[n] = mesh->z[n - 1]; }
    double xmax = -1.0e30, ymax = -1.0e30, zmax = -1.0e30, ymin = 1.0e30, zmin = 1.0e30;
    for (int n = 1; n <= nodes; n++) {
        xmax = mx2(xmax, x[n]); ymax = mx2(ymax, y[n]); zmax = mx2(zmax, z[n]);
        ymin = mn2(ymin, y[n]); zmin = mn2(zmin, z[n]);
    }
    std::vector<int> nod[4], nc[4];
    for (int k = 0; k < 4; k++) { nod[k].assign(ntot + 1, 0); nc[k].assign(ntot + 1, 0); }
    std::vector<int> iblank(ntot + 1, 0);
    for (int e = 1; e <= neles; e++) {
        const int32_t* r = mesh->elem + 9 * (size_t)(e - 1);
        for (int k = 0; k < 4; k++) { nod[k][e] = r[k]; nc[k][e] = r[4 + k]; }
        iblank[e] = r[8];
    }
    std::vector<double> xcel(ntot + 1, 0.0), ycel(ntot + 1, 0.0), zcel(ntot + 1, 0.0), vol(ntot + 1, 0.0),
        dl(ntot + 1, 0.0), dd(ntot + 1, 0.0);
    std::vector<double> sc(12 * (size_t)(ntot + 1), 0.0), fch(12 * (size_t)(ntot + 1), 0.0),
        fcv(12 * (size_t)(ntot + 1), 0.0);
    auto SC = [&](int k, int i) -> double& { return sc[(size_t)k * (ntot + 1) + i]; };
    auto FCH = [&](int k, int i) -> double& { return fch[(size_t)k * (ntot + 1) + i]; };
    auto FCV = [&](int k, int i) -> double& { return fcv[(size_t)k * (ntot + 1) + i]; };
    // per-cell loops below are independent across cells (each writes only
    // its own slots), so they run on all host cores with identical results
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= neles; i++) {
        for (int f = 0; f < 4; f++) {
            int n1 = nod[GEO_FACE[f][0] - 1][i], n2 = nod[GEO_FACE[f][1] - 1][i], n3 = nod[GEO_FACE[f][2] - 1][i];
            double dxyA = (x[n1] - x[n2]) * (y[n1] + y[n2]);
            double dxyB = (x[n2] - x[n3]) * (y[n2] + y[n3]);
            double dxyC = (x[n3] - x[n1]) * (y[n3] + y[n1]);
            double dyzA = (y[n1] - y[n2]) * (z[n1] + z[n2]);
            double dyzB = (y[n2] - y[n3]) * (z[n2] + z[n3]);
            double dyzC = (y[n3] - y[n1]) * (z[n3] + z[n1]);
            double dzxA = (z[n1] - z[n2]) * (x[n1] + x[n2]);
            double dzxB = (z[n2] - z[n3]) * (x[n2] + x[n3]);
            double dzxC = (z[n3] - z[n1]) * (x[n3] + x[n1]);
            SC(3 * f + 0, i) = 0.5 * (dyzA + dyzB + dyzC);
            SC(3 * f + 1, i) = 0.5 * (dzxA + dzxB + dzxC);
            SC(3 * f + 2, i) = 0.5 * (dxyA + dxyB + dxyC);
            int a = nod[HLL_FACE[f][0] - 1][i], b = nod[HLL_FACE[f][1] - 1][i], c = nod[HLL_FACE[f][2] - 1][i];
            FCH(f, i) = (x[a] + x[b] + x[c]) * 0.3333;
            FCH(4 + f, i) = (y[a] + y[b] + y[c]) * 0.3333;
            FCH(8 + f, i) = (z[a] + z[b] + z[c]) * 0.3333;
            a = nod[VIS_FACE[f][0] - 1][i]; b = nod[VIS_FACE[f][1] - 1][i]; c = nod[VIS_FACE[f][2] - 1][i];
            FCV(f, i) = (x[a] + x[b] + x[c]) / 3.0;
            FCV(4 + f, i) = (y[a] + y[b] + y[c]) / 3.0;
            FCV(8 + f, i) = (z[a] + z[b] + z[c]) / 3.0;
        }
        int n1 = nod[0][i], n2 = nod[1][i], n3 = nod[2][i], n4 = nod[3][i];
        double x1 = x[n1], x2 = x[n2], x3 = x[n3], x4 = x[n4];
        double y1 = y[n1], y2 = y[n2], y3 = y[n3], y4 = y[n4];
        double z1 = z[n1], z2 = z[n2], z3 = z[n3], z4 = z[n4];
        xcel[i] = 0.25 * (x1 + x2 + x3 + x4);
        ycel[i] = 0.25 * (y1 + y2 + y3 + y4);
        zcel[i] = 0.25 * (z1 + z2 + z3 + z4);
        double dl12 = std::sqrt(sq(x1 - x2) + sq(y1 - y2) + sq(z1 - z2));
        double dl13 = std::sqrt(sq(x1 - x3) + sq(y1 - y3) + sq(z1 - z3));
        double dl14 = std::sqrt(sq(x1 - x4) + sq(y1 - y4) + sq(z1 - z4));
        double dl23 = std::sqrt(sq(x2 - x3) + sq(y2 - y3) + sq(z2 - z3));
        double dl42 = std::sqrt(sq(x4 - x2) + sq(y4 - y2) + sq(z4 - z2));
        double dl43 = std::sqrt(sq(x4 - x3) + sq(y4 - y3) + sq(z4 - z3));
        dl[i] = mn2(mn2(mn2(mn2(mn2(dl12, dl13), dl14), dl23), dl42), dl43);
        double v6 = det3(x2, x3, x4, y2, y3, y4, z2, z3, z4) - det3(x1, x3, x4, y1, y3, y4, z1, z3, z4) +
                    det3(x1, x2, x4, y1, y2, y4, z1, z2, z4) - det3(x1, x2, x3, y1, y2, y3, z1, z2, z3);
        vol[i] = std::fabs(v6) / 6.0;
    }
    std::vector<int> gpar(nghosts), gid(nghosts), gtyp(nghosts), gside(nghosts);
    for (int g = 0; g < nghosts; g++) {
        const int32_t* r = mesh->ghost + 4 * (size_t)g;
        gpar[g] = r[0]; gid[g] = r[1]; gtyp[g] = r[2]; gside[g] = r[3];
    }
    for (int g = 0; g < nghosts; g++) {   // mirrored ghost centroids, sequential
        int np = gpar[g], ng = gid[g], ns = gside[g];
        int n1 = nod[GEO_FACE[ns - 1][0] - 1][np], n2 = nod[GEO_FACE[ns - 1][1] - 1][np],
            n3 = nod[GEO_FACE[ns - 1][2] - 1][np];
        double xcf = (x[n1] + x[n2] + x[n3]) / 3.0;
        double ycf = (y[n1] + y[n2] + y[n3]) / 3.0;
        double zcf = (z[n1] + z[n2] + z[n3]) / 3.0;
        xcel[ng] = 2.0 * xcf - xcel[np];
        ycel[ng] = 2.0 * ycf - ycel[np];
        zcel[ng] = 2.0 * zcf - zcel[np];
        vol[ng] = vol[np];
        nc[0][ng] = ng; nc[1][ng] = ng; nc[2][ng] = ng; nc[3][ng] = ng;
    }
    for (int g = 0; g < nghosts; g++) {   // wave-transmissive distance
        int np = gpar[g], nt = gtyp[g];
        int n1 = nod[0][np], n2 = nod[1][np], n3 = nod[2][np], n4 = nod[3][np];
        if (nt == 3) {
            double xc = (x[n1] + x[n2] + x[n3] + x[n4]) * 0.25;
            dd[np] = std::fabs(xmax - xc);
        } else if (nt == 51) {
            double yc = (y[n1] + y[n2] + y[n3] + y[n4]) * 0.25;
            dd[np] = (yc > 0) ? std::fabs(ymax - yc) : std::fabs(ymin - yc);
        } else if (nt == 53) {
            double zc = (z[n1] + z[n2] + z[n3] + z[n4]) * 0.25;
            dd[np] = (zc > (double)0.1f) ? std::fabs(zmax - zc) : std::fabs(zmin - zc);
        }
    }
    // --- static least-squares terms of the gradient and source operators ---
    std::vector<double> lsqa(NLSQ * (size_t)(neles + 1), 0.0), lsqb(NLSQ * (size_t)(neles + 1), 0.0);
    auto LA = [&](int k, int i) -> double& { return lsqa[(size_t)k * (neles + 1) + i]; };
    auto LB = [&](int k, int i) -> double& { return lsqb[(size_t)k * (neles + 1) + i]; };
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= neles; i++) {
        double xa[4], ya[4], za[4], wa[4], wb[4];
        for (int f = 0; f < 4; f++) {
            int nb = nc[f][i];
            xa[f] = xcel[nb] - xcel[i];
            ya[f] = ycel[nb] - ycel[i];
            za[f] = zcel[nb] - zcel[i];
            wa[f] = sq(xa[f]) + sq(ya[f]) + sq(za[f]);
            wb[f] = std::sqrt(sq(xa[f]) + sq(ya[f]) + sq(za[f]));
        }
        // src/sr_derivative.F90:163-176 and :255
        double a1 = sq(xa[0]) / wa[0] + sq(xa[1]) / wa[1] + sq(xa[2]) / wa[2] + sq(xa[3]) / wa[3];
        double a2 = sq(ya[0]) / wa[0] + sq(ya[1]) / wa[1] + sq(ya[2]) / wa[2] + sq(ya[3]) / wa[3];
        double a3 = sq(za[0]) / wa[0] + sq(za[1]) / wa[1] + sq(za[2]) / wa[2] + sq(za[3]) / wa[3];
        double b1 = xa[0] * ya[0] / wa[0] + xa[1] * ya[1] / wa[1] + xa[2] * ya[2] / wa[2] + xa[3] * ya[3] / wa[3];
        double b2 = xa[0] * za[0] / wa[0] + xa[1] * za[1] / wa[1] + xa[2] * za[2] / wa[2] + xa[3] * za[3] / wa[3];
        double b3 = za[0] * ya[0] / wa[0] + za[1] * ya[1] / wa[1] + za[2] * ya[2] / wa[2] + za[3] * ya[3] / wa[3];
        for (int f = 0; f < 4; f++) LA(f, i) = wa[f];
        LA(4, i) = a1; LA(5, i) = a2; LA(6, i) = a3; LA(7, i) = b1; LA(8, i) = b2; LA(9, i) = b3;
        LA(10, i) = det3(a1, b1, b2, b1, a2, b3, b2, b3, a3);
        // the correctly rounded reciprocals of the weights and the
        // determinant, which the device's shared-reciprocal division takes
        for (int f = 0; f < 4; f++) LA(11 + f, i) = 1.0 / wa[f];
        LA(15, i) = 1.0 / LA(10, i);
        // src/sr_source.F90:100-117
        a1 = sq(xa[0]) / wb[0] + sq(xa[1]) / wb[1] + sq(xa[2]) / wb[2] + sq(xa[3]) / wb[3];
        a2 = sq(ya[0]) / wb[0] + sq(ya[1]) / wb[1] + sq(ya[2]) / wb[2] + sq(ya[3]) / wb[3];
        a3 = sq(za[0]) / wb[0] + sq(za[1]) / wb[1] + sq(za[2]) / wb[2] + sq(za[3]) / wb[3];
        b1 = xa[0] * ya[0] / wb[0] + xa[1] * ya[1] / wb[1] + xa[2] * ya[2] / wb[2] + xa[3] * ya[3] / wb[3];
        b2 = xa[0] * za[0] / wb[0] + xa[1] * za[1] / wb[1] + xa[2] * za[2] / wb[2] + xa[3] * za[3] / wb[3];
        b3 = ya[0] * za[0] / wb[0] + ya[1] * za[1] / wb[1] + ya[2] * za[2] / wb[2] + ya[3] * za[3] / wb[3];
        for (int f = 0; f < 4; f++) LB(f, i) = wb[f];
        LB(4, i) = a1; LB(5, i) = a2; LB(6, i) = a3; LB(7, i) = b1; LB(8, i) = b2; LB(9, i) = b3;
        LB(10, i) = det3(a1, b1, b2, b1, a2, b3, b2, b3, a3);
        for (int f = 0; f < 4; f++) LB(11 + f, i) = 1.0 / wb[f];
        LB(15, i) = 1.0 / LB(10, i);
    }
    // --- aliasing: ghost slots that are elements, repeated, or ghost parents ---
    {
        std::vector<char> seen(ntot + 1, 0);
        int al = 0;
        for (int g = 0; g < nghosts && !al; g++) {
            if (gid[g] <= neles || seen[gid[g]]) al = 1;
            seen[gid[g]] = 1;
        }
        for (int g = 0; g < nghosts && !al; g++)
            if (gpar[g] > neles || seen[gpar[g]]) al = 1;
        // neighbours in the ghost range must be ghost slots that exist
        for (int e = 1; e <= neles && !al; e++)
            for (int k = 0; k < 4; k++)
                if (nc[k][e] > neles && !seen[nc[k][e]]) { al = 1; break; }
        cr.aliased = al;
    }
    // --- internal order: space-filling curve over element centroids ---
    std::vector<int> perm(neles + 1);   // 1-based reference id -> 0-based internal
    std::iota(perm.begin(), perm.end(), -1);
    if (params->renumber && !cr.aliased) {
        // centroids on a 1024^3 grid over the bounding cube (one scale for
        // all axes, so a thin domain does not stretch the curve), sorted by
        // Hilbert index
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int i = 1; i <= neles; i++) {
            double p[3] = {xcel[i], ycel[i], zcel[i]};
            for (int d = 0; d < 3; d++) { lo[d] = std::min(lo[d], p[d]); hi[d] = std::max(hi[d], p[d]); }
        }
        const double ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
        // FP64 wall layers of the FP32-arithmetic variants: the cells within
        // the layers first (group 0), then their other interior neighbours
        // (group 1), then the rest, each group along the curve.  The
        // layer kernels' cell lists are then contiguous ranges of the order,
        // and the FP32 kernels skip whole warps instead of scattered cells.
        // (The same breadth-first search over interior neighbours from the
        // cells next to a wall ghost of type 5 or 6 as wall_layers.)
        std::vector<uint8_t> group(neles + 1, 2);
        const bool fp32_arith = params->precision == HP_PREC_MIXED || params->precision == HP_PREC_FP32;
        if (fp32_arith && params->wall_fp64_layers > 0) {
            std::vector<int> gtype_of(ntot + 1, 0);
            for (int g = 0; g < nghosts; g++) gtype_of[gid[g]] = gtyp[g];
            std::vector<int> layer(neles + 1, 0), front;
            for (int e = 1; e <= neles; e++)
                for (int k = 0; k < 4; k++) {
                    const int j = nc[k][e];
                    if (j > neles && j <= ntot && (gtype_of[j] == 5 || gtype_of[j] == 6)) {
                        layer[e] = 1;
                        front.push_back(e);
                        break;
                    }
                }
            for (int k = 2; k <= params->wall_fp64_layers && !front.empty(); k++) {
                std::vector<int> next;
                for (int e : front)
                    for (int f = 0; f < 4; f++) {
                        const int j = nc[f][e];
                        if (j <= neles && layer[j] == 0) { layer[j] = k; next.push_back(j); }
                    }
                front.swap(next);
            }
            for (int e = 1; e <= neles; e++)
                if (layer[e] > 0) {
                    group[e] = 0;
                    for (int f = 0; f < 4; f++) {
                        const int j = nc[f][e];
                        if (j <= neles && layer[j] == 0) group[j] = 1;
                    }
                }
        }
        std::vector<std::pair<uint32_t, int>> key(neles);
#pragma omp parallel for schedule(static)
        for (int i = 1; i <= neles; i++) {
            double p[3] = {xcel[i], ycel[i], zcel[i]};
            uint32_t q[3];
            for (int d = 0; d < 3; d++) {
                double t = ext > 0.0 ? (p[d] - lo[d]) / ext : 0.0;
                q[d] = (uint32_t)std::min(1023.0, std::max(0.0, t * 1023.0));
            }
            key[i - 1] = {((uint32_t)group[i] << 30) | hilbert10(q[0], q[1], q[2]), i};
        }
        std::stable_sort(key.begin(), key.end());
        for (int r = 0; r < neles; r++) perm[key[r].second] = r;
    }
    // reference id (1-based, this case) -> slot of the handle: elements
    // after the earlier cases' elements, ghosts after all elements and the
    // earlier cases' ghosts (a single case keeps ghost g at neles + g; the
    // aliased ids of a merged mesh are element ids and map as such)
    auto map = [&](int id1) -> int { return id1 <= neles ? E0 + perm[id1] : Etot + G0 + (id1 - neles - 1); };
    for (int i = 1; i <= neles; i++) L.perm[E0 + i - 1] = E0 + perm[i];
    for (int g = 0; g < nghosts; g++) L.ghost_id[G0 + g] = map(gid[g]);
    cr.cell1 = E0 + perm[1];

    // --- device layout ---
    std::vector<int>& hnc = L.nc; std::vector<int>& hsnb = L.snb; std::vector<int>& hib = L.ib;
    std::vector<unsigned>& hfk = L.fk;
    std::vector<double>& hx = L.x; std::vector<double>& hy = L.y; std::vector<double>& hz = L.z;
    std::vector<double>& hvol = L.vol; std::vector<double>& hdl = L.dl; std::vector<double>& hdd = L.dd;
    std::vector<double>& hsc = L.sc; std::vector<double>& hfch = L.fch; std::vector<double>& hfcv = L.fcv;
    std::vector<double>& hla = L.la; std::vector<double>& hlb = L.lb;
    std::vector<int> slot_parent(ntot + 1, 0);
    for (int g = 0; g < nghosts; g++) slot_parent[gid[g]] = gpar[g];
    // slots t = map(i) are distinct for distinct i on meshes without aliased
    // ghost ids; aliased meshes keep the sequential order
#pragma omp parallel for schedule(static) if (!cr.aliased)
    for (int i = 1; i <= ntot; i++) {
        int t = map(i);
        hx[t] = xcel[i]; hy[t] = ycel[i]; hz[t] = zcel[i]; hvol[t] = vol[i]; hdd[t] = dd[i];
        if (i <= neles) {
            hdl[t] = dl[i];
            hib[t] = iblank[i];
            unsigned fk = 0;
            for (int k = 0; k < 4; k++) {
                int nb = nc[k][i];
                hnc[k * ld + t] = map(nb);
                int snb = nb;
                if (!cr.aliased && nb > neles) snb = slot_parent[nb];
                hsnb[k * ld + t] = cr.aliased ? map(nb) : map(snb);
                int nt = 0;
                if (nb > neles && nb <= neles + nghosts) nt = gtyp[nb - neles - 1];
                unsigned kind = 0;
                if (nt == 5) kind |= FK_WALL;
                if (nb <= neles || nb > neles + nghosts) kind |= FK_RECON;
                fk |= kind << (4 * k);
            }
            hfk[t] = fk;
            for (int k = 0; k < 12; k++) {
                hsc[k * ld + t] = SC(k, i); hfch[k * ld + t] = FCH(k, i); hfcv[k * ld + t] = FCV(k, i);
            }
            for (int k = 0; k < NLSQ; k++) { hla[k * ld + t] = LA(k, i); hlb[k * ld + t] = LB(k, i); }
        } else {
            for (int k = 0; k < 4; k++) { hnc[k * ld + t] = map(nc[k][i]); hsnb[k * ld + t] = map(nc[k][i]); }
        }
    }
    for (int g = 0; g < nghosts; g++) {
        L.gpar[G0 + g] = map(gpar[g]); L.gid[G0 + g] = map(gid[g]); L.gtyp[G0 + g] = gtyp[g];
    }
    return HP_OK;
}


extern "C" int hp_create_batch(const hp_mesh* meshes, int32_t ncase, const hp_params* params, hp_handle** out) {
    g_create_error.clear();
    if (!meshes || !params || !out || ncase < 1) return fail(nullptr, HP_E_ARG, "null argument or no case");
    *out = nullptr;
    if (params->myflux < 1 || params->myflux > 3)
        return fail(nullptr, HP_E_ARG, "myflux must be 1 (HLLC-Zien), 2 (HLLC-Batten) or 3 (Jameson)");
    if (params->myorder != 1 && params->myorder != 2)
        return fail(nullptr, HP_E_ARG, "myorder must be 1 or 2");
    if (params->block_size != 0 && (params->block_size < 64 || params->block_size > 512 || params->block_size % 32))
        return fail(nullptr, HP_E_ARG, "block_size must be 0 or a multiple of 32 in [64, 512]");
    if (params->use_graph < 0 || params->use_graph > 2)
        return fail(nullptr, HP_E_ARG, "use_graph must be 0 (launches), 1 (graph) or 2 (fused step)");
    if (params->face_mode < 0 || params->face_mode > 3)
        return fail(nullptr, HP_E_ARG, "face_mode must be 0 (face records), 1 (each side), 2 (colouring) or 3 (atomics)");
    if (params->wall_fp64_layers < 0) return fail(nullptr, HP_E_ARG, "wall_fp64_layers must be >= 0");
    if (params->five_phase) {
        if (!(params->rhoq > 0 && params->rhor > 0 && params->rhos > 0 && params->radq > 0 && params->radr > 0 &&
              params->rads > 0))
            return fail(nullptr, HP_E_ARG, "five-phase model: rhoq, rhor, rhos, radq, radr, rads must be positive");
        if (params->precision == HP_PREC_FP32)
            return fail(nullptr, HP_E_UNSUPPORTED, "five-phase model: not in the all-FP32 variant");
    }
    long long etot = 0, gtot = 0;
    for (int c = 0; c < ncase; c++) {
        const hp_mesh* mesh = meshes + c;
        const std::string tag = ncase > 1 ? "case " + std::to_string(c) + ": " : "";
        if (mesh->pghosts != 0)
            return fail(nullptr, HP_E_UNSUPPORTED,
                        tag + "proc_bc partition ghosts: give a partitioned mesh's parts halo elements instead "
                              "(hydraphase.partition, hp_set_halo)");
        if (mesh->nodes <= 0 || mesh->neles <= 0 || mesh->nghosts < 0 || !mesh->x || !mesh->y || !mesh->z ||
            !mesh->elem || (mesh->nghosts > 0 && !mesh->ghost))
            return fail(nullptr, HP_E_ARG, tag + "empty or incomplete mesh");
        etot += mesh->neles;
        gtot += mesh->nghosts;
    }
    if (etot + gtot > 2000000000LL) return fail(nullptr, HP_E_ARG, "more than 2e9 cells in one handle");
    auto* h = new hp_handle();
    h->prm = *params;
    h->ncase = ncase;
    Layout L((int)etot, (int)gtot);
    int e0 = 0, g0 = 0;
    for (int c = 0; c < ncase; c++) {
        CaseRange cr;
        cr.e0 = e0; cr.ne = meshes[c].neles; cr.g0 = g0; cr.ng = meshes[c].nghosts;
        std::string err;
        int rc = fill_case(meshes + c, params, L, cr, err);
        if (rc != HP_OK) {
            delete h;
            return fail(nullptr, rc, (ncase > 1 ? "case " + std::to_string(c) + ": " : "") + err);
        }
        if (cr.aliased && ncase > 1) {
            delete h;
            return fail(nullptr, HP_E_UNSUPPORTED, "case " + std::to_string(c) +
                                                       ": aliased ghost ids cannot share a batch");
        }
        h->cases.push_back(cr);
        e0 += cr.ne;
        g0 += cr.ng;
    }
    h->aliased = h->cases[0].aliased;
    h->neles = L.neles; h->nghosts = L.nghosts; h->ntot = L.neles + L.nghosts; h->ld = L.ld;
    h->perm = std::move(L.perm);
    h->ghost_id = std::move(L.ghost_id);

    // --- parameters ---
    const hp_params& p = h->prm;
    const int neles = L.neles, nghosts = L.nghosts, ntot = neles + nghosts;
    const long long ld = L.ld;
    DevParams& P = h->dp;
    P.gamag = p.gamag; P.gamap = p.gamap; P.pinf = p.pinf; P.cpp = p.cpp; P.cpg = p.cpg; P.prg = p.prg;
    P.rrg = 287.0; P.prp = 10.0;
    P.emin = p.epslnmin; P.emax = p.epslnmax; P.phipzero = p.phipzero;
    P.ugmin = p.ugmin; P.vgmin = p.vgmin; P.wgmin = p.wgmin;
    P.upmin = p.upmin; P.vpmin = p.vpmin; P.wpmin = p.wpmin;
    P.tgmin = p.tgmin; P.tpmin = p.tpmin; P.pmin = p.pmin;
    P.as = p.as; P.ts = p.ts;
    P.c23 = (double)(2.00f / 3.00f); P.co2 = (double)(1.00f / 16.00f); P.co4 = (double)(1.00f / 1024.00f);
    P.fsd = 4.0 * p.surfacetension / p.diap;
    P.cfl = p.cfl; P.venkat_k = p.venkat_k > 0 ? p.venkat_k : 0.3; P.twall = p.twall; P.amup = 0.001;
    P.rk_scheme = p.rk_scheme; P.inviscid = p.inviscid; P.myorder = p.myorder; P.myflux = p.myflux;
    P.five_phase = p.five_phase ? 1 : 0;
    if (P.five_phase) {
        if (h->aliased) { delete h; return fail(nullptr, HP_E_UNSUPPORTED, "five-phase model: aliased ghost ids"); }
        const double rho[3] = {p.rhoq, p.rhor, p.rhos}, rad[3] = {p.radq, p.radr, p.rads};
        for (int d = 0; d < 3; d++) {   // src/main.F90:352-354
            P.rhod[d] = rho[d];
            P.radd[d] = rad[d];
            P.vold[d] = (4.0 / 3.0) * 3.1415926 * (rad[d] * rad[d] * rad[d]);
        }
        h->neq = 22;
    }
    P.r_emm = 1.0 / (P.emax - P.emin);
    P.r_gm1 = 1.0 / (P.gamag - 1.0);
    P.r_gamap = 1.0 / P.gamap;
    P.r_prg = 1.0 / P.prg;
    P.r_prp = 1.0 / P.prp;
    P.nstage = p.rk_scheme == 0 ? 4 : 3;
    switch (p.precision) {
        case HP_PREC_FP64_PARITY: h->var = &variant_fp64_parity; break;
        case HP_PREC_FP64: h->var = &variant_fp64; break;
        case HP_PREC_MIXED: h->var = &variant_mixed; break;
        case HP_PREC_FP32:
            if (h->aliased) { delete h; return fail(nullptr, HP_E_UNSUPPORTED, "fp32 variant: aliased ghost ids"); }
            h->var = &variant_fp32;
            break;
        default: delete h; return fail(nullptr, HP_E_ARG, "unknown precision mode");
    }

    // --- device memory: one arena ---
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { delete h; return fail(nullptr, HP_E_CUDA, "no CUDA device"); }
    h->device = dev;
    const size_t D = sizeof(double), I = sizeof(int), gb = h->var->grad_bytes;
    // --- unique faces for the face-based fluxes of the FP32-arithmetic
    // variants: a face belongs to its lower-id element (or to its element
    // when the other side is a ghost); meshes whose neighbour lists are not
    // mutual, and aliased meshes, keep the cell-centric fluxes ---
    std::vector<int> hf_i, hf_code, hcface;
    if (gb != D && !h->aliased && h->prm.face_mode != 1) {
        hcface.assign(4 * (size_t)ld, 0);
        bool mutual = true;
        for (int t = 0; t < neles && mutual; t++)
            for (int f = 0; f < 4; f++) {
                const int j = L.nc[(size_t)f * ld + t];
                if (j < neles && j < t) continue;
                int fj = -1;
                if (j < neles)
                    for (int k = 0; k < 4; k++)
                        if (L.nc[(size_t)k * ld + j] == t) { fj = k; break; }
                if (j < neles && fj < 0) { mutual = false; break; }
                const int id = (int)hf_i.size();
                hf_i.push_back(t);
                hf_code.push_back(f);
                hcface[(size_t)f * ld + t] = id + 1;
                if (j < neles) hcface[(size_t)fj * ld + j] = -(id + 1);
            }
        if (!mutual) { hf_i.clear(); hf_code.clear(); hcface.clear(); }
    }
    const int nface = (int)hf_i.size();
    // face mode 2: greedy colouring of the faces in id order, so that no two
    // faces of a colour touch the same element (tets: at most 7 colours)
    std::vector<int> hf_color;
    int ncolor = 0, fcoff[33] = {0};
    if (nface > 0 && h->prm.face_mode == 2) {
        std::vector<uint32_t> used((size_t)ld, 0u);
        std::vector<int> col(nface);
        for (int t = 0; t < nface; t++) {
            const int i = hf_i[t], j = L.nc[(size_t)hf_code[t] * ld + i];
            uint32_t busy = used[i] | (j < neles ? used[j] : 0u);
            int c = 0;
            while (c < 31 && (busy & (1u << c))) c++;   // a tet face meets at most 6 others
            col[t] = c;
            used[i] |= 1u << c;
            if (j < neles) used[j] |= 1u << c;
            ncolor = std::max(ncolor, c + 1);
        }
        for (int t = 0; t < nface; t++) fcoff[col[t] + 1]++;
        for (int c = 0; c < ncolor; c++) fcoff[c + 1] += fcoff[c];
        hf_color.assign(nface, 0);
        std::vector<int> pos(fcoff, fcoff + ncolor);
        for (int t = 0; t < nface; t++) hf_color[pos[col[t]]++] = t;
    } else if (nface > 0 && h->prm.face_mode == 3) {
        hf_color.assign(nface, 0);   // unused by the atomic scatter; keeps the array defined
    }
    // --- FP64 wall layers of the FP32-arithmetic variants ---
    std::vector<int> hwall, hgwall;
    std::vector<unsigned char> hwclass;
    if (gb != D && p.wall_fp64_layers > 0) {
        if (h->aliased) {
            delete h;
            return fail(nullptr, HP_E_UNSUPPORTED, "FP64 wall layers: aliased ghost ids");
        }
        wall_layers(L, neles, nghosts, ld, p.wall_fp64_layers, hwall, hgwall, hwclass);
    }
    h->nwall = (int)hwall.size();
    h->ngwall = (int)hgwall.size();
    // with the layer-first cell order (one case, renumbered) both lists are
    // the leading cells 0, 1, ...: the layer kernels then run as whole-mesh
    // launches over that prefix
    {
        bool pre = h->nwall > 0;
        for (int k = 0; k < h->ngwall && pre; k++) pre = hgwall[k] == k;
        for (int k = 0; k < h->nwall && pre; k++) pre = hwall[k] == k;
        h->wprefix = pre ? 1 : 0;
    }
    Arena& A = h->arena;
    auto plan = [&](Arena& a) { plan_arena(h, a, neles, nghosts, ld, gb, ncase, nface); };
    Arena probe;
    plan(probe);
    A.size = probe.used + 256;
    // The arenas come from the device's stream-ordered pool.  Keeping freed
    // arenas in the pool (release threshold: never) lets a server that
    // creates and destroys cases reuse their memory instead of mapping new
    // memory for each case; memory the pool holds but does not use counts
    // as free below.
    cudaMemPool_t pool = nullptr;
    size_t pool_spare = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX, reserved = 0, used = 0;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
            pool_spare = (size_t)(reserved - used);
    }
    cudaGetLastError();
    size_t freeb = 0, totalb = 0;
    cudaMemGetInfo(&freeb, &totalb);
    freeb += pool_spare;
    if (A.size > freeb) {
        delete h;
        return fail(nullptr, HP_E_NOMEM, "case needs " + std::to_string(A.size >> 20) + " MiB, " +
                                             std::to_string(freeb >> 20) + " MiB free");
    }
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return fail(nullptr, HP_E_CUDA, "stream creation failed");
    }
    cudaStream_t st = h->stream;
    // stream-ordered allocation: creating or destroying a case does not
    // synchronise the device under the other cases' work
    if (cudaMallocAsync((void**)&A.base, A.size, st) != cudaSuccess) {
        cudaGetLastError();
        cudaStreamDestroy(st);
        delete h;
        return fail(nullptr, HP_E_NOMEM, "allocation of the case arena failed");
    }
    A.used = 0;
    plan(A);
    DevMesh& m = h->dm;
    m.neles = neles; m.nghosts = nghosts; m.ntot = ntot; m.aliased = h->aliased; m.ld = ld;
    m.ncase = ncase;
    if (ncase == 1) m.cid = nullptr;
    auto up = [&](const void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice, st);
    };
    cudaError_t e = cudaMemsetAsync(A.base, 0, A.size, st);
    if (e == cudaSuccess) e = up(m.nc, L.nc.data(), 4 * ld * I);
    if (e == cudaSuccess) e = up(m.snb, L.snb.data(), 4 * ld * I);
    if (e == cudaSuccess) e = up(m.fk, L.fk.data(), ld * sizeof(unsigned));
    if (e == cudaSuccess) e = up(m.iblank, L.ib.data(), ld * I);
    if (e == cudaSuccess) e = up(m.xc, L.x.data(), ld * D);
    if (e == cudaSuccess) e = up(m.yc, L.y.data(), ld * D);
    if (e == cudaSuccess) e = up(m.zc, L.z.data(), ld * D);
    if (e == cudaSuccess) e = up(m.vol, L.vol.data(), ld * D);
    // the limiter's (K dl)^3 with the host's pow (src/sr_VK.F90:34): a
    // device cube rounds differently from pow in rare near-tie cases
#pragma omp parallel for schedule(static)
    for (long long t = 0; t < ld; t++) L.eps2[t] = std::pow(P.venkat_k * L.dl[t], 3.0);
    if (e == cudaSuccess) e = up(m.dl, L.dl.data(), ld * D);
    if (e == cudaSuccess) e = up(m.eps2, L.eps2.data(), ld * D);
    if (e == cudaSuccess) e = up(m.dd, L.dd.data(), ld * D);
    if (e == cudaSuccess) e = up(m.sc, L.sc.data(), 12 * ld * D);
    if (e == cudaSuccess) e = up(m.fch, L.fch.data(), 12 * ld * D);
    if (e == cudaSuccess) e = up(m.fcv, L.fcv.data(), 12 * ld * D);
    // neighbour centroid differences of the FP64 gradient and source LSQ
    // (the subtraction the kernels would do on the gathered centroids)
    std::vector<double> hdxn(12 * (size_t)ld, 0.0);
#pragma omp parallel for schedule(static)
    for (long long t = 0; t < neles; t++)
        for (int f = 0; f < 4; f++) {
            const int j = L.nc[(size_t)f * ld + t];
            hdxn[(size_t)(3 * f) * ld + t] = L.x[j] - L.x[t];
            hdxn[(size_t)(3 * f + 1) * ld + t] = L.y[j] - L.y[t];
            hdxn[(size_t)(3 * f + 2) * ld + t] = L.z[j] - L.z[t];
        }
    if (e == cudaSuccess) e = up(m.dxn, hdxn.data(), 12 * ld * D);
    if (e == cudaSuccess) e = up(m.lsqa, L.la.data(), NLSQ * ld * D);
    if (e == cudaSuccess) e = up(m.lsqb, L.lb.data(), NLSQ * ld * D);
    if (e == cudaSuccess && nghosts) e = up(m.g_par, L.gpar.data(), nghosts * (size_t)I);
    if (e == cudaSuccess && nghosts) e = up(m.g_id, L.gid.data(), nghosts * (size_t)I);
    if (e == cudaSuccess && nghosts) e = up(m.g_type, L.gtyp.data(), nghosts * (size_t)I);
    if (e == cudaSuccess) e = up(h->d_perm, h->perm.data(), neles * (size_t)I);
    if (e == cudaSuccess && nghosts) e = up(h->d_gid, h->ghost_id.data(), nghosts * (size_t)I);
    if (e == cudaSuccess && nface) e = up(m.f_i, hf_i.data(), nface * (size_t)I);
    if (e == cudaSuccess && nface) e = up(m.f_code, hf_code.data(), nface * (size_t)I);
    if (e == cudaSuccess && nface) e = up(m.cface, hcface.data(), 4 * (size_t)ld * I);
    m.face_mode = nface > 0 ? h->prm.face_mode : 0;
    m.ncolor = ncolor;
    for (int c = 0; c <= ncolor; c++) m.fcoff[c] = fcoff[c];
    if (e == cudaSuccess && nface && m.fcolor) e = up(m.fcolor, hf_color.data(), nface * (size_t)I);
    if (e == cudaSuccess && h->nwall) e = up(m.wcells, hwall.data(), hwall.size() * (size_t)I);
    if (e == cudaSuccess && h->nwall) e = up(m.gcells, hgwall.data(), hgwall.size() * (size_t)I);
    if (e == cudaSuccess && h->nwall) e = up(m.wclass, hwclass.data(), (size_t)ld);
    // hwall, hgwall and hwclass are local vectors
    if (e == cudaSuccess && h->nwall) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && ncase > 1) {
        std::vector<int> cid(neles);
        for (int c = 0; c < ncase; c++)
            for (int i = 0; i < h->cases[c].ne; i++) cid[h->cases[c].e0 + i] = c;
        e = up(m.cid, cid.data(), neles * (size_t)I);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // cid is a local vector
    }
    if (e == cudaSuccess) e = cudaMallocHost((void**)&h->h_diag, (size_t)h->max_diag * 8 * D * ncase);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&h->h_scal, sizeof(DevScalars));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&h->h_sync, sizeof(GridSync));
    // the fused step: plain two-phase meshes on a device with cooperative
    // launch, in the parity variant.  The variants built with FMA contraction
    // keep the graph: the fused kernel is another compilation of the same
    // bodies, whose contractions (and so roundings) may differ from those of
    // the separate kernels, and a case must give the same result whichever
    // way it runs (alone or in a batch of another size class).
    if (e == cudaSuccess && h->prm.use_graph == 2 && h->var == &variant_fp64_parity && !h->aliased &&
        h->neq == 10 && h->nwall == 0 && P.myflux != 3 && !(m.nface > 0 && m.face_mode >= 2)) {
        int coop = 0;
        if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && coop)
            h->fused = h->var->fused_grid(m, P);
        cudaGetLastError();
    }
    for (int c = 0; c < ncase && e == cudaSuccess; c++) {
        DevScalars s0{};
        double v = 1.0e8;
        std::memcpy(&s0.dtmin_bits, &v, 8);
        s0.cell1 = h->cases[c].cell1;
        *h->h_scal = s0;
        e = cudaMemcpyAsync(h->ds.s + c, h->h_scal, sizeof s0, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) {
        std::string msg = std::string("device upload failed: ") + cudaGetErrorString(e);
        hp_destroy(h);
        return fail(nullptr, HP_E_CUDA, msg);
    }
    *out = h;
    return HP_OK;
}


extern "C" int hp_create(const hp_mesh* mesh, const hp_params* params, hp_handle** out) {
    return hp_create_batch(mesh, 1, params, out);
}

static int output_join(OutSlot& s) {
    if (!s.ticket) return HP_OK;
    if (s.writer.joinable()) s.writer.join();
    s.ticket = 0;
    return s.rc;
}

extern "C" int hp_destroy(hp_handle* h) {
    if (!h) return HP_OK;
    for (OutSlot& o : h->out) {
        output_join(o);
        if (o.ready) cudaEventDestroy(o.ready);
        if (o.copied) cudaEventDestroy(o.copied);
        if (o.d_buf) cudaFree(o.d_buf);
        if (o.h_buf) cudaFreeHost(o.h_buf);
    }
    if (h->ostream) cudaStreamDestroy(h->ostream);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->d_overset) cudaFreeAsync(h->d_overset, h->stream);
    if (h->d_halo) cudaFreeAsync(h->d_halo, h->stream);
    if (h->d_xlist) cudaFreeAsync(h->d_xlist, h->stream);
    if (h->arena.base) {
        cudaFreeAsync(h->arena.base, h->stream);
        cudaStreamSynchronize(h->stream);
    }
    if (h->h_diag) cudaFreeHost(h->h_diag);
    if (h->h_scal) cudaFreeHost(h->h_scal);
    if (h->h_sync) cudaFreeHost(h->h_sync);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return HP_OK;
}

// Upload cu (elements, reference order, column-major) and set cn = cu.
// --- state transfer ----------------------------------------------------------
// Caller arrays are in reference order (10 x neles, column-major); the device
// keeps internal (renumbered) order with leading dimension ld.  Transfers go
// straight between the caller's buffer and a device staging area (cn1, which
// holds no live data between steps: every step writes it before reading it),
// and the permutation runs on the device.
namespace {
struct Cols6 { int c[6]; };

// dst[k*ld + idx[i]] = src[k*n + i], k < ncol
__global__ void k_scatter_cols(const double* __restrict__ src, int n, int ncol, const int* __restrict__ idx,
                               double* __restrict__ dst, long long ld) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * ncol) return;
    int k = (int)(t / n), i = (int)(t - (long long)k * n);
    dst[(size_t)k * ld + idx[i]] = src[(size_t)k * n + i];
}
// dst[k*n + i] = src[(col0 + k)*ld + idx[i]], k < ncol
__global__ void k_gather_cols(const double* __restrict__ src, long long ld, int col0, int n, int ncol,
                              const int* __restrict__ idx, double* __restrict__ dst) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * ncol) return;
    int k = (int)(t / n), i = (int)(t - (long long)k * n);
    dst[(size_t)k * n + i] = src[(size_t)(col0 + k) * ld + idx[i]];
}
// ghost primitives into their columns of pr.  One thread per column walks
// the ghost list in order, so repeated ghost ids keep the last value, as the
// reference's sequential restart read does (src/main.F90:433-438).
__global__ void k_scatter_ghost_prims(const double* __restrict__ src, int ng, Cols6 cols, const int* __restrict__ gid,
                                      double* __restrict__ pr, long long ld, int ordered) {
    if (ordered) {
        int v = threadIdx.x;
        if (blockIdx.x != 0 || v >= 6) return;
        for (int g = 0; g < ng; g++) pr[(size_t)cols.c[v] * ld + gid[g]] = src[(size_t)v * ng + g];
        return;
    }
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6LL * ng) return;
    int v = (int)(t / ng), g = (int)(t - (long long)v * ng);
    pr[(size_t)cols.c[v] * ld + gid[g]] = src[(size_t)v * ng + g];
}
__global__ void k_gather_ghost_prims(const double* __restrict__ pr, long long ld, Cols6 cols, int ng,
                                     const int* __restrict__ gid, double* __restrict__ dst) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6LL * ng) return;
    int v = (int)(t / ng), g = (int)(t - (long long)v * ng);
    dst[(size_t)v * ng + g] = pr[(size_t)cols.c[v] * ld + gid[g]];
}
// p[k*ld + start + i] = v and dst[k*ld + start + i] = src[k*ld + start + i],
// k < ncol, i < count (one case's element or ghost range)
__global__ void k_fill_cols(double* __restrict__ p, long long ld, int ncol, int start, int count, double v) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)count * ncol) return;
    int k = (int)(t / count), i = (int)(t - (long long)k * count);
    p[(size_t)k * ld + start + i] = v;
}
__global__ void k_copy_cols(double* __restrict__ dst, const double* __restrict__ src, long long ld, int ncol, int start,
                            int count) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)count * ncol) return;
    int k = (int)(t / count), i = (int)(t - (long long)k * count);
    dst[(size_t)k * ld + start + i] = src[(size_t)k * ld + start + i];
}
inline unsigned blocks_for(long long n, int b) { return (unsigned)((n + b - 1) / b); }
const Cols6 GHOST_COLS = {{P_UG, P_VG, P_WG, P_PG, P_TG, P_ROG}};
}  // namespace

// One case's state: its element slots get the caller's cu in internal order,
// its ghost slots zero; cn = cu on both ranges; its primitive slots zero
// except the restart's ghost values; its scalars restart at `time`.
static int upload_state(hp_handle* h, int c, double time, const double* cu_elem, const double* ghost_prims) {
    const CaseRange& cr = h->cases[c];
    const long long ld = h->ld;
    const int ne = cr.ne, ng = cr.ng, gs = h->neles + cr.g0;
    cudaStream_t st = h->stream;
    CUDA_OK(h, cudaStreamSynchronize(st));
    const int nq = h->neq;
    CUDA_OK(h, cudaMemcpyAsync(h->ds.cn1, cu_elem, nq * (size_t)ne * sizeof(double), cudaMemcpyHostToDevice, st));
    if (ng) k_fill_cols<<<blocks_for((long long)nq * ng, 256), 256, 0, st>>>(h->ds.cu, ld, nq, gs, ng, 0.0);
    k_scatter_cols<<<blocks_for((long long)nq * ne, 256), 256, 0, st>>>(h->ds.cn1, ne, nq, h->d_perm + cr.e0,
                                                                         h->ds.cu, ld);
    k_copy_cols<<<blocks_for((long long)nq * ne, 256), 256, 0, st>>>(h->ds.cn, h->ds.cu, ld, nq, cr.e0, ne);
    if (ng) k_copy_cols<<<blocks_for((long long)nq * ng, 256), 256, 0, st>>>(h->ds.cn, h->ds.cu, ld, nq, gs, ng);
    // primitives: zero, then the restart's ghost values (src/main.F90:433-438)
    k_fill_cols<<<blocks_for((long long)NPR * ne, 256), 256, 0, st>>>(h->ds.pr, ld, NPR, cr.e0, ne, 0.0);
    if (ng) k_fill_cols<<<blocks_for((long long)NPR * ng, 256), 256, 0, st>>>(h->ds.pr, ld, NPR, gs, ng, 0.0);
    CUDA_OK(h, cudaGetLastError());
    if (ghost_prims && ng) {
        CUDA_OK(h, cudaMemcpyAsync(h->d_gstage, ghost_prims, 6 * (size_t)ng * sizeof(double),
                                   cudaMemcpyHostToDevice, st));
        if (h->aliased)
            k_scatter_ghost_prims<<<1, 32, 0, st>>>(h->d_gstage, ng, GHOST_COLS, h->d_gid + cr.g0, h->ds.pr, ld, 1);
        else
            k_scatter_ghost_prims<<<blocks_for(6LL * ng, 256), 256, 0, st>>>(h->d_gstage, ng, GHOST_COLS,
                                                                             h->d_gid + cr.g0, h->ds.pr, ld, 0);
        CUDA_OK(h, cudaGetLastError());
    }
    DevScalars s0{};
    double v = 1.0e8;
    std::memcpy(&s0.dtmin_bits, &v, 8);
    s0.time = time;
    s0.cell1 = cr.cell1;
    *h->h_scal = s0;
    CUDA_OK(h, cudaMemcpyAsync(h->ds.s + c, h->h_scal, sizeof s0, cudaMemcpyHostToDevice, st));
    CUDA_OK(h, cudaStreamSynchronize(st));
    h->started = false;
    if (h->state_set.size() != (size_t)h->ncase) h->state_set.assign(h->ncase, 0);
    h->state_set[c] = 1;
    h->have_state = std::all_of(h->state_set.begin(), h->state_set.end(), [](char x) { return x != 0; });
    return HP_OK;
}

// A batch's cases step together from their first step on; a case's state can
// be replaced only before that (a single case can be reset at any time).
static int check_settable(hp_handle* h, int c) {
    if (c < 0 || c >= h->ncase) return fail(h, HP_E_ARG, "case index out of range");
    if (h->ncase > 1 && h->started)
        return fail(h, HP_E_STATE, "the cases of a batch are set before its first step");
    return HP_OK;
}

extern "C" int hp_init_uniform(hp_handle* h) {
    if (!h) return HP_E_ARG;
    const hp_params& p = h->prm;
    const double rrg = 287.0;
    // src/main.F90:397-402 and src/sr_init_cond.F90:177-195
    double rogmin = p.pmin / (rrg * p.tgmin);
    double ropmin = (p.pmin + p.pinf) * p.gamap / ((p.gamap - 1.0) * p.cpp * p.tpmin);
    double egtmin = rrg * p.tgmin / (p.gamag - 1.0) + 0.5 * (sq(p.ugmin) + sq(p.vgmin) + sq(p.wgmin));
    double eptmin = (p.cpp * p.tpmin) / p.gamap + p.pinf / ropmin + 0.5 * (sq(p.upmin) + sq(p.vpmin) + sq(p.wpmin));
    int rc = check_settable(h, 0);
    if (rc) return rc;
    std::vector<double> cu;
    double phip = p.epslninf, phig = 1 - p.epslninf;
    double v[10] = {phig * rogmin, phig * rogmin * p.ugmin, phig * rogmin * p.vgmin, phig * rogmin * p.wgmin,
                    phig * rogmin * egtmin, phip * ropmin, phip * ropmin * p.upmin, phip * ropmin * p.vpmin,
                    phip * ropmin * p.wpmin, phip * ropmin * eptmin};
    double vq[12] = {};
    if (h->neq == 22) {   // src/sr_init_cond.F90:180-208
        phig = 1 - phip - p.epslninf - p.epslninf - p.epslninf;
        v[0] = phig * rogmin; v[1] = phig * rogmin * p.ugmin; v[2] = phig * rogmin * p.vgmin;
        v[3] = phig * rogmin * p.wgmin; v[4] = phig * rogmin * egtmin;
        const double rho[3] = {p.rhoq, p.rhor, p.rhos}, ini[3] = {p.phiqinit, p.phirinit, p.phisinit};
        for (int d = 0; d < 3; d++) {
            vq[4 * d] = ini[d] * rho[d];
            vq[4 * d + 1] = ini[d] * rho[d] * p.upmin;
            vq[4 * d + 2] = ini[d] * rho[d] * p.vpmin;
            vq[4 * d + 3] = ini[d] * rho[d] * p.wpmin;
        }
    }
    for (int c = 0; c < h->ncase; c++) {
        const int ne = h->cases[c].ne;
        cu.assign(h->neq * (size_t)ne, 0.0);
        for (int k = 0; k < h->neq; k++)
            for (int i = 0; i < ne; i++) cu[(size_t)k * ne + i] = k < 10 ? v[k] : vq[k - 10];
        rc = upload_state(h, c, 0.0, cu.data(), nullptr);
        if (rc) return rc;
    }
    return HP_OK;
}

extern "C" int hp_set_state(hp_handle* h, double time, const double* cu_elem, const double* ghost_prims) {
    return hp_set_state_case(h, 0, time, cu_elem, ghost_prims);
}

extern "C" int hp_set_state_case(hp_handle* h, int32_t c, double time, const double* cu_elem,
                                 const double* ghost_prims) {
    if (!h || !cu_elem) return HP_E_ARG;
    int rc = check_settable(h, c);
    if (rc) return rc;
    return upload_state(h, c, time, cu_elem, ghost_prims);
}

// zero every case's per-call step counter (the row index of its diagnostics)
static cudaError_t reset_step_counters(hp_handle* h) {
    return cudaMemset2DAsync(&h->ds.s->step_in_call, sizeof(DevScalars), 0, sizeof(int), h->ncase, h->stream);
}

// exchange points of a part on several GPUs: the caller's callback with the
// handle's stream
static void exchange_point(void* ctx, int point) {
    hp_handle* h = static_cast<hp_handle*>(ctx);
    h->xfn(h->xuser, point, static_cast<void*>(h->stream));
}

static int run_steps(hp_handle* h, int n) {
    cudaStream_t st = h->stream;
    const int block = h->prm.block_size;
    if (!h->started) {
        h->var->enqueue_start(h->dm, &h->ds, h->dp, st, block, nullptr);
        h->started = true;
    }
    // the fused step needs a plain mesh: no exchange callback, overset
    // fringe or halo (set after creation), nothing else it leaves out
    const bool fused = h->prm.use_graph == 2 && h->fused > 0 && !h->xfn && h->dm.nfringe == 0 && h->dm.nhalo == 0;
    if (fused) {
        for (int k = 0; k < n; k++)
            CUDA_OK(h, h->var->enqueue_fused(h->dm, &h->ds, h->dp, st, h->d_sync, h->fused));
    } else if (h->xfn) {
        const StepHook hook{nullptr, nullptr, exchange_point, h};
        for (int k = 0; k < n; k++) h->var->enqueue_step(h->dm, &h->ds, h->dp, st, block, &hook);
    } else if (h->prm.use_graph) {
        if (!h->gexec) {
            CUDA_OK(h, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            h->var->enqueue_step(h->dm, &h->ds, h->dp, st, block, nullptr);
            CUDA_OK(h, cudaStreamEndCapture(st, &h->graph));
            CUDA_OK(h, cudaGraphInstantiate(&h->gexec, h->graph, 0));
        }
        for (int k = 0; k < n; k++) CUDA_OK(h, cudaGraphLaunch(h->gexec, st));
    } else {
        for (int k = 0; k < n; k++) h->var->enqueue_step(h->dm, &h->ds, h->dp, st, block, nullptr);
    }
    CUDA_OK(h, cudaGetLastError());
    return HP_OK;
}

// After fused steps that the caller waits for anyway: a grid barrier whose
// wait gave up (bounded spin) is reported, and the barrier is reset.
static int check_fused(hp_handle* h) {
    if (h->fused <= 0 || h->prm.use_graph != 2) return HP_OK;
    CUDA_OK(h, cudaMemcpyAsync(h->h_sync, h->d_sync, sizeof(GridSync), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OK(h, cudaStreamSynchronize(h->stream));
    if (h->h_sync->err == 0) return HP_OK;
    CUDA_OK(h, cudaMemsetAsync(h->d_sync, 0, sizeof(GridSync), h->stream));
    return fail(h, HP_E_CUDA, "fused step: a grid barrier wait gave up; the step did not complete");
}

extern "C" int hp_step(hp_handle* h, int32_t nsteps, hp_diag* diag) {
    if (!h || nsteps < 0) return HP_E_ARG;
    if (!h->have_state) return fail(h, HP_E_STATE, "hp_step before hp_init_uniform/hp_set_state");
    int done = 0;
    while (done < nsteps) {
        int chunk = std::min(nsteps - done, h->max_diag);
        CUDA_OK(h, reset_step_counters(h));
        int rc = run_steps(h, chunk);
        if (rc) return rc;
        if (diag) {
            // rows of case c start at c * max_diag on the device, at
            // c * nsteps in the caller's array
            for (int c = 0; c < h->ncase; c++)
                CUDA_OK(h, cudaMemcpyAsync(h->h_diag + (size_t)c * h->max_diag * 8,
                                           h->ds.diag + (size_t)c * h->max_diag * 8,
                                           (size_t)chunk * 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CUDA_OK(h, cudaStreamSynchronize(h->stream));
            if (int frc = check_fused(h)) return frc;
            for (int c = 0; c < h->ncase; c++)
                for (int k = 0; k < chunk; k++) {
                    const double* d = h->h_diag + ((size_t)c * h->max_diag + k) * 8;
                    hp_diag& o = diag[(size_t)c * nsteps + done + k];
                    o.time = d[0]; o.dt = d[1]; o.velmag = d[2];
                    for (int j = 0; j < 4; j++) o.diff[j] = d[3 + j];
                    o.nan_cells = d[7];
                }
        }
        done += chunk;
    }
    return HP_OK;
}

extern "C" int hp_step_timed(hp_handle* h, int32_t nsteps, double* device_ms) {
    if (!h || nsteps < 0 || !device_ms) return HP_E_ARG;
    if (!h->have_state) return fail(h, HP_E_STATE, "hp_step_timed before the state is set");
    cudaEvent_t a, b;
    CUDA_OK(h, cudaEventCreate(&a));
    CUDA_OK(h, cudaEventCreate(&b));
    if (!h->started) {   // the first step's start-of-step pass is not timed
        h->var->enqueue_start(h->dm, &h->ds, h->dp, h->stream, h->prm.block_size, nullptr);
        h->started = true;
    }
    CUDA_OK(h, reset_step_counters(h));
    CUDA_OK(h, cudaEventRecord(a, h->stream));
    int rc = run_steps(h, nsteps);
    CUDA_OK(h, cudaEventRecord(b, h->stream));
    CUDA_OK(h, cudaEventSynchronize(b));
    float ms = 0.f;
    CUDA_OK(h, cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *device_ms = ms;
    if (rc) return rc;
    return check_fused(h);
}

namespace {
struct ProfCtx {
    cudaStream_t st;
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;
    cudaError_t err = cudaSuccess;
};
void prof_mark(void* c, int kind) {
    auto* p = static_cast<ProfCtx*>(c);
    cudaEvent_t e;
    cudaError_t r = cudaEventCreate(&e);
    if (r == cudaSuccess) r = cudaEventRecord(e, p->st);
    if (r != cudaSuccess) { p->err = r; return; }
    p->ev.push_back(e);
    p->kind.push_back(kind);
}
}  // namespace

extern "C" int hp_profile_steps(hp_handle* h, int32_t nsteps, double* ms_per_kind, int64_t* launches_per_kind,
                                int32_t nkinds) {
    if (!h || nsteps <= 0 || !ms_per_kind || !launches_per_kind || nkinds < (int)KK_COUNT) return HP_E_ARG;
    if (!h->have_state) return fail(h, HP_E_STATE, "hp_profile_steps before the state is set");
    for (int k = 0; k < nkinds; k++) { ms_per_kind[k] = 0.0; launches_per_kind[k] = 0; }
    ProfCtx ctx;
    ctx.st = h->stream;
    StepHook hook{prof_mark, &ctx, h->xfn ? exchange_point : nullptr, h};
    if (!h->started) {
        h->var->enqueue_start(h->dm, &h->ds, h->dp, h->stream, h->prm.block_size, nullptr);
        h->started = true;
    }
    CUDA_OK(h, reset_step_counters(h));
    for (int k = 0; k < nsteps; k++) {
        h->var->enqueue_step(h->dm, &h->ds, h->dp, h->stream, h->prm.block_size, &hook);
        if (ctx.err != cudaSuccess) break;
    }
    CUDA_OK(h, ctx.err);
    CUDA_OK(h, cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i + 1 < ctx.ev.size(); i++) {
        int kd = ctx.kind[i];
        if (kd >= (int)KK_COUNT) continue;
        float ms = 0.f;
        CUDA_OK(h, cudaEventElapsedTime(&ms, ctx.ev[i], ctx.ev[i + 1]));
        ms_per_kind[kd] += ms;
        launches_per_kind[kd] += 1;
    }
    for (auto e : ctx.ev) cudaEventDestroy(e);
    return HP_OK;
}

extern "C" int hp_set_overset(hp_handle* h, const hp_overset* ov) {
    if (!h || !ov) return HP_E_ARG;
    if (h->neq == 22) return fail(h, HP_E_UNSUPPORTED, "five-phase model: no overset fringe tables");
    if (h->ncase != 1) return fail(h, HP_E_UNSUPPORTED, "overset tables: single-case handles only");
    const int nf = ov->nfringe, ne = h->neles;
    if (nf < 0 || (nf > 0 && (!ov->fringe || !ov->donor || !ov->weight)))
        return fail(h, HP_E_ARG, "overset table: missing arrays");
    // [fringe | donor column-major 4 x nf] ints, then [weight 4 x nf] doubles
    std::vector<int> iv(5 * (size_t)nf);
    std::vector<double> wv(4 * (size_t)nf);
    for (int f = 0; f < nf; f++) {
        const int e = ov->fringe[f];
        if (e < 1 || e > ne) return fail(h, HP_E_ARG, "overset table: fringe id out of range");
        iv[f] = h->perm[e - 1];
        for (int k = 0; k < 4; k++) {
            const int d = ov->donor[4 * (size_t)f + k];
            if (d < 1 || d > ne) return fail(h, HP_E_ARG, "overset table: donor id out of range");
            iv[(size_t)(1 + k) * nf + f] = h->perm[d - 1];
            wv[(size_t)k * nf + f] = ov->weight[4 * (size_t)f + k];
        }
    }
    cudaStream_t st = h->stream;
    if (h->d_overset) {
        CUDA_OK(h, cudaFreeAsync(h->d_overset, st));
        h->d_overset = nullptr;
    }
    h->dm.nfringe = 0;
    h->dm.fr = nullptr; h->dm.fdon = nullptr; h->dm.fw = nullptr;
    if (nf > 0) {
        const size_t ib = ((5 * (size_t)nf * sizeof(int)) + 255) & ~size_t(255);
        CUDA_OK(h, cudaMallocAsync(&h->d_overset, ib + 4 * (size_t)nf * sizeof(double), st));
        char* base = static_cast<char*>(h->d_overset);
        CUDA_OK(h, cudaMemcpyAsync(base, iv.data(), iv.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        CUDA_OK(h, cudaMemcpyAsync(base + ib, wv.data(), wv.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        h->dm.nfringe = nf;
        h->dm.fr = reinterpret_cast<const int*>(base);
        h->dm.fdon = reinterpret_cast<const int*>(base) + nf;
        h->dm.fw = reinterpret_cast<const double*>(base + ib);
    }
    CUDA_OK(h, cudaStreamSynchronize(st));
    // a captured step holds the mesh description it was launched with
    if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
    if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
    return HP_OK;
}

// a captured step holds the mesh description it was launched with
static void drop_graph(hp_handle* h) {
    if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
    if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
}

// Slot of element e (1-based, reference order) of case c; -1 if out of range.
static int slot_of(const hp_handle* h, int c, int e) {
    if (c < 0 || c >= h->ncase || e < 1 || e > h->cases[c].ne) return -1;
    return h->perm[(size_t)h->cases[c].e0 + e - 1];
}

extern "C" int hp_set_halo(hp_handle* h, int32_t n, const int32_t* dst_case, const int32_t* dst_elem,
                           const int32_t* src_case, const int32_t* src_elem) {
    if (!h || n < 0 || (n > 0 && (!dst_case || !dst_elem || !src_case || !src_elem))) return HP_E_ARG;
    if (h->neq == 22) return fail(h, HP_E_UNSUPPORTED, "five-phase model: no partition halos");
    if (h->started) return fail(h, HP_E_STATE, "hp_set_halo after the first step");
    std::vector<int> iv(2 * (size_t)n);
    std::vector<char> role(h->neles, 0);   // 1 destination, 2 source
    for (int t = 0; t < n; t++) {
        const int d = slot_of(h, dst_case[t], dst_elem[t]), q = slot_of(h, src_case[t], src_elem[t]);
        if (d < 0 || q < 0) return fail(h, HP_E_ARG, "halo table: case or element out of range");
        if (role[d] != 0 || role[q] == 1)
            return fail(h, HP_E_ARG, "halo table: a destination repeats or is also a source");
        role[d] = 1;
        role[q] = 2;
        iv[t] = d;
        iv[(size_t)n + t] = q;
    }
    cudaStream_t st = h->stream;
    if (h->d_halo) {
        CUDA_OK(h, cudaFreeAsync(h->d_halo, st));
        h->d_halo = nullptr;
    }
    h->dm.nhalo = 0;
    h->dm.hdst = nullptr; h->dm.hsrc = nullptr;
    if (n > 0) {
        CUDA_OK(h, cudaMallocAsync(reinterpret_cast<void**>(&h->d_halo), iv.size() * sizeof(int), st));
        CUDA_OK(h, cudaMemcpyAsync(h->d_halo, iv.data(), iv.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        h->dm.nhalo = n;
        h->dm.hdst = h->d_halo;
        h->dm.hsrc = h->d_halo + n;
    }
    CUDA_OK(h, cudaStreamSynchronize(st));
    drop_graph(h);
    return HP_OK;
}

extern "C" int hp_set_exchange(hp_handle* h, hp_exchange_fn fn, void* user) {
    if (!h) return HP_E_ARG;
    if (h->neq == 22) return fail(h, HP_E_UNSUPPORTED, "five-phase model: no partition exchange");
    if (fn && h->ncase != 1) return fail(h, HP_E_UNSUPPORTED, "exchange callbacks: single-case handles only");
    h->xfn = fn;
    h->xuser = user;
    drop_graph(h);
    return HP_OK;
}

extern "C" int hp_set_halo_lists(hp_handle* h, int32_t nsend, const int32_t* send_elem, int32_t nrecv,
                                 const int32_t* recv_elem) {
    if (!h || nsend < 0 || nrecv < 0 || (nsend && !send_elem) || (nrecv && !recv_elem)) return HP_E_ARG;
    if (h->neq == 22) return fail(h, HP_E_UNSUPPORTED, "five-phase model: no partition exchange");
    if (h->ncase != 1) return fail(h, HP_E_UNSUPPORTED, "halo lists: single-case handles only");
    std::vector<int> iv((size_t)nsend + nrecv);
    for (int t = 0; t < nsend + nrecv; t++) {
        const int s = slot_of(h, 0, t < nsend ? send_elem[t] : recv_elem[t - nsend]);
        if (s < 0) return fail(h, HP_E_ARG, "halo lists: element out of range");
        iv[t] = s;
    }
    cudaStream_t st = h->stream;
    if (h->d_xlist) {
        CUDA_OK(h, cudaFreeAsync(h->d_xlist, st));
        h->d_xlist = nullptr;
    }
    h->nsend = h->nrecv = 0;
    if (!iv.empty()) {
        CUDA_OK(h, cudaMallocAsync(reinterpret_cast<void**>(&h->d_xlist), iv.size() * sizeof(int), st));
        CUDA_OK(h, cudaMemcpyAsync(h->d_xlist, iv.data(), iv.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    }
    h->nsend = nsend;
    h->nrecv = nrecv;
    CUDA_OK(h, cudaStreamSynchronize(st));
    return HP_OK;
}

// buf[10 * t + k] <-> cn(list[t], k) for the 10 conserved variables (cell
// major, so the cells of one peer form one contiguous block)
template <bool PACK>
__global__ void k_halo_buf(double* cn, long long ld, const int* list, int n, double* buf) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = list[t];
    for (int k = 0; k < 10; k++) {
        if (PACK) buf[10 * (size_t)t + k] = cn[(size_t)k * ld + i];
        else cn[(size_t)k * ld + i] = buf[10 * (size_t)t + k];
    }
}

extern "C" int hp_halo_pack(hp_handle* h, double* buf) {
    if (!h || (h->nsend > 0 && !buf)) return HP_E_ARG;
    if (h->nsend > 0)
        k_halo_buf<true><<<(h->nsend + 255) / 256, 256, 0, h->stream>>>(h->ds.cn, h->ld, h->d_xlist, h->nsend, buf);
    CUDA_OK(h, cudaGetLastError());
    return HP_OK;
}

extern "C" int hp_halo_unpack(hp_handle* h, const double* buf) {
    if (!h || (h->nrecv > 0 && !buf)) return HP_E_ARG;
    if (h->nrecv > 0)
        k_halo_buf<false><<<(h->nrecv + 255) / 256, 256, 0, h->stream>>>(h->ds.cn, h->ld, h->d_xlist + h->nsend,
                                                                          h->nrecv, const_cast<double*>(buf));
    CUDA_OK(h, cudaGetLastError());
    return HP_OK;
}

extern "C" int hp_dtmin_ptr(hp_handle* h, uint64_t** bits) {
    if (!h || !bits) return HP_E_ARG;
    *bits = reinterpret_cast<uint64_t*>(&h->ds.s[0].dtmin_bits);
    return HP_OK;
}

extern "C" int hp_estimate_bytes(const hp_mesh* mesh, const hp_params* params, int64_t* bytes) {
    if (!mesh || !params || !bytes || mesh->neles <= 0 || mesh->nghosts < 0) return HP_E_ARG;
    hp_handle probe_h;
    const long long ld = ((long long)mesh->neles + mesh->nghosts + 63) / 64 * 64;
    const size_t gb = (params->precision == HP_PREC_MIXED || params->precision == HP_PREC_FP32) ? sizeof(float)
                                                                                                : sizeof(double);
    Arena probe;
    const int nface = gb == sizeof(double) || params->face_mode == 1 ? 0
                                                                      : (int)((4LL * mesh->neles + mesh->nghosts) / 2);
    probe_h.neq = params->five_phase ? 22 : 10;
    probe_h.prm.face_mode = params->face_mode;
    if (gb != sizeof(double) && params->wall_fp64_layers > 0)   // bound: every cell in the layers
        probe_h.nwall = probe_h.ngwall = mesh->neles;
    plan_arena(&probe_h, probe, mesh->neles, mesh->nghosts, ld, gb, 1, nface);
    *bytes = (int64_t)(probe.used + 256);
    return HP_OK;
}

extern "C" int hp_estimate_batch_bytes(const hp_mesh* meshes, int32_t ncase, const hp_params* params,
                                       int64_t* bytes) {
    if (!meshes || !params || !bytes || ncase < 1) return HP_E_ARG;
    long long ne = 0, ng = 0;
    for (int c = 0; c < ncase; c++) {
        if (meshes[c].neles <= 0 || meshes[c].nghosts < 0) return HP_E_ARG;
        ne += meshes[c].neles;
        ng += meshes[c].nghosts;
    }
    hp_handle probe_h;
    const long long ld = (ne + ng + 63) / 64 * 64;
    const size_t gb = (params->precision == HP_PREC_MIXED || params->precision == HP_PREC_FP32) ? sizeof(float)
                                                                                                : sizeof(double);
    Arena probe;
    const int nface = gb == sizeof(double) || params->face_mode == 1 ? 0 : (int)((4 * ne + ng) / 2);
    probe_h.neq = params->five_phase ? 22 : 10;
    probe_h.prm.face_mode = params->face_mode;
    if (gb != sizeof(double) && params->wall_fp64_layers > 0)   // bound: every cell in the layers
        probe_h.nwall = probe_h.ngwall = (int)ne;
    plan_arena(&probe_h, probe, (int)ne, (int)ng, ld, gb, ncase, nface);
    *bytes = (int64_t)(probe.used + 256);
    return HP_OK;
}

extern "C" int hp_case_count(const hp_handle* h, int32_t* ncase) {
    if (!h || !ncase) return HP_E_ARG;
    *ncase = h->ncase;
    return HP_OK;
}

extern "C" int hp_poll(hp_handle* h, int32_t* busy) {
    if (!h || !busy) return HP_E_ARG;
    cudaError_t e = cudaStreamQuery(h->stream);
    if (e == cudaErrorNotReady) { *busy = 1; return HP_OK; }
    *busy = 0;
    CUDA_OK(h, e);
    return HP_OK;
}

extern "C" int hp_sync(hp_handle* h) {
    if (!h) return HP_E_ARG;
    CUDA_OK(h, cudaStreamSynchronize(h->stream));
    return HP_OK;
}

extern "C" int hp_get_state(hp_handle* h, double* time, double* cu_elem, double* ghost_prims) {
    return hp_get_state_case(h, 0, time, cu_elem, ghost_prims);
}

extern "C" int hp_get_state_case(hp_handle* h, int32_t c, double* time, double* cu_elem, double* ghost_prims) {
    if (!h) return HP_E_ARG;
    if (c < 0 || c >= h->ncase) return fail(h, HP_E_ARG, "case index out of range");
    const CaseRange& cr = h->cases[c];
    const long long ld = h->ld;
    const int ne = cr.ne, ng = cr.ng;
    cudaStream_t st = h->stream;
    if (time) {
        CUDA_OK(h, cudaMemcpyAsync(h->h_scal, h->ds.s + c, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
    }
    if (cu_elem) {
        const int nq = h->neq;
        k_gather_cols<<<blocks_for((long long)nq * ne, 256), 256, 0, st>>>(h->ds.cu, ld, 0, ne, nq,
                                                                            h->d_perm + cr.e0, h->ds.cn1);
        CUDA_OK(h, cudaGetLastError());
        CUDA_OK(h, cudaMemcpyAsync(cu_elem, h->ds.cn1, nq * (size_t)ne * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    if (ghost_prims && ng) {
        k_gather_ghost_prims<<<blocks_for(6LL * ng, 256), 256, 0, st>>>(h->ds.pr, ld, GHOST_COLS, ng,
                                                                        h->d_gid + cr.g0, h->d_gstage);
        CUDA_OK(h, cudaGetLastError());
        CUDA_OK(h, cudaMemcpyAsync(ghost_prims, h->d_gstage, 6 * (size_t)ng * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
    }
    CUDA_OK(h, cudaStreamSynchronize(st));
    if (time) *time = h->h_scal->time;
    return HP_OK;
}

// --- asynchronous output -----------------------------------------------------
// No counterpart in the reference, which stops its time loop to write.  The
// snapshot (time, cu in reference order, ghost primitives and, for Tecplot,
// the 13 cell-centred fields) is taken on the handle's stream, so it is the
// state after the steps enqueued before the call; the device-to-host copy
// runs on a second stream and the files are written by a host thread, both
// overlapping the steps enqueued after it.
namespace hp {
cudaError_t launch_tecplot_fields(const double* cu, long long ld, int ne, const int* perm, const DevParams& P,
                                  double* out, cudaStream_t st);
}

extern "C" int hp_output_async(hp_handle* h, int32_t c, const hp_mesh* mesh, const char* restart_path,
                               const char* tecplot_path, int32_t* ticket) {
    if (!h || !ticket || (!restart_path && !tecplot_path)) return HP_E_ARG;
    if (h->neq == 22) return fail(h, HP_E_UNSUPPORTED, "five-phase model: no asynchronous restart/Tecplot output (two-phase layout)");
    if (c < 0 || c >= h->ncase) return fail(h, HP_E_ARG, "case index out of range");
    const CaseRange& cr = h->cases[c];
    if (tecplot_path && (!mesh || mesh->neles != cr.ne || !mesh->elem || !mesh->x || !mesh->y || !mesh->z))
        return fail(h, HP_E_ARG, "Tecplot output needs the case's mesh");
    const int ne = cr.ne, ng = cr.ng;
    const long long ld = h->ld;
    // an idle slot, else the older request, which is waited for first
    OutSlot* o = !h->out[0].ticket ? &h->out[0]
                 : !h->out[1].ticket ? &h->out[1]
                 : (h->out[0].ticket < h->out[1].ticket ? &h->out[0] : &h->out[1]);
    output_join(*o);
    const size_t nstate = 1 + 10 * (size_t)ne + 6 * (size_t)ng;
    const size_t need = nstate + (tecplot_path ? 13 * (size_t)ne : 0);
    if (o->cap < need) {
        if (o->d_buf) cudaFree(o->d_buf);
        if (o->h_buf) cudaFreeHost(o->h_buf);
        o->d_buf = nullptr; o->h_buf = nullptr; o->cap = 0;
        CUDA_OK(h, cudaMalloc((void**)&o->d_buf, need * sizeof(double)));
        CUDA_OK(h, cudaMallocHost((void**)&o->h_buf, need * sizeof(double)));
        o->cap = need;
    }
    if (!o->ready) CUDA_OK(h, cudaEventCreateWithFlags(&o->ready, cudaEventDisableTiming));
    if (!o->copied) CUDA_OK(h, cudaEventCreateWithFlags(&o->copied, cudaEventDisableTiming));
    if (!h->ostream) CUDA_OK(h, cudaStreamCreateWithFlags(&h->ostream, cudaStreamNonBlocking));
    cudaStream_t st = h->stream;
    double* d = o->d_buf;
    CUDA_OK(h, cudaMemcpyAsync(d, (const char*)(h->ds.s + c) + offsetof(DevScalars, time), sizeof(double),
                               cudaMemcpyDeviceToDevice, st));
    k_gather_cols<<<blocks_for(10LL * ne, 256), 256, 0, st>>>(h->ds.cu, ld, 0, ne, 10, h->d_perm + cr.e0, d + 1);
    CUDA_OK(h, cudaGetLastError());
    if (ng) {
        k_gather_ghost_prims<<<blocks_for(6LL * ng, 256), 256, 0, st>>>(h->ds.pr, ld, GHOST_COLS, ng,
                                                                        h->d_gid + cr.g0, d + 1 + 10 * (size_t)ne);
        CUDA_OK(h, cudaGetLastError());
    }
    if (tecplot_path) CUDA_OK(h, hp::launch_tecplot_fields(h->ds.cu, ld, ne, h->d_perm + cr.e0, h->dp, d + nstate, st));
    CUDA_OK(h, cudaEventRecord(o->ready, st));
    CUDA_OK(h, cudaStreamWaitEvent(h->ostream, o->ready, 0));
    CUDA_OK(h, cudaMemcpyAsync(o->h_buf, d, need * sizeof(double), cudaMemcpyDeviceToHost, h->ostream));
    CUDA_OK(h, cudaEventRecord(o->copied, h->ostream));
    o->ticket = h->next_ticket++;
    o->rc = HP_OK;
    const std::string rp = restart_path ? restart_path : "", tp = tecplot_path ? tecplot_path : "";
    o->writer = std::thread([o, rp, tp, ne, ng, nstate, mesh]() {
        if (cudaEventSynchronize(o->copied) != cudaSuccess) { o->rc = HP_E_CUDA; return; }
        const double* b = o->h_buf;
        int rc = HP_OK;
        if (!rp.empty()) rc = hp_write_restart(rp.c_str(), ne, ng, b[0], b + 1, b + 1 + 10 * (size_t)ne);
        if (rc == HP_OK && !tp.empty()) rc = hp_write_tecplot(tp.c_str(), mesh, b + nstate);
        o->rc = rc;
    });
    *ticket = o->ticket;
    return HP_OK;
}

extern "C" int hp_output_wait(hp_handle* h, int32_t ticket) {
    if (!h) return HP_E_ARG;
    for (OutSlot& o : h->out)
        if (o.ticket && o.ticket == ticket) {
            const int rc = output_join(o);
            return rc == HP_OK ? HP_OK : fail(h, rc, "asynchronous output failed");
        }
    return fail(h, HP_E_ARG, "unknown or already collected output ticket");
}

extern "C" int hp_get_prims(hp_handle* h, double* prims) {
    if (!h || !prims) return HP_E_ARG;
    const long long ld = h->ld;
    const int ne = h->cases[0].ne;   // case 0 (the only one of a single-case handle)
    cudaStream_t st = h->stream;
    // cn1 stages at most 10 columns at a time
    for (int c0 = 0; c0 < NPR; c0 += 10) {
        const int nc = NPR - c0 < 10 ? NPR - c0 : 10;
        k_gather_cols<<<blocks_for((long long)nc * ne, 256), 256, 0, st>>>(h->ds.pr, ld, c0, ne, nc, h->d_perm + h->cases[0].e0,
                                                                          h->ds.cn1);
        CUDA_OK(h, cudaGetLastError());
        CUDA_OK(h, cudaMemcpyAsync(prims + (size_t)c0 * ne, h->ds.cn1, (size_t)nc * ne * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
        CUDA_OK(h, cudaStreamSynchronize(st));
    }
    return HP_OK;
}

extern "C" int hp_device_state(hp_handle* h, double** cu_dev, int64_t* ld) {
    if (!h) return HP_E_ARG;
    if (cu_dev) *cu_dev = h->ds.cu;
    if (ld) *ld = h->ld;
    return HP_OK;
}

extern "C" int hp_info(const hp_handle* h, int64_t* kernels_per_step, int64_t* device_bytes, int64_t* aliased) {
    if (!h) return HP_E_ARG;
    if (kernels_per_step) {
        // k_step_begin, smooth x2, bc, visc, stages x (prim, bc, grad, flux), prim end,
        // k_step_end, prim start
        // (the Jameson flux, myflux 3, computes no gradients)
        const int grad = h->prm.myorder == 2 && h->prm.myflux != 3 ? 1 : 0;
        int64_t n = 1 + 2 + (h->nghosts ? 1 : 0) + (h->prm.inviscid ? 0 : 1);
        int64_t per_stage = 1 + (h->nghosts ? 1 : 0) + grad + 1;
        if (h->aliased) per_stage += grad + 1;
        if (h->dm.nfringe > 0) per_stage += 1;
        if (h->dm.nface > 0)   // k_faceflux; or the scatter kernels of face modes 2 (one per colour), 3
            per_stage += h->dm.face_mode == 2 ? h->dm.ncolor : 1;
        if (h->dm.nface > 0 && !h->prm.inviscid && h->var->face_visc) n += 1;   // k_vis_gather
        n += (int64_t)h->dp.nstage * per_stage + 3;
        if (h->aliased) n += 2;
        if (h->neq == 22) n += 2 + (int64_t)h->dp.nstage * (2 + (h->nghosts ? 1 : 0));   // k_qrs_*
        if (h->nwall > 0)   // FP64 wall layers: viscous once, gradients and fluxes per stage
            n += (h->prm.inviscid ? 0 : 1) + (int64_t)h->dp.nstage * (grad + 1);
        if (h->prm.use_graph == 2 && h->fused > 0 && !h->xfn && h->dm.nfringe == 0 && h->dm.nhalo == 0)
            n = 1;   // the fused step
        *kernels_per_step = n;
    }
    if (device_bytes) *device_bytes = (int64_t)h->arena.size;
    if (aliased) *aliased = h->aliased;
    return HP_OK;
}
