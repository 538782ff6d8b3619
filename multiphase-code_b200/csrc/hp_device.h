// hp_device.h -- device-side layout of one case (mesh + state) and the
// per-variant kernel entry table.  Shared by the host code (hp_host.cu) and
// every precision variant (hp_variant_*.cu).
//
// Layout in HBM: structure of arrays, one column per variable, leading
// dimension `ld` (= ntot rounded up to 64 cells) so each column starts on a
// 512-byte boundary.  Cell ids are 0-based internally: elements [0, neles),
// boundary ghosts [neles, neles + nghosts) -- the reference's 1-based ids
// minus one (src/main.F90:103).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/hydraphase.h"   // HP_IBLANK_HALO*, HP_X_*

namespace hp {

enum { NEQ = 10, NPR = 14, NGR = 33, NLSQ = 16 };

// primitive columns (the reference's ug,vg,wg,tg,pg,pp,phig,phip,up,vp,wp,
// tp,rog,rop of src/mod_GlobalVariables.F90:13)
enum { P_UG = 0, P_VG, P_WG, P_TG, P_PG, P_PP, P_PHIG, P_PHIP, P_UP, P_VP,
       P_WP, P_TP, P_ROG, P_ROP };
// stored gradient columns (x,y,z per field), src/sr_derivative.F90:259-309
enum { G_UG = 0, G_VG = 3, G_WG = 6, G_TG = 9, G_UP = 12, G_VP = 15,
       G_WP = 18, G_TP = 21, G_PG = 24, G_PP = 27, G_PHIG = 30 };

// face kind bits per cell, 4 bits per face: bit 0 = wall (ghost type 5),
// bit 1 = MUSCL-reconstruct across the face (interior or partition ghost).
enum { FK_WALL = 1, FK_RECON = 2 };

struct DevParams {
    double gamag, gamap, pinf, cpp, cpg, prg, rrg, prp;
    double emin, emax, phipzero;
    double ugmin, vgmin, wgmin, upmin, vpmin, wpmin, tgmin, tpmin, pmin;
    double as, ts, c23, co2, co4, fsd;   // fsd = 4 sigma / d
    double cfl, venkat_k, twall, amup;
    // correctly rounded reciprocals of constant divisors
    double r_emm, r_gm1, r_gamap, r_prg, r_prp;
    int rk_scheme, inviscid, myorder, nstage;
    int myflux;   // 1 HLLC-Zien, 2 HLLC-Batten (src/mod_Fluxmodule.F90:8-11)
    // five-phase model: dispersed phases q, r, s (conserved columns 10-21)
    int five_phase;
    double rhod[3], radd[3], vold[3];   // densities, radii, particle volumes
};

// A handle holds one case or a batch of cases whose meshes are concatenated:
// the elements of case c occupy [elem_base_c, elem_base_c + neles_c) and its
// ghosts a range of [neles, neles + nghosts); neighbour ids point into the
// same case only, so every kernel sweeps all cases in one launch.  `cid`
// maps an element to its case (null for a single case: case 0).
struct DevMesh {
    int neles, nghosts, ntot, aliased;
    long long ld;
    int ncase;
    const int* cid;         // [neles] case of each element, or null
    const int* nc;          // [4][ld] face neighbours
    const int* snb;         // [4][ld] neighbours as smoothing sees them
    const unsigned* fk;     // [ld] face kind nibbles
    const int* iblank;      // [ld]
    const double *xc, *yc, *zc, *vol, *dl, *dd;   // [ld]
    // limiter epsilon^2 = (K dl)^3 per cell (src/sr_VK.F90:34), evaluated
    // once at set-up with the host's pow, as the reference evaluates it
    const double* eps2;     // [ld]
    const double* sc;       // [12][ld] face area vectors sc1x..sc4z
    const double* fch;      // [12][ld] face centroids, 0.3333 factor (HLLC, VK)
    const double* fcv;      // [12][ld] face centroids, /3 (viscous)
    // geometry-only least-squares terms, evaluated once at set-up with the
    // reference's expressions: [0..3] weights, [4..9] a1 a2 a3 b1 b2 b3,
    // [10] the determinant, [11..14] and [15] the correctly rounded
    // reciprocals of the weights and of the determinant; LSQA for the 1/r^2
    // cell gradients (src/sr_derivative.F90:163-176,255), LSQB for the 1/r
    // gradient of alpha_g in the sources (src/sr_source.F90:100-117)
    const double* dxn;      // [12][ld] centroid of neighbour f minus the
                            // cell's (x, y, z of face 1, then 2, 3, 4)
    const double* lsqa;     // [NLSQ][ld]
    const double* lsqb;     // [NLSQ][ld]
    const int *g_par, *g_id, *g_type;   // [nghosts] ghost list (reference order)
    // overset fringe (nfringe = 0: none): cells, 4 donor cells each and
    // barycentric weights, [4][nfringe] column-major
    // unique faces (FP32-arithmetic variants; nface = 0: cell-centric
    // fluxes): owner cell and local face of each, and per cell and local
    // face the signed face id + 1 (negative when the cell is not the owner)
    int nface;
    long long fld;          // leading dimension of the face-flux columns
    const int* f_i;
    const int* f_code;      // local face of the owner (bits 0-1)
    const int* cface;       // [4][ld]
    // face modes 2 (colouring) and 3 (atomics): the face fluxes are added
    // to a per-cell accumulator instead of stored as records.  Mode 2 takes
    // the faces colour by colour (no two faces of a colour share a cell, so
    // each colour adds without atomics, in a fixed order); fcolor lists the
    // face ids colour by colour, colour c at [fcoff[c], fcoff[c + 1]).
    int face_mode;
    int ncolor;
    const int* fcolor;      // [nface]
    int fcoff[33];
    int nfringe;
    const int* fr;
    const int* fdon;
    const double* fw;
    // partition halo (nhalo = 0: none): after every RK stage cell hdst[t]
    // takes the conserved state of cell hsrc[t] (the parts of one mesh as
    // the cases of a batch); the cases then share one dt
    int nhalo;
    const int* hdst;
    const int* hsrc;
    // FP64 wall layers of the FP32-arithmetic variants (nwall = 0: none):
    // the cells within a few layers of a wall ghost (wcells, ascending) take
    // their viscous terms, fluxes, sources and RK update from the FP64
    // kernels over these lists; gcells adds their interior neighbours, whose
    // FP64 gradients those fluxes reconstruct from; wclass[i] != 0 marks the
    // cells of wcells, which the FP32 kernels leave alone (2: no neighbour
    // outside the layers, so not even their FP32 gradients are read)
    int nwall, ngwall;
    int wprefix;            // 1: wcells and gcells are 0, 1, ... (the layer
                            // cells first in the cell order, see hp_host.cu)
    const int* wcells;
    const int* gcells;
    const unsigned char* wclass;   // [ld]
};

// Per-case scalars (one entry per case of the handle).
struct DevScalars {
    unsigned long long dtmin_bits;    // running min of dl/(a+|u|), skips NaN
    unsigned long long diff_bits[4];  // running max |cn - cu|, skips NaN
    unsigned long long nan_count;
    double dt, time, velmag;
    int total;                        // step counter (src/main.F90:522)
    int step_in_call;
    double fcarry[10];                // stale-flux carry (aliased meshes)
    int err_flags;
    int cell1;                        // internal id of the case's cell 1
};

// R values per face record of the face-based variants: 48 bytes in FP32, read
// as three 16-byte loads
constexpr int FACE_REC = 12;

template <class R>
struct DevState {
    double *cn, *cu, *cn1;   // [10][ld]
    double* pr;              // [14][ld]
    R* prr;                  // [14][ld] primitives in R: pr itself when R is
                             // double, a float copy otherwise
    R* gr;                   // [33][ld]
    double* phi;             // [ld]
    double *anu, *d2q;       // [2][ld], [10][ld]
    double *d24, *vis;       // [10][ld], [8][ld]
    double* egt;             // [2][ld] ghost egtotal/eptotal (aliased meshes)
    // five-phase model only (null otherwise): cn, cu, cn1, d2q and d24 then
    // hold 22 columns
    double* qpr;             // [12][ld] phi, u, v, w of q, r, s
    double* anuq;            // [3][ld] their JST switches
    double* qdrag;           // [9][ld] drag of q, r, s on the liquid (x, y, z)
    double* racc;            // [10][ld] face modes 2, 3: the cells' face sums
    R* ff;                   // [nface][FACE_REC] face records (face-based
                             // variants): 10 flux components, the wall flag
                             // (1: pressure terms only), one pad
    DevScalars* s;
    double* diag;            // [max_steps][8]
    int max_diag;
    double* gr64;            // [33][ld] FP64 gradients of the wall layers
                             // (FP32 variants with nwall > 0; else null)
};

// The FP64 view of an FP32-arithmetic state for the wall-layer kernels: the
// FP64 primitives as their primitives and gr64 as their gradients; every
// other array is shared.
template <class R>
inline DevState<double> fp64_view(const DevState<R>& s) {
    DevState<double> v;
    v.cn = s.cn; v.cu = s.cu; v.cn1 = s.cn1; v.pr = s.pr; v.prr = s.pr; v.gr = s.gr64; v.phi = s.phi;
    v.anu = s.anu; v.d2q = s.d2q; v.d24 = s.d24; v.vis = s.vis; v.egt = s.egt;
    v.qpr = s.qpr; v.anuq = s.anuq; v.qdrag = s.qdrag; v.racc = s.racc; v.ff = nullptr;
    v.s = s.s; v.diag = s.diag; v.max_diag = s.max_diag; v.gr64 = s.gr64;
    return v;
}

// FP64 kernels over the wall-layer lists, provided by the FP64 variant and
// called by the FP32-arithmetic variants' step.
struct WallFp64 {
    void (*visc)(const DevMesh&, const DevState<double>&, const DevParams&, cudaStream_t);
    void (*grad)(const DevMesh&, const DevState<double>&, const DevParams&, cudaStream_t);
    void (*flux)(const DevMesh&, const DevState<double>&, const DevParams&, cudaStream_t, int stage);
};
extern const WallFp64 wall_fp64;

// Grid-wide barrier of the fused step kernel (zeroed at set-up): arrivals,
// generation, and a flag set when a wait gave up (its spin is bounded).
struct GridSync {
    unsigned count;
    unsigned gen;
    int err;
    int pad;
};

// Kernel kinds, for per-kernel timing (hp_profile_steps).
enum KernelKind {
    KK_PRIM_START = 0, KK_STEP_BEGIN, KK_SMOOTH1, KK_SMOOTH2, KK_BC_VISC, KK_VISC,
    KK_PRIM_STAGE, KK_BC, KK_GRAD, KK_FLUX, KK_PRIM_END, KK_STEP_END, KK_SERIAL,
    KK_OVERSET, KK_HALO, KK_QRS, KK_COUNT
};

// Optional hook called before every launch (and with KK_COUNT after the
// last one) so the host can bracket each kernel with CUDA events.
struct StepHook {
    void (*mark)(void* ctx, int kind);      // before each kernel (may be null)
    void* ctx;
    // exchange points of a part run on several GPUs (may be null):
    // HP_X_DT before the step's dt is formed, HP_X_HALO after each RK stage
    void (*exchange)(void* ctx, int point);
    void* xctx;
};

// What one precision variant provides to the host.
struct Variant {
    const char* name;
    size_t grad_bytes;  // sizeof(R) of the gradient columns
    // enqueue the start-of-step primitive recovery + dt contributions
    void (*enqueue_start)(const DevMesh&, const void* st, const DevParams&,
                          cudaStream_t, int block, const StepHook* hook);
    // enqueue one full step (after enqueue_start of the same step)
    void (*enqueue_step)(const DevMesh&, const void* st, const DevParams&,
                         cudaStream_t, int block, const StepHook* hook);
    // 1 when the viscous fluxes are evaluated once per face on meshes with a
    // face list (k_facevisc + k_vis_gather instead of one kernel)
    int face_visc;
    // fused step (one cooperative launch per step): the grid it runs with on
    // this device (blocks of 128 threads), and the launch of one step
    int (*fused_grid)(const DevMesh&, const DevParams&);
    cudaError_t (*enqueue_fused)(const DevMesh&, const void* st, const DevParams&, cudaStream_t,
                                 GridSync* sync, int grid);
};

extern const Variant variant_fp64_parity;
extern const Variant variant_fp64;
extern const Variant variant_mixed;
extern const Variant variant_fp32;

}  // namespace hp
