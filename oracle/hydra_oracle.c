/*
 * hydra_oracle.c -- sequential FP64 CPU restatement of the reference's
 * explicit residual-and-update path.  TEST INFRASTRUCTURE ONLY (see
 * hydra_oracle.h): it is the checker for the CUDA path, never the product.
 *
 * Every routine names the reference routine (file:line, relative to the
 * reference project HydraPhase_60_FPC_5mill/) it restates.  Expressions keep
 * the reference's operand order so that an IEEE-754 FP64 build without
 * contraction (-ffp-contract=off) reproduces its rounding.  Two compiler
 * dependent behaviours are modelled explicitly:
 *   - Fortran MIN/MAX with a NaN argument (nan_mode, see mn2/mx2);
 *   - the HLLC face flux of a face where no wave-speed branch is taken keeps
 *     the value of the previously evaluated face (sr_hllcbatten.F90:464-529
 *     assigns FSTARA only inside the IF chain).
 */
#include "hydra_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NEQ 10

enum { G_UG = 0, G_VG = 3, G_WG = 6, G_TG = 9, G_UP = 12, G_VP = 15,
       G_WP = 18, G_TP = 21, G_PG = 24, G_PP = 27, G_PHIG = 30, G_ROG = 33,
       G_ROP = 36, NGRAD = 39 };

struct or_case {
    or_params p;
    int nodes, neles, nghosts, ntot;
    double *x, *y, *z;                       /* [nodes+1] */
    int *nod[4];                             /* nod(i,k), [ntot+1] */
    int *nc[4];                              /* nc1..nc4, [ntot+1] */
    int *iblank;
    int *nparent, *nghost, *ntype, *nside;   /* [nghosts+1] */
    int nbc[8];                              /* counts per list */
    int *bcl[8];                             /* 2,3,5,51,53,6,7 lists */
    double *xcel, *ycel, *zcel, *vol, *dl, *dd;
    double *sc[12];                          /* sc1x,sc1y,sc1z,...,sc4z */
    double *ug, *vg, *wg, *pg, *pp, *tg, *phig, *up, *vp, *wp, *phip, *tp;
    double *rop, *rog, *ag, *ap, *egtotal, *eptotal, *phi;
    double *cn, *cu, *cn1, *rhs, *d24, *d2q, *anu;
    int neq;                                 /* 10, or 22 with the five-phase model */
    /* five-phase model: dispersed-phase primitives (phi, u, v, w of q, r, s) */
    double *phiq, *phir, *phis, *uq, *vq, *wq, *ur, *vr, *wr, *us, *vs, *ws;
    double volq, volr, vols;                 /* particle volumes, src/main.F90:352-354 */
    double *vis[8];                          /* ug,vg,wg,tg,up,vp,wp,tp */
    double *g[NGRAD];
    double xmax, ymax, zmax, ymin, zmin;
    double rrg, co2, co4, c23, cmug, gravity, prp, foursigmabyd;
    double rogmin, ropmin, egtotalmin, eptotalmin;
    double time, dt, dtmin;
    int total;
    double fstar[10];                        /* stale HLLC flux carry */
    int aliased;                             /* ghost ids alias elements/each other */
    int nfringe;                             /* overset fringe cells (0: none) */
    int *ofr, *odon;                         /* [nfringe], [4*nfringe] 1-based */
    double *ow;                              /* [4*nfringe] */
};

/* Cell loops run in parallel only when the result cannot depend on the
 * order (no aliased ghosts); ghost loops always run in reference order. */
#define PAR(S) ((S)->aliased == 0 && g_threads > 1)

/* ------------------------------------------------------------------ */
/* Fortran MIN/MAX.  nan_mode 0: the pre-GCC-9 gfortran expansion
 *   m = a1; if (a2 < m || isnan(m)) m = a2; ...
 * which skips a NaN argument unless it comes first.  nan_mode 1: MIN_EXPR
 * as expanded on x86-64 SSE, (a < b ? a : b), returning b on NaN.        */
static int g_nan_mode = 0;
static int g_threads = 1;       /* OpenMP threads for non-aliased meshes */

void or_set_threads(int n) { g_threads = n > 0 ? n : 1; }
static inline double mn2(double a, double b) {
    if (g_nan_mode == 0) return (b < a || isnan(a)) ? b : a;
    return (a < b) ? a : b;
}
static inline double mx2(double a, double b) {
    if (g_nan_mode == 0) return (b > a || isnan(a)) ? b : a;
    return (a > b) ? a : b;
}
static inline double mn3(double a, double b, double c) { return mn2(mn2(a, b), c); }
static inline double mx3(double a, double b, double c) { return mx2(mx2(a, b), c); }
static inline double mn5(double a, double b, double c, double d, double e) {
    return mn2(mn2(mn2(mn2(a, b), c), d), e);
}
static inline double mx5(double a, double b, double c, double d, double e) {
    return mx2(mx2(mx2(mx2(a, b), c), d), e);
}
static inline double mn4(double a, double b, double c, double d) {
    return mn2(mn2(mn2(a, b), c), d);
}

/* det() and fvenkat() of src/mod_MatrixOps.F90:4-18 */
static inline double det(double A11, double A21, double A31, double A12,
                         double A22, double A32, double A13, double A23,
                         double A33) {
    return A11 * (A22 * A33 - A23 * A32) - A21 * (A12 * A33 - A13 * A32) +
           A31 * (A12 * A23 - A13 * A22);
}
static inline double fvenkat(double delp, double delm, double epssq) {
    return (((delp * delp + epssq) * delm + 2.0 * delm * delm * delp) /
            (delp * delp + 2.0 * delm * delm + delp * delm + epssq)) / delm;
}
static inline double sq(double a) { return a * a; }

/* Single-precision literals of the reference, promoted to double. */
#define R4(v) ((double)(float)(v))

#define CN(i, k) S->cn[((size_t)(k)-1) * (size_t)S->ntot + (size_t)(i)-1]
#define CU(i, k) S->cu[((size_t)(k)-1) * (size_t)S->ntot + (size_t)(i)-1]
#define CN1(i, k) S->cn1[((size_t)(k)-1) * (size_t)S->ntot + (size_t)(i)-1]
#define D2Q(i, k) S->d2q[((size_t)(k)-1) * (size_t)S->ntot + (size_t)(i)-1]
#define ANU(i, k) S->anu[((size_t)(k)-1) * (size_t)S->ntot + (size_t)(i)-1]
#define RHS(i, k) S->rhs[((size_t)(k)-1) * (size_t)S->neles + (size_t)(i)-1]
#define D24(i, k) S->d24[((size_t)(k)-1) * (size_t)S->neles + (size_t)(i)-1]

static double *dalloc(size_t n) { return (double *)calloc(n, sizeof(double)); }
static int *ialloc(size_t n) { return (int *)calloc(n, sizeof(int)); }

/* ------------------------------------------------------------------ */
/* Face node triples of sr_geometry.F90:149-158 (area vectors) and of   */
/* sr_hllcbatten.F90:79-115 / sr_VK.F90:52-63 (centroids, 0.3333 factor)*/
static const int GEO_FACE[4][3] = {{2, 3, 4}, {4, 3, 1}, {2, 4, 1}, {3, 2, 1}};
static const int HLL_FACE[4][3] = {{2, 4, 3}, {3, 4, 1}, {4, 2, 1}, {2, 3, 1}};

static void geometry(or_case *S) {
    /* src/sr_geometry.F90:112-124 bounding box */
    S->xmax = -1.0e30; S->ymax = -1.0e30; S->zmax = -1.0e30;
    S->ymin = 1.0e30; S->zmin = 1.0e30;
    for (int n = 1; n <= S->nodes; n++) {
        S->xmax = mx2(S->xmax, S->x[n]);
        S->ymax = mx2(S->ymax, S->y[n]);
        S->zmax = mx2(S->zmax, S->z[n]);
        S->ymin = mn2(S->ymin, S->y[n]);
        S->zmin = mn2(S->zmin, S->z[n]);
    }
    const double *x = S->x, *y = S->y, *z = S->z;
    /* src/sr_geometry.F90:147-239 face vectors, centroid, dl, volume */
    for (int i = 1; i <= S->neles; i++) {
        for (int f = 0; f < 4; f++) {
            int n1 = S->nod[GEO_FACE[f][0] - 1][i];
            int n2 = S->nod[GEO_FACE[f][1] - 1][i];
            int n3 = S->nod[GEO_FACE[f][2] - 1][i];
            double dxyA = (x[n1] - x[n2]) * (y[n1] + y[n2]);
            double dxyB = (x[n2] - x[n3]) * (y[n2] + y[n3]);
            double dxyC = (x[n3] - x[n1]) * (y[n3] + y[n1]);
            double dyzA = (y[n1] - y[n2]) * (z[n1] + z[n2]);
            double dyzB = (y[n2] - y[n3]) * (z[n2] + z[n3]);
            double dyzC = (y[n3] - y[n1]) * (z[n3] + z[n1]);
            double dzxA = (z[n1] - z[n2]) * (x[n1] + x[n2]);
            double dzxB = (z[n2] - z[n3]) * (x[n2] + x[n3]);
            double dzxC = (z[n3] - z[n1]) * (x[n3] + x[n1]);
            S->sc[3 * f + 0][i] = 0.5 * (dyzA + dyzB + dyzC);
            S->sc[3 * f + 1][i] = 0.5 * (dzxA + dzxB + dzxC);
            S->sc[3 * f + 2][i] = 0.5 * (dxyA + dxyB + dxyC);
        }
        int n1 = S->nod[0][i], n2 = S->nod[1][i], n3 = S->nod[2][i], n4 = S->nod[3][i];
        double x1 = x[n1], x2 = x[n2], x3 = x[n3], x4 = x[n4];
        double y1 = y[n1], y2 = y[n2], y3 = y[n3], y4 = y[n4];
        double z1 = z[n1], z2 = z[n2], z3 = z[n3], z4 = z[n4];
        S->xcel[i] = 0.25 * (x1 + x2 + x3 + x4);
        S->ycel[i] = 0.25 * (y1 + y2 + y3 + y4);
        S->zcel[i] = 0.25 * (z1 + z2 + z3 + z4);
        double dl12 = sqrt(sq(x1 - x2) + sq(y1 - y2) + sq(z1 - z2));
        double dl13 = sqrt(sq(x1 - x3) + sq(y1 - y3) + sq(z1 - z3));
        double dl14 = sqrt(sq(x1 - x4) + sq(y1 - y4) + sq(z1 - z4));
        double dl23 = sqrt(sq(x2 - x3) + sq(y2 - y3) + sq(z2 - z3));
        double dl42 = sqrt(sq(x4 - x2) + sq(y4 - y2) + sq(z4 - z2));
        double dl43 = sqrt(sq(x4 - x3) + sq(y4 - y3) + sq(z4 - z3));
        S->dl[i] = mn2(mn2(mn2(mn2(mn2(dl12, dl13), dl14), dl23), dl42), dl43);
        double v6 = det(x2, x3, x4, y2, y3, y4, z2, z3, z4) -
                    det(x1, x3, x4, y1, y3, y4, z1, z3, z4) +
                    det(x1, x2, x4, y1, y2, y4, z1, z2, z4) -
                    det(x1, x2, x3, y1, y2, y3, z1, z2, z3);
        S->vol[i] = fabs(v6) / 6.0;
    }
    /* src/sr_geometry.F90:245-289 mirrored ghost centroids (sequential:
     * ghost ids may alias element ids in merged meshes) */
    for (int i = 1; i <= S->nghosts; i++) {
        int np = S->nparent[i], ng = S->nghost[i], ns = S->nside[i];
        if (ns < 1 || ns > 4) continue;
        int n1 = S->nod[GEO_FACE[ns - 1][0] - 1][np];
        int n2 = S->nod[GEO_FACE[ns - 1][1] - 1][np];
        int n3 = S->nod[GEO_FACE[ns - 1][2] - 1][np];
        double xcf = (x[n1] + x[n2] + x[n3]) / 3.0;
        double ycf = (y[n1] + y[n2] + y[n3]) / 3.0;
        double zcf = (z[n1] + z[n2] + z[n3]) / 3.0;
        S->xcel[ng] = 2.0 * xcf - S->xcel[np];
        S->ycel[ng] = 2.0 * ycf - S->ycel[np];
        S->zcel[ng] = 2.0 * zcf - S->zcel[np];
        S->vol[ng] = S->vol[np];
        S->nc[0][ng] = ng; S->nc[1][ng] = ng; S->nc[2][ng] = ng; S->nc[3][ng] = ng;
    }
    /* src/sr_geometry.F90:295-347 wave-transmissive distance dd */
    for (int i = 1; i <= S->nghosts; i++) {
        int np = S->nparent[i], nt = S->ntype[i];
        int n1 = S->nod[0][np], n2 = S->nod[1][np], n3 = S->nod[2][np], n4 = S->nod[3][np];
        if (nt == 3) {
            double xc = (x[n1] + x[n2] + x[n3] + x[n4]) * 0.25;
            S->dd[np] = fabs(S->xmax - xc);
        } else if (nt == 51) {
            double yc = (y[n1] + y[n2] + y[n3] + y[n4]) * 0.25;
            S->dd[np] = (yc > 0) ? fabs(S->ymax - yc) : fabs(S->ymin - yc);
        } else if (nt == 53) {
            double zc = (z[n1] + z[n2] + z[n3] + z[n4]) * 0.25;
            S->dd[np] = (zc > R4(0.1)) ? fabs(S->zmax - zc) : fabs(S->zmin - zc);
        }
    }
}

/* ------------------------------------------------------------------ */
or_case *or_create(const or_params *p, int32_t nodes, int32_t neles,
                   int32_t nghosts, const double *x, const double *y,
                   const double *z, const int32_t *elem, const int32_t *ghost) {
    if (p->myflux < 1 || p->myflux > 3) return NULL;   /* mod_Fluxmodule.F90:14-16 stops */
    or_case *S = (or_case *)calloc(1, sizeof(or_case));
    S->p = *p;
    g_nan_mode = p->nan_mode;
    S->nodes = nodes; S->neles = neles; S->nghosts = nghosts;
    S->ntot = neles + nghosts;
    size_t nt1 = (size_t)S->ntot + 1;
    S->x = dalloc(nodes + 1); S->y = dalloc(nodes + 1); S->z = dalloc(nodes + 1);
    for (int n = 1; n <= nodes; n++) { S->x[n] = x[n - 1]; S->y[n] = y[n - 1]; S->z[n] = z[n - 1]; }
    for (int k = 0; k < 4; k++) { S->nod[k] = ialloc(nt1); S->nc[k] = ialloc(nt1); }
    S->iblank = ialloc(nt1);
    for (int e = 0; e < neles; e++) {
        const int32_t *r = elem + 9 * (size_t)e;
        int nel = e + 1;
        for (int k = 0; k < 4; k++) { S->nod[k][nel] = r[k]; S->nc[k][nel] = r[4 + k]; }
        S->iblank[nel] = r[8];
    }
    S->nparent = ialloc(nghosts + 1); S->nghost = ialloc(nghosts + 1);
    S->ntype = ialloc(nghosts + 1); S->nside = ialloc(nghosts + 1);
    static const int types[7] = {2, 3, 5, 51, 53, 6, 7};
    for (int t = 0; t < 7; t++) S->bcl[t] = ialloc(nghosts + 1);
    for (int i = 1; i <= nghosts; i++) {
        const int32_t *r = ghost + 4 * (size_t)(i - 1);
        S->nparent[i] = r[0]; S->nghost[i] = r[1]; S->ntype[i] = r[2]; S->nside[i] = r[3];
        for (int t = 0; t < 7; t++)
            if (r[2] == types[t]) S->bcl[t][++S->nbc[t]] = i;   /* main.F90:239-275 */
    }
    {
        char *seen = (char *)calloc(nt1, 1);
        for (int i = 1; i <= nghosts && !S->aliased; i++) {
            int g = S->nghost[i];
            if (g <= neles || seen[g]) S->aliased = 1;
            seen[g] = 1;
        }
        for (int i = 1; i <= nghosts && !S->aliased; i++)
            if (S->nparent[i] > neles || seen[S->nparent[i]]) S->aliased = 1;
        free(seen);
    }
    S->xcel = dalloc(nt1); S->ycel = dalloc(nt1); S->zcel = dalloc(nt1);
    S->vol = dalloc(nt1); S->dl = dalloc(nt1); S->dd = dalloc(nt1);
    for (int k = 0; k < 12; k++) S->sc[k] = dalloc(nt1);
    double **prims[] = {&S->ug, &S->vg, &S->wg, &S->pg, &S->pp, &S->tg, &S->phig,
                        &S->up, &S->vp, &S->wp, &S->phip, &S->tp, &S->rop, &S->rog,
                        &S->ag, &S->ap, &S->egtotal, &S->eptotal, &S->phi};
    for (size_t k = 0; k < sizeof(prims) / sizeof(prims[0]); k++) *prims[k] = dalloc(nt1);
    S->neq = p->five_phase ? 22 : NEQ;          /* src/main.F90:114-124 */
    size_t nn = (size_t)S->ntot * S->neq;
    S->cn = dalloc(nn); S->cu = dalloc(nn); S->cn1 = dalloc(nn); S->d2q = dalloc(nn);
    S->anu = dalloc((size_t)S->ntot * 3);
    S->rhs = dalloc((size_t)neles * S->neq); S->d24 = dalloc((size_t)neles * S->neq);
    if (p->five_phase) {
        double **q[] = {&S->phiq, &S->phir, &S->phis, &S->uq, &S->vq, &S->wq,
                        &S->ur, &S->vr, &S->wr, &S->us, &S->vs, &S->ws};
        for (size_t k = 0; k < sizeof(q) / sizeof(q[0]); k++) *q[k] = dalloc(nt1);
        S->volq = (4.0 / 3.0) * 3.1415926 * (p->radq * p->radq * p->radq);
        S->volr = (4.0 / 3.0) * 3.1415926 * (p->radr * p->radr * p->radr);
        S->vols = (4.0 / 3.0) * 3.1415926 * (p->rads * p->rads * p->rads);
    }
    for (int k = 0; k < 8; k++) S->vis[k] = dalloc((size_t)neles + 1);
    for (int k = 0; k < NGRAD; k++) S->g[k] = dalloc(nt1);

    /* src/main.F90:336-349 constants (single-precision literals promoted) */
    S->co2 = R4(1.00f / 16.00f);
    S->co4 = R4(1.00f / 1024.00f);
    S->c23 = R4(2.00f / 3.00f);
    S->cmug = R4(11.848e-8f) * sqrt(p->amolg);
    S->rrg = 287.0;
    S->gravity = 0.0;
    S->prp = 10.0;
    S->foursigmabyd = 4.0 * p->surfacetension / p->diap;
    S->time = 0.0;
    S->dtmin = 1.0e8;
    S->total = 0;
    geometry(S);
    /* src/main.F90:391-402 reference states */
    S->rogmin = p->pmin / (S->rrg * p->tgmin);
    S->ropmin = (p->pmin + p->pinf) * p->gamap / ((p->gamap - 1.0) * p->cpp * p->tpmin);
    S->egtotalmin = S->rrg * p->tgmin / (p->gamag - 1.0) +
                    0.5 * (sq(p->ugmin) + sq(p->vgmin) + sq(p->wgmin));
    S->eptotalmin = (p->cpp * p->tpmin) / p->gamap + p->pinf / S->ropmin +
                    0.5 * (sq(p->upmin) + sq(p->vpmin) + sq(p->wpmin));
    return S;
}

void or_destroy(or_case *S) {
    if (!S) return;
    free(S->x); free(S->y); free(S->z);
    for (int k = 0; k < 4; k++) { free(S->nod[k]); free(S->nc[k]); }
    free(S->iblank); free(S->nparent); free(S->nghost); free(S->ntype); free(S->nside);
    for (int t = 0; t < 7; t++) free(S->bcl[t]);
    free(S->xcel); free(S->ycel); free(S->zcel); free(S->vol); free(S->dl); free(S->dd);
    for (int k = 0; k < 12; k++) free(S->sc[k]);
    double *prims[] = {S->ug, S->vg, S->wg, S->pg, S->pp, S->tg, S->phig, S->up, S->vp,
                       S->wp, S->phip, S->tp, S->rop, S->rog, S->ag, S->ap, S->egtotal,
                       S->eptotal, S->phi};
    for (size_t k = 0; k < sizeof(prims) / sizeof(prims[0]); k++) free(prims[k]);
    free(S->cn); free(S->cu); free(S->cn1); free(S->d2q); free(S->anu);
    free(S->rhs); free(S->d24);
    free(S->phiq); free(S->phir); free(S->phis); free(S->uq); free(S->vq); free(S->wq);
    free(S->ur); free(S->vr); free(S->wr); free(S->us); free(S->vs); free(S->ws);
    for (int k = 0; k < 8; k++) free(S->vis[k]);
    for (int k = 0; k < NGRAD; k++) free(S->g[k]);
    free(S->ofr); free(S->odon); free(S->ow);
    free(S);
}

/* src/sr_init_cond.F90:177-226 followed by cn = cu (main.F90:478-482) */
void or_init_uniform(or_case *S) {
    const or_params *p = &S->p;
    for (int i = 1; i <= S->neles; i++) {
        double phip = p->epslninf;
        double phig = 1 - p->epslninf;
        CU(i, 1) = phig * S->rogmin;
        CU(i, 2) = phig * S->rogmin * p->ugmin;
        CU(i, 3) = phig * S->rogmin * p->vgmin;
        CU(i, 4) = phig * S->rogmin * p->wgmin;
        CU(i, 5) = phig * S->rogmin * S->egtotalmin;
        CU(i, 6) = phip * S->ropmin;
        CU(i, 7) = phip * S->ropmin * p->upmin;
        CU(i, 8) = phip * S->ropmin * p->vpmin;
        CU(i, 9) = phip * S->ropmin * p->wpmin;
        CU(i, 10) = phip * S->ropmin * S->eptotalmin;
        if (p->five_phase) {   /* src/sr_init_cond.F90:180-208 */
            phig = 1 - phip - p->epslninf - p->epslninf - p->epslninf;
            CU(i, 1) = phig * S->rogmin;
            CU(i, 2) = phig * S->rogmin * p->ugmin;
            CU(i, 3) = phig * S->rogmin * p->vgmin;
            CU(i, 4) = phig * S->rogmin * p->wgmin;
            CU(i, 5) = phig * S->rogmin * S->egtotalmin;
            const double rho[3] = {p->rhoq, p->rhor, p->rhos};
            const double ini[3] = {p->phiqinit, p->phirinit, p->phisinit};
            for (int d = 0; d < 3; d++) {
                CU(i, 11 + 4 * d) = ini[d] * rho[d];
                CU(i, 12 + 4 * d) = ini[d] * rho[d] * p->upmin;
                CU(i, 13 + 4 * d) = ini[d] * rho[d] * p->vpmin;
                CU(i, 14 + 4 * d) = ini[d] * rho[d] * p->wpmin;
            }
        }
    }
    memcpy(S->cn, S->cu, sizeof(double) * (size_t)S->ntot * S->neq);
}

void or_set_state(or_case *S, double time, const double *cu_elem,
                  const double *ghost_prims) {
    S->time = time;
    for (int k = 1; k <= S->neq; k++)
        for (int i = 1; i <= S->neles; i++)
            CU(i, k) = cu_elem[(size_t)(k - 1) * S->neles + (i - 1)];
    if (ghost_prims) {
        double *dst[6] = {S->ug, S->vg, S->wg, S->pg, S->tg, S->rog};
        for (int v = 0; v < 6; v++)
            for (int i = 1; i <= S->nghosts; i++)
                dst[v][S->nghost[i]] = ghost_prims[(size_t)v * S->nghosts + (i - 1)];
    }
    memcpy(S->cn, S->cu, sizeof(double) * (size_t)S->ntot * S->neq);
}

/* ------------------------------------------------------------------ */
/* Phase clamp + smooth blending + density/energy re-derivation shared by
 * src/sr_primitive.F90:102-161 and src/sr_primitiveplusbc.F90:114-172.   */
static void prim_tail(or_case *S, int i) {
    const or_params *p = &S->p;
    double emin = p->epslnmin, emax = p->epslnmax;
    if (S->phig[i] < emin) {
        S->phig[i] = emin; S->phip[i] = 1.0 - S->phig[i];
        S->ug[i] = S->up[i]; S->vg[i] = S->vp[i]; S->wg[i] = S->wp[i];
        S->tg[i] = S->tp[i]; S->pg[i] = S->pp[i];
    }
    if (S->phip[i] < emin) {
        S->phip[i] = emin; S->phig[i] = 1.0 - S->phip[i];
        S->up[i] = S->ug[i]; S->vp[i] = S->vg[i]; S->wp[i] = S->wg[i];
        S->tp[i] = S->tg[i]; S->pp[i] = S->pg[i];
    }
    if (S->phig[i] >= emin && S->phig[i] <= emax) {
        double psig = (S->phig[i] - emin) / (emax - emin);
        double f = -(psig * psig * (2.0 * psig - 3.0));
        S->ug[i] = f * S->ug[i] + (1.0 - f) * S->up[i];
        S->vg[i] = f * S->vg[i] + (1.0 - f) * S->vp[i];
        S->wg[i] = f * S->wg[i] + (1.0 - f) * S->wp[i];
        S->tg[i] = f * S->tg[i] + (1.0 - f) * S->tp[i];
        S->pg[i] = f * S->pg[i] + (1.0 - f) * S->pp[i];
    }
    if (S->phip[i] >= emin && S->phip[i] <= emax) {
        double psig = (S->phip[i] - emin) / (emax - emin);
        double f = -(psig * psig * (2.0 * psig - 3.0));
        S->up[i] = f * S->up[i] + (1.0 - f) * S->ug[i];
        S->vp[i] = f * S->vp[i] + (1.0 - f) * S->vg[i];
        S->wp[i] = f * S->wp[i] + (1.0 - f) * S->wg[i];
        S->tp[i] = f * S->tp[i] + (1.0 - f) * S->tg[i];
        S->pp[i] = f * S->pp[i] + (1.0 - f) * S->pg[i];
    }
    double gamag = p->gamag, gamap = p->gamap, pinf = p->pinf, cpp = p->cpp;
    S->rog[i] = S->pg[i] / (S->rrg * S->tg[i]);
    S->rop[i] = (S->pp[i] + pinf) * gamap / ((gamap - 1.0) * cpp * S->tp[i]);
    double eg = S->pg[i] / ((gamag - 1.0) * S->rog[i]);
    double ep = (S->pp[i] + gamap * pinf) / ((gamap - 1.0) * S->rop[i]);
    S->egtotal[i] = eg + 0.5 * (sq(S->ug[i]) + sq(S->vg[i]) + sq(S->wg[i]));
    S->eptotal[i] = ep + 0.5 * (sq(S->up[i]) + sq(S->vp[i]) + sq(S->wp[i]));
    CN(i, 1) = S->phig[i] * S->rog[i];
    CN(i, 2) = S->phig[i] * S->rog[i] * S->ug[i];
    CN(i, 3) = S->phig[i] * S->rog[i] * S->vg[i];
    CN(i, 4) = S->phig[i] * S->rog[i] * S->wg[i];
    CN(i, 5) = S->phig[i] * S->rog[i] * S->egtotal[i];
    CN(i, 6) = S->phip[i] * S->rop[i];
    CN(i, 7) = S->phip[i] * S->rop[i] * S->up[i];
    CN(i, 8) = S->phip[i] * S->rop[i] * S->vp[i];
    CN(i, 9) = S->phip[i] * S->rop[i] * S->wp[i];
    CN(i, 10) = S->phip[i] * S->rop[i] * S->eptotal[i];
}

/* Conserved -> primitives through the pressure-equilibrium quadratic,
 * src/sr_primitive.F90:23-97 (with_sound = 0) and
 * src/sr_primitiveplusbc.F90:36-110 (with_sound = 1: ag, ap). */
static void prim_head(or_case *S, int i, int with_sound) {
    const or_params *p = &S->p;
    double gamag = p->gamag, gamap = p->gamap, pinf = p->pinf;
    S->ug[i] = CN(i, 2) / CN(i, 1);
    S->vg[i] = CN(i, 3) / CN(i, 1);
    S->wg[i] = CN(i, 4) / CN(i, 1);
    S->up[i] = CN(i, 7) / CN(i, 6);
    S->vp[i] = CN(i, 8) / CN(i, 6);
    S->wp[i] = CN(i, 9) / CN(i, 6);
    double eg = CN(i, 5) / CN(i, 1) - 0.5 * (sq(S->ug[i]) + sq(S->vg[i]) + sq(S->wg[i]));
    double ep = CN(i, 10) / CN(i, 6) - 0.5 * (sq(S->up[i]) + sq(S->vp[i]) + sq(S->wp[i]));
    double fs = S->foursigmabyd;
    if (p->five_phase) {
        /* src/sr_primitive.F90:56-80: the dispersed phases take their share
         * of the volume out of the pressure-equilibrium quadratic */
        double emin = p->epslnmin;
        double phq = mn2(mx2(CN(i, 11) / p->rhoq, emin), 1.0 - emin);
        double phr = mn2(mx2(CN(i, 15) / p->rhor, emin), 1.0 - emin);
        double phs = mn2(mx2(CN(i, 19) / p->rhos, emin), 1.0 - emin);
        double aaa = mn2(mx2(1.0 - phq - phr - phs, emin), 1.0 - emin);
        double bbb = (aaa * pinf * gamap) - (CN(i, 1) * (gamag - 1.0) * eg) - (CN(i, 6) * (gamap - 1.0) * ep);
        double ccc = (CN(i, 1) * (gamag - 1.0) * eg * (gamap * pinf));
        S->pg[i] = (-bbb + sqrt(sq(bbb) + 4.0 * aaa * ccc)) / (2.0 * aaa);
        S->pp[i] = S->pg[i] + fs;
        S->rog[i] = S->pg[i] / ((gamag - 1.0) * eg);
        S->rop[i] = (S->pp[i] + pinf * gamap) / ((gamap - 1.0) * ep);
        S->tg[i] = S->pg[i] / (S->rog[i] * S->rrg);
        S->tp[i] = ((S->pp[i] + pinf) * gamap) / ((gamap - 1.0) * S->rop[i] * p->cpp);
        S->phig[i] = mn2(mx2(CN(i, 1) / S->rog[i], emin), 1.0 - emin);
        S->phip[i] = mn2(mx2(CN(i, 6) / S->rop[i], emin), 1.0 - emin);
        if (with_sound) {
            S->ag[i] = sqrt((gamag * S->pg[i]) / S->rog[i]);
            S->ap[i] = sqrt((gamap * (S->pp[i] + pinf)) / S->rop[i]);
        }
        return;
    }
    double bbb = (fs + pinf * gamap) - (CN(i, 1) * (gamag - 1.0) * eg) -
                 (CN(i, 6) * (gamap - 1.0) * ep);
    double ccc = CN(i, 1) * (gamag - 1.0) * eg * (fs + pinf * gamap);
    S->pg[i] = (-bbb + sqrt(sq(bbb) + 4.0 * ccc)) * 0.5;
    S->pp[i] = S->pg[i] + fs;
    S->phig[i] = (CN(i, 1) * (gamag - 1.0) * eg) / S->pg[i];
    S->phip[i] = 1.0 - S->phig[i];
    S->rog[i] = CN(i, 1) / S->phig[i];
    S->rop[i] = CN(i, 6) / S->phip[i];
    S->tg[i] = S->pg[i] / (S->rog[i] * S->rrg);
    S->tp[i] = ((S->pp[i] + pinf) * gamap) / ((gamap - 1.0) * S->rop[i] * p->cpp);
    if (with_sound) {
        S->ag[i] = sqrt((gamag * S->pg[i]) / S->rog[i]);
        S->ap[i] = sqrt((gamap * (S->pp[i] + pinf)) / S->rop[i]);
    }
}

void or_primitive(or_case *S) {          /* src/sr_primitive.F90:18-178 */
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) { prim_head(S, i, 0); prim_tail(S, i); }
}

/* Ghost density / energy / cn of the BC loops (sr_primitiveplusbc.F90). */
static void ghost_energy_tail(or_case *S, int ng) {
    const or_params *p = &S->p;
    S->rog[ng] = S->pg[ng] / (S->rrg * S->tg[ng]);
    S->rop[ng] = p->gamap * (S->pp[ng] + p->pinf) / ((p->gamap - 1.0) * p->cpp * S->tp[ng]);
    double eg = S->rrg * S->tg[ng] / (p->gamag - 1.0);
    double ep = p->cpp * S->tp[ng] / p->gamap + p->pinf / S->rop[ng];
    S->egtotal[ng] = eg + 0.5 * (sq(S->ug[ng]) + sq(S->vg[ng]) + sq(S->wg[ng]));
    S->eptotal[ng] = ep + 0.5 * (sq(S->up[ng]) + sq(S->vp[ng]) + sq(S->wp[ng]));
}

/* Ghost states per boundary type.  viscous = 0: src/sr_primitiveplusbc.F90
 * :198-592 (with energies); viscous = 1: src/sr_viscousgp.F90:71-446
 * (primitives only; keeps the reference's wg(ng) = -wg(ng) in type 53). */
static void bc_fill(or_case *S, int viscous) {
    const or_params *p = &S->p;
    double rrg = S->rrg, gamag = p->gamag, gamap = p->gamap, pinf = p->pinf, cpp = p->cpp;
    double dt = S->dt;
    /* type 2: subsonic inflow */
    for (int ii = 1; ii <= S->nbc[0]; ii++) {
        int i = S->bcl[0][ii], np = S->nparent[i], ng = S->nghost[i];
        if (p->five_phase) {   /* sr_primitiveplusbc.F90:210-216, sr_viscousgp.F90:83-88 */
            S->phiq[ng] = p->epslnmin; S->phir[ng] = p->epslnmin; S->phis[ng] = p->epslnmin;
            S->phip[ng] = p->phipzero;
            S->phig[ng] = 1.0 - S->phip[ng] - S->phiq[ng] - S->phir[ng] - S->phis[ng];
        } else {
            S->phip[ng] = p->phipzero;
            S->phig[ng] = 1.0 - S->phip[ng];
        }
        S->ug[ng] = p->ugmin; S->vg[ng] = p->vgmin; S->wg[ng] = p->wgmin;
        S->tg[ng] = p->tgmin;
        S->pg[ng] = S->pg[np];
        S->rog[ng] = S->pg[ng] / (rrg * S->tg[ng]);
        S->up[ng] = 0.99 * p->ugmin; S->vp[ng] = 0.99 * p->vgmin; S->wp[ng] = 0.99 * p->wgmin;
        S->tp[ng] = p->tgmin;
        S->pp[ng] = S->pp[np];
        S->rop[ng] = gamap * (S->pg[ng] + pinf) / ((gamap - 1.0) * cpp * S->tp[ng]);
        if (!viscous) {
            double eg = S->pg[ng] / (S->rog[ng] * (gamag - 1.0));
            double ep = (S->pp[ng] + gamap * pinf) / (S->rop[ng] * (gamap - 1.0));
            S->egtotal[ng] = eg + 0.5 * (sq(S->ug[ng]) + sq(S->vg[ng]) + sq(S->wg[ng]));
            S->eptotal[ng] = ep + 0.5 * (sq(S->up[ng]) + sq(S->vp[ng]) + sq(S->wp[ng]));
        }
    }
    /* type 3: wave-transmissive subsonic outflow */
    for (int ii = 1; ii <= S->nbc[1]; ii++) {
        int i = S->bcl[1][ii], np = S->nparent[i], ng = S->nghost[i];
        S->phig[ng] = S->phig[np];
        S->phip[ng] = S->phip[np];
        double wT = S->ug[np];
        double wU = S->ug[np] + sqrt(gamag * S->pg[np] / S->rog[np]);
        double alphaT = wT * dt / S->dd[np];
        double alphaU = wU * dt / S->dd[np];
        double fracT = 1 / (1 + alphaT);
        double fracU = 1 / (1 + alphaU);
        if (S->total == 1) {
            S->ug[ng] = S->ug[np]; S->vg[ng] = S->vg[np]; S->wg[ng] = S->wg[np];
            S->tg[ng] = S->tg[np]; S->pg[ng] = p->pmin;
        }
        if (S->ug[np] > S->ug[ng]) {
            S->ug[ng] = S->ug[ng] * fracU + (1 - fracU) * (2.0 * S->ug[np] - S->ug[ng]);
            S->vg[ng] = S->vg[ng] * fracT + (1 - fracT) * (2.0 * S->vg[np] - S->vg[ng]);
            S->wg[ng] = S->wg[ng] * fracT + (1 - fracT) * (2.0 * S->wg[np] - S->wg[ng]);
            S->tg[ng] = S->tg[ng] * fracT + (1 - fracT) * (2.0 * S->tg[np] - S->tg[ng]);
        } else {
            S->ug[ng] = S->ug[np]; S->vg[ng] = S->vg[np]; S->wg[ng] = S->wg[np];
            S->tg[ng] = S->tg[np];
        }
        S->pg[ng] = p->pmin;
        S->rog[ng] = S->pg[ng] / (rrg * S->tg[ng]);
        S->vp[ng] = S->vp[np]; S->up[ng] = S->up[np]; S->wp[ng] = S->wp[np];
        S->pp[ng] = p->pmin;
        S->tp[ng] = S->tp[np];
        S->rop[ng] = gamap * (S->pp[ng] + pinf) / ((gamap - 1.0) * cpp * S->tp[ng]);
        if (!viscous) {
            double eg = rrg * S->tg[ng] / (gamag - 1.0);
            double ep = cpp * S->tp[ng] / gamap + pinf / S->rop[ng];
            S->egtotal[ng] = eg + 0.5 * (sq(S->ug[ng]) + sq(S->vg[ng]) + sq(S->wg[ng]));
            S->eptotal[ng] = ep + 0.5 * (sq(S->up[ng]) + sq(S->vp[ng]) + sq(S->wp[ng]));
        }
    }
    /* type 5: slip (reflecting) wall */
    for (int ii = 1; ii <= S->nbc[2]; ii++) {
        int i = S->bcl[2][ii], np = S->nparent[i], ng = S->nghost[i];
        S->phig[ng] = S->phig[np];
        S->ug[ng] = -S->ug[np]; S->vg[ng] = -S->vg[np]; S->wg[ng] = -S->wg[np];
        S->tg[ng] = S->tg[np];
        S->phip[ng] = S->phip[np];
        S->up[ng] = -S->up[np]; S->vp[ng] = -S->vp[np]; S->wp[ng] = -S->wp[np];
        S->tp[ng] = S->tp[np];
        S->pg[ng] = S->pg[np]; S->pp[ng] = S->pp[np];
        if (viscous) {
            S->rog[ng] = S->pg[ng] / (rrg * S->tg[ng]);
            S->rop[ng] = gamap * (S->pp[ng] + pinf) / ((gamap - 1.0) * cpp * S->tp[ng]);
        } else {
            ghost_energy_tail(S, ng);
        }
    }
    /* types 51 (y) and 53 (z): lateral reflect / transmissive */
    for (int lat = 0; lat < 2; lat++) {
        int list = 3 + lat;
        for (int ii = 1; ii <= S->nbc[list]; ii++) {
            int i = S->bcl[list][ii], np = S->nparent[i], ng = S->nghost[i];
            double *vn = lat == 0 ? S->vg : S->wg;       /* normal velocity */
            double *t1 = S->ug, *t2 = lat == 0 ? S->wg : S->vg;
            double wT = vn[np];
            double wU = vn[np] + sqrt(gamag * S->pg[np] / S->rog[np]);
            double alphaT = wT * dt / S->dd[np];
            double alphaU = wU * dt / S->dd[np];
            double fracT = 1 / (1 + alphaT);
            double fracU = 1 / (1 + alphaU);
            (void)fracU;
            if (vn[np] > vn[ng]) {
                if (viscous && lat == 1) vn[ng] = -vn[ng];   /* sr_viscousgp.F90:408 */
                else vn[ng] = -vn[np];
                /* update order of the reference: u first, then the other
                 * tangential component, then T */
                if (lat == 0) {
                    S->ug[ng] = S->ug[ng] * fracT + (1 - fracT) * (2.0 * S->ug[np] - S->ug[ng]);
                    S->wg[ng] = S->wg[ng] * fracT + (1 - fracT) * (2.0 * S->wg[np] - S->wg[ng]);
                } else {
                    S->ug[ng] = S->ug[ng] * fracT + (1 - fracT) * (2.0 * S->ug[np] - S->ug[ng]);
                    S->vg[ng] = S->vg[ng] * fracT + (1 - fracT) * (2.0 * S->vg[np] - S->vg[ng]);
                }
                S->tg[ng] = S->tg[ng] * fracT + (1 - fracT) * (2.0 * S->tg[np] - S->tg[ng]);
            } else {
                t1[ng] = t1[np];
                vn[ng] = -vn[np];
                t2[ng] = t2[np];
                S->tg[ng] = S->tg[np];
            }
            S->pg[ng] = S->pg[np];
            S->phig[ng] = S->phig[np];
            S->phip[ng] = S->phip[np];
            S->up[ng] = S->up[np]; S->vp[ng] = S->vp[np]; S->wp[ng] = S->wp[np];
            if (lat == 0) S->vp[ng] = -S->vp[np]; else S->wp[ng] = -S->wp[np];
            S->tp[ng] = S->tp[np];
            S->pg[ng] = S->pg[np]; S->pp[ng] = S->pp[np];
            if (viscous) {
                S->rog[ng] = S->pg[ng] / (rrg * S->tg[ng]);
                S->rop[ng] = gamap * (S->pp[ng] + pinf) / ((gamap - 1.0) * cpp * S->tp[ng]);
            } else {
                ghost_energy_tail(S, ng);
            }
        }
    }
    /* type 6 (addition): no-slip isothermal wall at twall */
    for (int ii = 1; ii <= S->nbc[5]; ii++) {
        int i = S->bcl[5][ii], np = S->nparent[i], ng = S->nghost[i];
        S->phig[ng] = S->phig[np]; S->phip[ng] = S->phip[np];
        S->ug[ng] = -S->ug[np]; S->vg[ng] = -S->vg[np]; S->wg[ng] = -S->wg[np];
        S->up[ng] = -S->up[np]; S->vp[ng] = -S->vp[np]; S->wp[ng] = -S->wp[np];
        S->tg[ng] = 2.0 * p->twall - S->tg[np];
        S->tp[ng] = 2.0 * p->twall - S->tp[np];
        S->pg[ng] = S->pg[np]; S->pp[ng] = S->pp[np];
        if (viscous) {
            S->rog[ng] = S->pg[ng] / (rrg * S->tg[ng]);
            S->rop[ng] = gamap * (S->pp[ng] + pinf) / ((gamap - 1.0) * cpp * S->tp[ng]);
        } else {
            ghost_energy_tail(S, ng);
        }
    }
    /* type 7 (addition): far field, free stream of the inflow limits */
    for (int ii = 1; ii <= S->nbc[6]; ii++) {
        int i = S->bcl[6][ii], ng = S->nghost[i];
        S->phip[ng] = p->phipzero; S->phig[ng] = 1.0 - S->phip[ng];
        S->ug[ng] = p->ugmin; S->vg[ng] = p->vgmin; S->wg[ng] = p->wgmin;
        S->up[ng] = p->upmin; S->vp[ng] = p->vpmin; S->wp[ng] = p->wpmin;
        S->tg[ng] = p->tgmin; S->tp[ng] = p->tpmin;
        S->pg[ng] = p->pmin; S->pp[ng] = p->pmin + S->foursigmabyd;
        if (viscous) {
            S->rog[ng] = S->pg[ng] / (rrg * S->tg[ng]);
            S->rop[ng] = gamap * (S->pp[ng] + pinf) / ((gamap - 1.0) * cpp * S->tp[ng]);
        } else {
            ghost_energy_tail(S, ng);
        }
    }
}

void or_primitiveplusbc(or_case *S) {    /* src/sr_primitiveplusbc.F90 */
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) { prim_head(S, i, 1); prim_tail(S, i); }
    bc_fill(S, 0);
    /* ghost cn, src/sr_primitiveplusbc.F90:602-631 */
    for (int i = 1; i <= S->nghosts; i++) {
        int ng = S->nghost[i];
        CN(ng, 1) = S->phig[ng] * S->rog[ng];
        CN(ng, 2) = S->phig[ng] * S->rog[ng] * S->ug[ng];
        CN(ng, 3) = S->phig[ng] * S->rog[ng] * S->vg[ng];
        CN(ng, 4) = S->phig[ng] * S->rog[ng] * S->wg[ng];
        CN(ng, 5) = S->phig[ng] * S->rog[ng] * S->egtotal[ng];
        CN(ng, 6) = S->phip[ng] * S->rop[ng];
        CN(ng, 7) = S->phip[ng] * S->rop[ng] * S->up[ng];
        CN(ng, 8) = S->phip[ng] * S->rop[ng] * S->vp[ng];
        CN(ng, 9) = S->phip[ng] * S->rop[ng] * S->wp[ng];
        CN(ng, 10) = S->phip[ng] * S->rop[ng] * S->eptotal[ng];
    }
}

/* ------------------------------------------------------------------ */
/* Inverse-distance^2 least squares over the 4 face neighbours,
 * src/sr_derivative.F90:45-322 (including the missing /wt4 in cTp2). */
void or_derivative(or_case *S) {
    double *fld[13] = {S->ug, S->vg, S->wg, S->tg, S->up, S->vp, S->wp, S->tp,
                       S->pg, S->pp, S->phig, S->rog, S->rop};
    static const int gidx[13] = {G_UG, G_VG, G_WG, G_TG, G_UP, G_VP, G_WP, G_TP,
                                 G_PG, G_PP, G_PHIG, G_ROG, G_ROP};
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) {
        if (S->iblank[i] != 1) continue;
        int n1 = S->nc[0][i], n2 = S->nc[1][i], n3 = S->nc[2][i], n4 = S->nc[3][i];
        double xi = S->xcel[i], yi = S->ycel[i], zi = S->zcel[i];
        double xa = S->xcel[n1] - xi, xb = S->xcel[n2] - xi, xc = S->xcel[n3] - xi, xd = S->xcel[n4] - xi;
        double ya = S->ycel[n1] - yi, yb = S->ycel[n2] - yi, yc = S->ycel[n3] - yi, yd = S->ycel[n4] - yi;
        double za = S->zcel[n1] - zi, zb = S->zcel[n2] - zi, zc = S->zcel[n3] - zi, zd = S->zcel[n4] - zi;
        double wt1 = sq(xa) + sq(ya) + sq(za);
        double wt2 = sq(xb) + sq(yb) + sq(zb);
        double wt3 = sq(xc) + sq(yc) + sq(zc);
        double wt4 = sq(xd) + sq(yd) + sq(zd);
        double a1 = sq(xa) / wt1 + sq(xb) / wt2 + sq(xc) / wt3 + sq(xd) / wt4;
        double a2 = sq(ya) / wt1 + sq(yb) / wt2 + sq(yc) / wt3 + sq(yd) / wt4;
        double a3 = sq(za) / wt1 + sq(zb) / wt2 + sq(zc) / wt3 + sq(zd) / wt4;
        double b1 = xa * ya / wt1 + xb * yb / wt2 + xc * yc / wt3 + xd * yd / wt4;
        double b2 = xa * za / wt1 + xb * zb / wt2 + xc * zc / wt3 + xd * zd / wt4;
        double b3 = za * ya / wt1 + zb * yb / wt2 + zc * yc / wt3 + zd * yd / wt4;
        double dnr = det(a1, b1, b2, b1, a2, b3, b2, b3, a3);
        for (int v = 0; v < 13; v++) {
            double *q = fld[v];
            double qi = q[i];
            double qa = q[n1] - qi, qb = q[n2] - qi, qc = q[n3] - qi, qd = q[n4] - qi;
            double c1 = qa * xa / wt1 + qb * xb / wt2 + qc * xc / wt3 + qd * xd / wt4;
            double c2;
            if (gidx[v] == G_TP)   /* cTp2 lacks the /wt4 (sr_derivative.F90:225) */
                c2 = qa * ya / wt1 + qb * yb / wt2 + qc * yc / wt3 + qd * yd;
            else
                c2 = qa * ya / wt1 + qb * yb / wt2 + qc * yc / wt3 + qd * yd / wt4;
            double c3 = qa * za / wt1 + qb * zb / wt2 + qc * zc / wt3 + qd * zd / wt4;
            S->g[gidx[v] + 0][i] = det(c1, c2, c3, b1, a2, b3, b2, b3, a3) / dnr;
            S->g[gidx[v] + 1][i] = det(a1, b1, b2, c1, c2, c3, b2, b3, a3) / dnr;
            S->g[gidx[v] + 2][i] = det(a1, b1, b2, b1, a2, b3, c1, c2, c3) / dnr;
        }
    }
}

/* Venkatakrishnan limiter, src/sr_VK.F90:32-301 */
static double venk_face(double dface, double vmax, double vmin, double vi, double epssq) {
    if (dface > 0.0) return fvenkat(vmax - vi, dface, epssq);
    if (dface < 0.0) return fvenkat(vmin - vi, dface, epssq);
    return 1.0;
}

void or_venkat(or_case *S) {
    const double *x = S->x, *y = S->y, *z = S->z;
    double K = S->p.venkat_k;
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) {
        if (S->iblank[i] != 1) continue;
        double epssq = pow(K * S->dl[i], 3.0);
        double x0 = S->xcel[i], y0 = S->ycel[i], z0 = S->zcel[i];
        int ne[4] = {S->nc[0][i], S->nc[1][i], S->nc[2][i], S->nc[3][i]};
        double fx[4], fy[4], fz[4];
        for (int f = 0; f < 4; f++) {
            int a = S->nod[HLL_FACE[f][0] - 1][i], b = S->nod[HLL_FACE[f][1] - 1][i],
                c = S->nod[HLL_FACE[f][2] - 1][i];
            fx[f] = (x[a] + x[b] + x[c]) * 0.3333 - x0;
            fy[f] = (y[a] + y[b] + y[c]) * 0.3333 - y0;
            fz[f] = (z[a] + z[b] + z[c]) * 0.3333 - z0;
        }
        double *fields[4] = {S->pg, S->pp, S->rog, S->rop};
        static const int gi[4] = {G_PG, G_PP, G_ROG, G_ROP};
        double ph[4][4];
        for (int v = 0; v < 4; v++) {
            double *q = fields[v];
            double gx = S->g[gi[v]][i], gy = S->g[gi[v] + 1][i], gz = S->g[gi[v] + 2][i];
            double vmax = mx5(q[i], q[ne[0]], q[ne[1]], q[ne[2]], q[ne[3]]);
            double vmin = mn5(q[i], q[ne[0]], q[ne[1]], q[ne[2]], q[ne[3]]);
            for (int f = 0; f < 4; f++) {
                double d = fx[f] * gx + fy[f] * gy + fz[f] * gz;
                ph[v][f] = venk_face(d, vmax, vmin, q[i], epssq);
            }
        }
        double phi = mn4(ph[0][0], ph[0][1], ph[0][2], ph[0][3]);
        phi = mn5(phi, ph[1][0], ph[1][1], ph[1][2], ph[1][3]);
        phi = mn5(phi, ph[2][0], ph[2][1], ph[2][2], ph[2][3]);
        phi = mn5(phi, ph[3][0], ph[3][1], ph[3][2], ph[3][3]);
        S->phi[i] = phi;
    }
    for (int i = 1; i <= S->nghosts; i++) S->phi[S->nghost[i]] = S->phi[S->nparent[i]];
}

/* ------------------------------------------------------------------ */
/* JST dissipation, src/sr_smooth.F90:19-374 */
void or_smooth(or_case *S) {
    for (int i = 1; i <= S->nghosts; i++) {
        int ng = S->nghost[i], np = S->nparent[i];
        S->pg[ng] = S->pg[np];
        S->pp[ng] = S->pp[np];
        for (int k = 1; k <= 10; k++) CN(ng, k) = CN(np, k);
    }
    const double e6 = R4(1.0e-6);
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) {
        int a = S->nc[0][i], b = S->nc[1][i], c = S->nc[2][i], d = S->nc[3][i];
        double *pg = S->pg, *pp = S->pp;
        double anun = fabs(pg[a] - pg[i]) + fabs(pg[b] - pg[i]) + fabs(pg[c] - pg[i]) + fabs(pg[d] - pg[i]);
        double anud = fabs(pg[a] + pg[i]) + fabs(pg[b] + pg[i]) + fabs(pg[c] + pg[i]) + fabs(pg[d] + pg[i]);
        double anupg = anun / anud;
#define SW(K)                                                                          \
    anun = fabs(CN(a, K) - CN(i, K)) + fabs(CN(b, K) - CN(i, K)) + fabs(CN(c, K) - CN(i, K)) + \
           fabs(CN(d, K) - CN(i, K));                                                  \
    anud = fabs(CN(a, K) + CN(i, K)) + fabs(CN(b, K) + CN(i, K)) + fabs(CN(c, K) + CN(i, K)) + \
           fabs(CN(d, K) + CN(i, K));
        SW(5);
        ANU(i, 1) = anupg + anun / (anud + e6);
        SW(1);
        ANU(i, 1) = ANU(i, 1) + anun / (anud + e6);
        anun = fabs(pp[a] - pp[i]) + fabs(pp[b] - pp[i]) + fabs(pp[c] - pp[i]) + fabs(pp[d] - pp[i]);
        anud = fabs(pp[a] + pp[i]) + fabs(pp[b] + pp[i]) + fabs(pp[c] + pp[i]) + fabs(pp[d] + pp[i]);
        double anupp = anun / anud;
        SW(6);
        ANU(i, 2) = anupp + anun / (anud + e6);
        SW(10);
        ANU(i, 2) = ANU(i, 2) + anun / (anud + e6);
#undef SW
        for (int k = 1; k <= 10; k++)
            D2Q(i, k) = CN(a, k) - CN(i, k) + CN(b, k) - CN(i, k) + CN(c, k) - CN(i, k) +
                        CN(d, k) - CN(i, k);
    }
    for (int i = 1; i <= S->nghosts; i++) {
        int ng = S->nghost[i], np = S->nparent[i];
        for (int k = 1; k <= 10; k++) D2Q(ng, k) = D2Q(np, k);
        ANU(ng, 1) = ANU(np, 1);
        ANU(ng, 2) = ANU(np, 2);
    }
    double dt = S->dt;
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) {
        int nb[4] = {S->nc[0][i], S->nc[1][i], S->nc[2][i], S->nc[3][i]};
        for (int set = 0; set < 2; set++) {
            double e2[4], e4[4], d2c[4], d4c[4];
            for (int f = 0; f < 4; f++) {
                e2[f] = S->co2 * mx2(ANU(i, set + 1), ANU(nb[f], set + 1));
                e4[f] = mx2(0.0, S->co4 - e2[f]);
                double d24nc = 0.5 * (S->vol[i] / dt + S->vol[nb[f]] / dt);
                d2c[f] = e2[f] * d24nc;
                d4c[f] = e4[f] * d24nc;
            }
            for (int k = 1 + 5 * set; k <= 5 + 5 * set; k++) {
                double d2 = d2c[0] * (CN(nb[0], k) - CN(i, k)) + d2c[1] * (CN(nb[1], k) - CN(i, k)) +
                            d2c[2] * (CN(nb[2], k) - CN(i, k)) + d2c[3] * (CN(nb[3], k) - CN(i, k));
                double d4 = d4c[0] * (D2Q(nb[0], k) - D2Q(i, k)) + d4c[1] * (D2Q(nb[1], k) - D2Q(i, k)) +
                            d4c[2] * (D2Q(nb[2], k) - D2Q(i, k)) + d4c[3] * (D2Q(nb[3], k) - D2Q(i, k));
                D24(i, k) = d2 - d4;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Phase clamp + blending of a reconstructed face state
 * (src/sr_hllcbatten.F90:228-318). q = {phig,ug,vg,wg,tg,pg,phip,up,vp,wp,tp,pp} */
static void face_blend(const or_params *p, double *phig, double *phip, double *ug,
                       double *vg, double *wg, double *tg, double *pg, double *up,
                       double *vp, double *wp, double *tp, double *ppv) {
    double emin = p->epslnmin, emax = p->epslnmax;
    if (*phig < emin) {
        *phig = emin; *phip = 1.0 - *phig;
        *ug = *up; *vg = *vp; *wg = *wp; *tg = *tp; *pg = *ppv;
    }
    if (*phip < emin) {
        *phip = emin; *phig = 1.0 - *phip;
        *up = *ug; *vp = *vg; *wp = *wg; *tp = *tg; *ppv = *pg;
    }
    if (*phig >= emin && *phig <= emax) {
        double psig = (*phig - emin) / (emax - emin);
        double f = -(psig * psig * (2.0 * psig - 3.0));
        *ug = f * *ug + (1.0 - f) * *up;
        *vg = f * *vg + (1.0 - f) * *vp;
        *wg = f * *wg + (1.0 - f) * *wp;
        *tg = f * *tg + (1.0 - f) * *tp;
        *pg = f * *pg + (1.0 - f) * *ppv;
    }
    if (*phip >= emin && *phip <= emax) {
        double psig = (*phip - emin) / (emax - emin);
        double f = -(psig * psig * (2.0 * psig - 3.0));
        *up = f * *up + (1.0 - f) * *ug;
        *vp = f * *vp + (1.0 - f) * *vg;
        *wp = f * *wp + (1.0 - f) * *wg;
        *tp = f * *tp + (1.0 - f) * *tg;
        *ppv = f * *ppv + (1.0 - f) * *pg;
    }
}

/* HLLC face loop.  zien = 0: HLLC-Batten, src/sr_hllcbatten.F90:59-556
 * (wave speeds, contact and branch per phase).  zien = 1: HLLC-Zien,
 * src/sr_hllczien.F90:62-502: the same reconstruction, blending and wall
 * terms, then wave speeds over both phases (:348-349), a mixture contact
 * speed (:351-363), star pressures against it (:365-366) and one branch for
 * all ten fluxes (:446-487).  The reference does not ship a run of it:
 * parity for zien = 1 is against this restatement only. */
static void hllc_zien_face(double *F, double area, double enx, double eny, double enz,
                           double phigL, double phipL, double rogL, double ropL, double ugL, double vgL,
                           double wgL, double upL, double vpL, double wpL, double pgL, double ppL,
                           double egL, double hgL, double qgL, double agL, double epL, double hpL,
                           double qpL, double apL,
                           double phigR, double phipR, double rogR, double ropR, double ugR, double vgR,
                           double wgR, double upR, double vpR, double wpR, double pgR, double ppR,
                           double egR, double hgR, double qgR, double agR, double epR, double hpR,
                           double qpR, double apR);

static void hllc_faces(or_case *S, int zien) {
    const or_params *p = &S->p;
    const double eps8 = R4(1.0e-8), eps6 = R4(1.0e-6);
    double rrg = S->rrg, gamag = p->gamag, gamap = p->gamap, pinf = p->pinf, cpp = p->cpp;
    int neles = S->neles, nghosts = S->nghosts;
    const int par = PAR(S);
#pragma omp parallel for num_threads(g_threads) if (par) schedule(static)
    for (int i = 1; i <= neles; i++) {
        if (S->iblank[i] != 1) continue;
        double Floc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        double *F = par ? Floc : S->fstar;
        for (int k = 1; k <= 10; k++) RHS(i, k) = 0.0;
        for (int f = 0; f < 4; f++) {
            int n1 = S->nod[HLL_FACE[f][0] - 1][i], n2 = S->nod[HLL_FACE[f][1] - 1][i],
                n3 = S->nod[HLL_FACE[f][2] - 1][i];
            int neigh = S->nc[f][i];
            double scx = S->sc[3 * f][i], scy = S->sc[3 * f + 1][i], scz = S->sc[3 * f + 2][i];
            double xf = (S->x[n1] + S->x[n2] + S->x[n3]) * 0.3333;
            double yf = (S->y[n1] + S->y[n2] + S->y[n3]) * 0.3333;
            double zf = (S->z[n1] + S->z[n2] + S->z[n3]) * 0.3333;
            double area = sqrt(scx * scx + scy * scy + scz * scz);
            double enx = scx / area, eny = scy / area, enz = scz / area;
            int nt = 0;
            if (neigh > neles && neigh <= neles + nghosts) nt = S->ntype[neigh - neles];
            double rogL = S->rog[i], ugL = S->ug[i], vgL = S->vg[i], wgL = S->wg[i],
                   tgL = S->tg[i], phigL = S->phig[i], ropL = S->rop[i], upL = S->up[i],
                   vpL = S->vp[i], wpL = S->wp[i], tpL = S->tp[i], pgL = S->pg[i], ppL = S->pp[i];
            double rogR = S->rog[neigh], ugR = S->ug[neigh], vgR = S->vg[neigh],
                   wgR = S->wg[neigh], tgR = S->tg[neigh], phigR = S->phig[neigh],
                   ropR = S->rop[neigh], upR = S->up[neigh], vpR = S->vp[neigh],
                   wpR = S->wp[neigh], tpR = S->tp[neigh], pgR = S->pg[neigh], ppR = S->pp[neigh];
            (void)rogL; (void)ropL; (void)rogR; (void)ropR;
            /* Zien reconstructs across element faces only (src/sr_hllczien.F90:168);
             * Batten across partition ghosts too, which this oracle has none of */
            if (p->myorder == 2 && (neigh <= neles || (!zien && neigh > neles + nghosts))) {
                double phimin = mn2(S->phi[i], S->phi[neigh]);
                double xf0 = xf - S->xcel[i], yf0 = yf - S->ycel[i], zf0 = zf - S->zcel[i];
                double xfn = xf - S->xcel[neigh], yfn = yf - S->ycel[neigh], zfn = zf - S->zcel[neigh];
#define REC(v, q, G, c)                                                                 \
    v = v + phimin * (xf##q * S->g[G][c] + yf##q * S->g[G + 1][c] + zf##q * S->g[G + 2][c])
                REC(phigL, 0, G_PHIG, i); REC(ugL, 0, G_UG, i); REC(vgL, 0, G_VG, i);
                REC(wgL, 0, G_WG, i); REC(tgL, 0, G_TG, i); REC(pgL, 0, G_PG, i);
                REC(phigR, n, G_PHIG, neigh); REC(ugR, n, G_UG, neigh); REC(vgR, n, G_VG, neigh);
                REC(wgR, n, G_WG, neigh); REC(tgR, n, G_TG, neigh); REC(pgR, n, G_PG, neigh);
                REC(upL, 0, G_UP, i); REC(vpL, 0, G_VP, i); REC(wpL, 0, G_WP, i);
                REC(tpL, 0, G_TP, i); REC(ppL, 0, G_PP, i);
                REC(upR, n, G_UP, neigh); REC(vpR, n, G_VP, neigh); REC(wpR, n, G_WP, neigh);
                REC(tpR, n, G_TP, neigh); REC(ppR, n, G_PP, neigh);
#undef REC
            }
            double phipL = 1.0 - phigL, phipR = 1.0 - phigR;
            face_blend(p, &phigL, &phipL, &ugL, &vgL, &wgL, &tgL, &pgL, &upL, &vpL, &wpL, &tpL, &ppL);
            rogL = pgL / (rrg * tgL);
            ropL = gamap * (ppL + pinf) / ((gamap - 1.0) * cpp * tpL);
            face_blend(p, &phigR, &phipR, &ugR, &vgR, &wgR, &tgR, &pgR, &upR, &vpR, &wpR, &tpR, &ppR);
            rogR = pgR / (rrg * tgR);
            ropR = gamap * (ppR + pinf) / ((gamap - 1.0) * cpp * tpR);
            if (nt == 5) {
                RHS(i, 2) = RHS(i, 2) + phigL * pgL * enx * area;
                RHS(i, 3) = RHS(i, 3) + phigL * pgL * eny * area;
                RHS(i, 4) = RHS(i, 4) + phigL * pgL * enz * area;
                RHS(i, 7) = RHS(i, 7) + phipL * ppL * enx * area;
                RHS(i, 8) = RHS(i, 8) + phipL * ppL * eny * area;
                RHS(i, 9) = RHS(i, 9) + phipL * ppL * enz * area;
                continue;
            }
            double egL = rrg * tgL / (gamag - 1.0) + 0.5 * (sq(ugL) + sq(vgL) + sq(wgL));
            double hgL = egL + pgL / rogL;
            double qgL = ugL * enx + vgL * eny + wgL * enz;
            double agL = sqrt(gamag * pgL / rogL);
            double egR = rrg * tgR / (gamag - 1.0) + 0.5 * (sq(ugR) + sq(vgR) + sq(wgR));
            double hgR = egR + pgR / rogR;
            double qgR = ugR * enx + vgR * eny + wgR * enz;
            double agR = sqrt(gamag * pgR / rogR);
            double epL = (cpp * tpL) / gamap + pinf / ropL + 0.5 * (sq(upL) + sq(vpL) + sq(wpL));
            double hpL = epL + ppL / ropL;
            double qpL = upL * enx + vpL * eny + wpL * enz;
            double apL = sqrt(gamap * (ppL + pinf) / ropL);
            double epR = (cpp * tpR) / gamap + pinf / ropR + 0.5 * (sq(upR) + sq(vpR) + sq(wpR));
            double hpR = epR + ppR / ropR;
            double qpR = upR * enx + vpR * eny + wpR * enz;
            double apR = sqrt(gamap * (ppR + pinf) / ropR);
            if (zien) {
                hllc_zien_face(F, area, enx, eny, enz, phigL, phipL, rogL, ropL, ugL, vgL, wgL, upL, vpL, wpL,
                               pgL, ppL, egL, hgL, qgL, agL, epL, hpL, qpL, apL, phigR, phipR, rogR, ropR, ugR,
                               vgR, wgR, upR, vpR, wpR, pgR, ppR, egR, hgR, qgR, agR, epR, hpR, qpR, apR);
                for (int k = 1; k <= 10; k++) RHS(i, k) = RHS(i, k) + F[k - 1];
                continue;
            }
            double sgl = mn3(qgL - agL, qgR - agR, eps8);
            double spl = mn3(qpL - apL, qpR - apR, eps8);
            double sgr = mx3(qgL + agL, qgR + agR, eps8);
            double spr = mx3(qpL + apL, qpR + apR, eps8);
            double sgnr = pgR - pgL + rogL * qgL * (sgl - qgL) - rogR * qgR * (sgr - qgR);
            double sgdr = rogL * (sgl - qgL) - rogR * (sgr - qgR);
            double sgstar = sgnr / (sgdr + eps8);
            double spnr = ppR - ppL + ropL * qpL * (spl - qpL) - ropR * qpR * (spr - qpR);
            double spdr = ropL * (spl - qpL) - ropR * (spr - qpR);
            double spstar = spnr / (spdr + eps8);
            double pgstar = mx2(pgL + rogL * (qgL - sgl) * (qgL - sgstar), eps6 * mn2(pgL, pgR));
            double ppstar = mx2(ppL + ropL * (qpL - spl) * (qpL - spstar), eps6 * mn2(ppL, ppR));
            double cnl[10], cnr[10], csl[10], csr[10], fl[10], fr[10];
            cnl[0] = phigL * rogL; cnl[1] = phigL * rogL * ugL; cnl[2] = phigL * rogL * vgL;
            cnl[3] = phigL * rogL * wgL; cnl[4] = phigL * rogL * egL;
            cnl[5] = phipL * ropL; cnl[6] = phipL * ropL * upL; cnl[7] = phipL * ropL * vpL;
            cnl[8] = phipL * ropL * wpL; cnl[9] = phipL * ropL * epL;
            cnr[0] = phigR * rogR; cnr[1] = phigR * rogR * ugR; cnr[2] = phigR * rogR * vgR;
            cnr[3] = phigR * rogR * wgR; cnr[4] = phigR * rogR * egR;
            cnr[5] = phipR * ropR; cnr[6] = phipR * ropR * upR; cnr[7] = phipR * ropR * vpR;
            cnr[8] = phipR * ropR * wpR; cnr[9] = phipR * ropR * epR;
            double dnrg = (sgstar - sgl) + eps6;
            csl[0] = (qgL - sgl) * cnl[0] / dnrg;
            csl[1] = ((qgL - sgl) * cnl[1] + phigL * (pgL * enx - pgstar * enx)) / dnrg;
            csl[2] = ((qgL - sgl) * cnl[2] + phigL * (pgL * eny - pgstar * eny)) / dnrg;
            csl[3] = ((qgL - sgl) * cnl[3] + phigL * (pgL * enz - pgstar * enz)) / dnrg;
            csl[4] = ((qgL - sgl) * cnl[4] + phigL * (pgL * qgL - pgstar * sgstar)) / dnrg;
            double dnrp = (spstar - spl) + eps6;
            csl[5] = (qpL - spl) * cnl[5] / dnrp;
            csl[6] = ((qpL - spl) * cnl[6] + phipL * (ppL * enx - ppstar * enx)) / dnrp;
            csl[7] = ((qpL - spl) * cnl[7] + phipL * (ppL * eny - ppstar * eny)) / dnrp;
            csl[8] = ((qpL - spl) * cnl[8] + phipL * (ppL * enz - ppstar * enz)) / dnrp;
            csl[9] = ((qpL - spl) * cnl[9] + phipL * (ppL * qpL - ppstar * spstar)) / dnrp;
            dnrg = (sgstar - sgr) + eps6;
            csr[0] = (qgR - sgr) * cnr[0] / dnrg;
            csr[1] = ((qgR - sgr) * cnr[1] + phigR * (pgR * enx - pgstar * enx)) / dnrg;
            csr[2] = ((qgR - sgr) * cnr[2] + phigR * (pgR * eny - pgstar * eny)) / dnrg;
            csr[3] = ((qgR - sgr) * cnr[3] + phigR * (pgR * enz - pgstar * enz)) / dnrg;
            csr[4] = ((qgR - sgr) * cnr[4] + phigR * (pgR * qgR - pgstar * sgstar)) / dnrg;
            dnrp = (spstar - spr) + eps6;
            csr[5] = (qpR - spr) * cnr[5] / dnrp;
            csr[6] = ((qpR - spr) * cnr[6] + phipR * (ppR * enx - ppstar * enx)) / dnrp;
            csr[7] = ((qpR - spr) * cnr[7] + phipR * (ppR * eny - ppstar * eny)) / dnrp;
            csr[8] = ((qpR - spr) * cnr[8] + phipR * (ppR * enz - ppstar * enz)) / dnrp;
            csr[9] = ((qpR - spr) * cnr[9] + phipR * (ppR * qpR - ppstar * spstar)) / dnrp;
            fl[0] = phigL * rogL * qgL;
            fl[1] = phigL * rogL * qgL * ugL + phigL * pgL * enx;
            fl[2] = phigL * rogL * qgL * vgL + phigL * pgL * eny;
            fl[3] = phigL * rogL * qgL * wgL + phigL * pgL * enz;
            fl[4] = phigL * rogL * qgL * hgL;
            fl[5] = phipL * ropL * qpL;
            fl[6] = phipL * ropL * qpL * upL + phipL * ppL * enx;
            fl[7] = phipL * ropL * qpL * vpL + phipL * ppL * eny;
            fl[8] = phipL * ropL * qpL * wpL + phipL * ppL * enz;
            fl[9] = phipL * ropL * qpL * hpL;
            fr[0] = phigR * rogR * qgR;
            fr[1] = phigR * rogR * qgR * ugR + phigR * pgR * enx;
            fr[2] = phigR * rogR * qgR * vgR + phigR * pgR * eny;
            fr[3] = phigR * rogR * qgR * wgR + phigR * pgR * enz;
            fr[4] = phigR * rogR * qgR * hgR;
            fr[5] = phipR * ropR * qpR;
            fr[6] = phipR * ropR * qpR * upR + phipR * ppR * enx;
            fr[7] = phipR * ropR * qpR * vpR + phipR * ppR * eny;
            fr[8] = phipR * ropR * qpR * wpR + phipR * ppR * enz;
            fr[9] = phipR * ropR * qpR * hpR;
            if (sgl > 0.0) {
                for (int k = 0; k < 5; k++) F[k] = fl[k] * area;
            } else if (sgl <= 0.0 && sgstar > 0.0) {
                for (int k = 0; k < 5; k++) F[k] = (fl[k] + sgl * (csl[k] - cnl[k])) * area;
            } else if (sgstar <= 0.0 && sgr >= 0.0) {
                for (int k = 0; k < 5; k++) F[k] = (fr[k] + sgr * (csr[k] - cnr[k])) * area;
            } else if (sgr < 0.0) {
                for (int k = 0; k < 5; k++) F[k] = fr[k] * area;
            }
            if (spl > 0.0) {
                for (int k = 5; k < 10; k++) F[k] = fl[k] * area;
            } else if (spl <= 0.0 && spstar > 0.0) {
                for (int k = 5; k < 10; k++) F[k] = (fl[k] + spl * (csl[k] - cnl[k])) * area;
            } else if (spstar <= 0.0 && spr >= 0.0) {
                for (int k = 5; k < 10; k++) F[k] = (fr[k] + spr * (csr[k] - cnr[k])) * area;
            } else if (spr < 0.0) {
                for (int k = 5; k < 10; k++) F[k] = fr[k] * area;
            }
            for (int k = 1; k <= 10; k++) RHS(i, k) = RHS(i, k) + F[k - 1];
        }
    }
}

/* One HLLC-Zien face, src/sr_hllczien.F90:348-487.  F keeps its previous
 * values when no branch is taken (NaN states), as the reference's FSTARA
 * variables do. */
static void hllc_zien_face(double *F, double area, double enx, double eny, double enz,
                           double phigL, double phipL, double rogL, double ropL, double ugL, double vgL,
                           double wgL, double upL, double vpL, double wpL, double pgL, double ppL,
                           double egL, double hgL, double qgL, double agL, double epL, double hpL,
                           double qpL, double apL,
                           double phigR, double phipR, double rogR, double ropR, double ugR, double vgR,
                           double wgR, double upR, double vpR, double wpR, double pgR, double ppR,
                           double egR, double hgR, double qgR, double agR, double epR, double hpR,
                           double qpR, double apR) {
    const double eps8 = R4(1.0e-8), eps6 = R4(1.0e-6);
    /* DMIN1/DMAX1 of five arguments, left to right */
    double sl = mn2(mn2(mn2(mn2(qgL - agL, qpL - apL), qgR - agR), qpR - apR), eps8);
    double sr = mx2(mx2(mx2(mx2(qgL + agL, qpL + apL), qgR + agR), qpR + apR), eps8);
    double rol = phigL * rogL + phipL * ropL;
    double roql = phigL * rogL * qgL + phipL * ropL * qpL;
    double ql = roql / rol;
    double prl = phigL * pgL + phipL * ppL;
    double ror = phigR * rogR + phipR * ropR;
    double roqr = phigR * rogR * qgR + phipR * ropR * qpR;
    double qr = roqr / ror;
    double prr = phigR * pgR + phipR * ppR;
    double snr = prr - prl + roql * (sl - ql) - roqr * (sr - qr);
    double sdr = rol * (sl - ql) - ror * (sr - qr);
    double sstar = snr / (sdr + eps8);
    double pgstar = mx2(pgL + rogL * (qgL - sl) * (qgL - sstar), eps6 * mn2(pgL, pgR));
    double ppstar = mx2(ppL + ropL * (qpL - sl) * (qpL - sstar), eps6 * mn2(ppL, ppR));
    double cnl[10], cnr[10], csl[10], csr[10], fl[10], fr[10];
    cnl[0] = phigL * rogL; cnl[1] = phigL * rogL * ugL; cnl[2] = phigL * rogL * vgL;
    cnl[3] = phigL * rogL * wgL; cnl[4] = phigL * rogL * egL;
    cnl[5] = phipL * ropL; cnl[6] = phipL * ropL * upL; cnl[7] = phipL * ropL * vpL;
    cnl[8] = phipL * ropL * wpL; cnl[9] = phipL * ropL * epL;
    cnr[0] = phigR * rogR; cnr[1] = phigR * rogR * ugR; cnr[2] = phigR * rogR * vgR;
    cnr[3] = phigR * rogR * wgR; cnr[4] = phigR * rogR * egR;
    cnr[5] = phipR * ropR; cnr[6] = phipR * ropR * upR; cnr[7] = phipR * ropR * vpR;
    cnr[8] = phipR * ropR * wpR; cnr[9] = phipR * ropR * epR;
    double dnr = (sstar - sl) + eps6;
    csl[0] = (qgL - sl) * cnl[0] / dnr;
    csl[1] = ((qgL - sl) * cnl[1] + phigL * (pgL * enx - pgstar * enx)) / dnr;
    csl[2] = ((qgL - sl) * cnl[2] + phigL * (pgL * eny - pgstar * eny)) / dnr;
    csl[3] = ((qgL - sl) * cnl[3] + phigL * (pgL * enz - pgstar * enz)) / dnr;
    csl[4] = ((qgL - sl) * cnl[4] + phigL * (pgL * qgL - pgstar * sstar)) / dnr;
    csl[5] = (qpL - sl) * cnl[5] / dnr;
    csl[6] = ((qpL - sl) * cnl[6] + phipL * (ppL * enx - ppstar * enx)) / dnr;
    csl[7] = ((qpL - sl) * cnl[7] + phipL * (ppL * eny - ppstar * eny)) / dnr;
    csl[8] = ((qpL - sl) * cnl[8] + phipL * (ppL * enz - ppstar * enz)) / dnr;
    csl[9] = ((qpL - sl) * cnl[9] + phipL * (ppL * qpL - ppstar * sstar)) / dnr;
    dnr = (sstar - sr) + eps6;
    csr[0] = (qgR - sr) * cnr[0] / dnr;
    csr[1] = ((qgR - sr) * cnr[1] + phigR * (pgR * enx - pgstar * enx)) / dnr;
    csr[2] = ((qgR - sr) * cnr[2] + phigR * (pgR * eny - pgstar * eny)) / dnr;
    csr[3] = ((qgR - sr) * cnr[3] + phigR * (pgR * enz - pgstar * enz)) / dnr;
    csr[4] = ((qgR - sr) * cnr[4] + phigR * (pgR * qgR - pgstar * sstar)) / dnr;
    csr[5] = (qpR - sr) * cnr[5] / dnr;
    csr[6] = ((qpR - sr) * cnr[6] + phipR * (ppR * enx - ppstar * enx)) / dnr;
    csr[7] = ((qpR - sr) * cnr[7] + phipR * (ppR * eny - ppstar * eny)) / dnr;
    csr[8] = ((qpR - sr) * cnr[8] + phipR * (ppR * enz - ppstar * enz)) / dnr;
    csr[9] = ((qpR - sr) * cnr[9] + phipR * (ppR * qpR - ppstar * sstar)) / dnr;
    fl[0] = phigL * rogL * qgL;
    fl[1] = phigL * rogL * qgL * ugL + phigL * pgL * enx;
    fl[2] = phigL * rogL * qgL * vgL + phigL * pgL * eny;
    fl[3] = phigL * rogL * qgL * wgL + phigL * pgL * enz;
    fl[4] = phigL * rogL * qgL * hgL;
    fl[5] = phipL * ropL * qpL;
    fl[6] = phipL * ropL * qpL * upL + phipL * ppL * enx;
    fl[7] = phipL * ropL * qpL * vpL + phipL * ppL * eny;
    fl[8] = phipL * ropL * qpL * wpL + phipL * ppL * enz;
    fl[9] = phipL * ropL * qpL * hpL;
    fr[0] = phigR * rogR * qgR;
    fr[1] = phigR * rogR * qgR * ugR + phigR * pgR * enx;
    fr[2] = phigR * rogR * qgR * vgR + phigR * pgR * eny;
    fr[3] = phigR * rogR * qgR * wgR + phigR * pgR * enz;
    fr[4] = phigR * rogR * qgR * hgR;
    fr[5] = phipR * ropR * qpR;
    fr[6] = phipR * ropR * qpR * upR + phipR * ppR * enx;
    fr[7] = phipR * ropR * qpR * vpR + phipR * ppR * eny;
    fr[8] = phipR * ropR * qpR * wpR + phipR * ppR * enz;
    fr[9] = phipR * ropR * qpR * hpR;
    if (sl >= 0.0) {
        for (int k = 0; k < 10; k++) F[k] = fl[k] * area;
    } else if (sl <= 0.0 && sstar > 0.0) {
        for (int k = 0; k < 10; k++) F[k] = (fl[k] + sl * (csl[k] - cnl[k])) * area;
    } else if (sstar <= 0.0 && sr >= 0.0) {
        for (int k = 0; k < 10; k++) F[k] = (fr[k] + sr * (csr[k] - cnr[k])) * area;
    } else if (sr <= 0.0) {
        for (int k = 0; k < 10; k++) F[k] = fr[k] * area;
    }
}

/* ------------------------------------------------------------------ */
/* Five-phase model: three dispersed phases q, r, s (variables 11-14,
 * 15-18, 19-22: mass and momentum, incompressible at rhoq, rhor, rhos). */

/* JST dissipation of variables 11-22, src/sr_dissipationqrs.F90:16-157:
 * switches from the liquid pressure, the liquid mass and each dispersed
 * mass; called after or_smooth, so ANU(:,1..3) may be reused. */
static void dissipation_qrs(or_case *S) {
    for (int i = 1; i <= S->nghosts; i++) {
        int ng = S->nghost[i], np = S->nparent[i];
        S->pp[ng] = S->pp[np];
        for (int k = 11; k <= 22; k++) CN(ng, k) = CN(np, k);
    }
    const double e16 = R4(1.0e-16);   /* 1.0E-16 is a REAL(4) literal */
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) {
        int a = S->nc[0][i], b = S->nc[1][i], c = S->nc[2][i], d = S->nc[3][i];
        double *pp = S->pp;
        double anun = fabs(pp[a] - pp[i]) + fabs(pp[b] - pp[i]) + fabs(pp[c] - pp[i]) + fabs(pp[d] - pp[i]);
        double anud = fabs(pp[a] + pp[i]) + fabs(pp[b] + pp[i]) + fabs(pp[c] + pp[i]) + fabs(pp[d] + pp[i]);
        double anupp = anun / anud;
#define SW(K)                                                                          \
    anun = fabs(CN(a, K) - CN(i, K)) + fabs(CN(b, K) - CN(i, K)) + fabs(CN(c, K) - CN(i, K)) + \
           fabs(CN(d, K) - CN(i, K));                                                  \
    anud = fabs(CN(a, K) + CN(i, K)) + fabs(CN(b, K) + CN(i, K)) + fabs(CN(c, K) + CN(i, K)) + \
           fabs(CN(d, K) + CN(i, K));
        SW(6);
        anupp = anupp + anun / (anud + e16);
        SW(11);
        ANU(i, 1) = anupp + anun / (anud + e16);
        SW(15);
        ANU(i, 2) = anupp + anun / (anud + e16);
        SW(19);
        ANU(i, 3) = anupp + anun / (anud + e16);
#undef SW
        for (int k = 11; k <= 22; k++)
            D2Q(i, k) = CN(a, k) - CN(i, k) + CN(b, k) - CN(i, k) + CN(c, k) - CN(i, k) +
                        CN(d, k) - CN(i, k);
    }
    for (int i = 1; i <= S->nghosts; i++) {
        int ng = S->nghost[i], np = S->nparent[i];
        for (int k = 11; k <= 22; k++) D2Q(ng, k) = D2Q(np, k);
        ANU(ng, 1) = ANU(np, 1);
        ANU(ng, 2) = ANU(np, 2);
        ANU(ng, 3) = ANU(np, 3);
    }
    double dt = S->dt;
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) {
        int nb[4] = {S->nc[0][i], S->nc[1][i], S->nc[2][i], S->nc[3][i]};
        double d24nc[4];
        for (int f = 0; f < 4; f++) d24nc[f] = 0.5 * (S->vol[i] / dt + S->vol[nb[f]] / dt);
        for (int set = 0; set < 3; set++) {
            double d2c[4], d4c[4];
            for (int f = 0; f < 4; f++) {
                double e2 = S->co2 * mx2(ANU(i, set + 1), ANU(nb[f], set + 1));
                double e4 = mx2(0.0, S->co4 - e2);
                d2c[f] = e2 * d24nc[f];
                d4c[f] = e4 * d24nc[f];
            }
            for (int k = 11 + 4 * set; k <= 14 + 4 * set; k++) {
                double d2 = d2c[0] * (CN(nb[0], k) - CN(i, k)) + d2c[1] * (CN(nb[1], k) - CN(i, k)) +
                            d2c[2] * (CN(nb[2], k) - CN(i, k)) + d2c[3] * (CN(nb[3], k) - CN(i, k));
                double d4 = d4c[0] * (D2Q(nb[0], k) - D2Q(i, k)) + d4c[1] * (D2Q(nb[1], k) - D2Q(i, k)) +
                            d4c[2] * (D2Q(nb[2], k) - D2Q(i, k)) + d4c[3] * (D2Q(nb[3], k) - D2Q(i, k));
                D24(i, k) = d2 - d4;
            }
        }
    }
}

/* Drag of the dispersed phases on the liquid, src/sr_sourceqrs.F90:42-199
 * with the constant liquid viscosity of the AMUP_CONSTANT build; every
 * element (the reference does not skip iblank != 1 here). */
static void source_qrs(or_case *S) {
    const or_params *p = &S->p;
    const double rho[3] = {p->rhoq, p->rhor, p->rhos}, rad[3] = {p->radq, p->radr, p->rads};
    const double vold[3] = {S->volq, S->volr, S->vols};
    double *phd[3] = {S->phiq, S->phir, S->phis};
    double *ud[3] = {S->uq, S->ur, S->us}, *vd[3] = {S->vq, S->vr, S->vs}, *wd[3] = {S->wq, S->wr, S->ws};
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) {
        double voli = S->vol[i];
        double amup = 0.001;
        for (int d = 0; d < 3; d++) {
            double du = S->up[i] - ud[d][i], dv = S->vp[i] - vd[d][i], dw = S->wp[i] - wd[d][i];
            double reyn = mx2(rho[d] * 2.0 * rad[d] * sqrt(sq(du) + sq(dv) + sq(dw)) / amup, 0.001);
            double relv = sqrt(sq(du) + sq(dv) + sq(dw));
            double cd;
            if (reyn < 0.1) cd = 24.0 / reyn;
            else if (reyn < 1000.0) cd = 0.48 + 28.0 / pow(reyn, 0.85);
            else cd = 0.48;
            double drag = 0.5 * cd * rho[d] * 3.1415926 * rad[d] * rad[d] * relv * (phd[d][i] / vold[d]);
            int k = 12 + 4 * d;
            RHS(i, k) = RHS(i, k) - drag * du * voli;
            RHS(i, k + 1) = RHS(i, k + 1) - drag * dv * voli - phd[d][i] * rho[d] * S->gravity * voli;
            RHS(i, k + 2) = RHS(i, k + 2) - drag * dw * voli;
            RHS(i, 7) = RHS(i, 7) + drag * du * voli;
            RHS(i, 8) = RHS(i, 8) + drag * dv * voli;
            RHS(i, 9) = RHS(i, 9) + drag * dw * voli;
        }
    }
}

/* Central fluxes of the dispersed phases, src/sr_jamesonqrs.F90:21-333:
 * volume fractions from their masses, renormalised with the two-phase
 * fractions; velocities; cn rewritten; ghost states for types 2, 3, 5; then
 * the face loop (no flux through type-5 walls) and sourceqrs. */
static void jameson_qrs(or_case *S) {
    const or_params *p = &S->p;
    const double emin = p->epslnmin;
    const double rho[3] = {p->rhoq, p->rhor, p->rhos};
    double *phd[3] = {S->phiq, S->phir, S->phis};
    double *ud[3] = {S->uq, S->ur, S->us}, *vd[3] = {S->vq, S->vr, S->vs}, *wd[3] = {S->wq, S->wr, S->ws};
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) {
        if (S->iblank[i] != 1) continue;
        for (int d = 0; d < 3; d++) phd[d][i] = mn2(mx2(CN(i, 11 + 4 * d) / rho[d], emin), 1.0 - emin);
        double phitotal = S->phig[i] + S->phip[i] + S->phiq[i] + S->phir[i] + S->phis[i];
        S->phig[i] = S->phig[i] / phitotal;
        S->phip[i] = S->phip[i] / phitotal;
        for (int d = 0; d < 3; d++) phd[d][i] = phd[d][i] / phitotal;
        for (int d = 0; d < 3; d++) {
            int k = 11 + 4 * d;
            ud[d][i] = CN(i, k + 1) / CN(i, k);
            vd[d][i] = CN(i, k + 2) / CN(i, k);
            wd[d][i] = CN(i, k + 3) / CN(i, k);
        }
        for (int d = 0; d < 3; d++) {
            int k = 11 + 4 * d;
            CN(i, k) = phd[d][i] * rho[d];
            CN(i, k + 1) = phd[d][i] * rho[d] * ud[d][i];
            CN(i, k + 2) = phd[d][i] * rho[d] * vd[d][i];
            CN(i, k + 3) = phd[d][i] * rho[d] * wd[d][i];
        }
    }
    for (int g = 1; g <= S->nghosts; g++) {
        int np = S->nparent[g], ng = S->nghost[g], nt = S->ntype[g];
        for (int k = 11; k <= 22; k++) CN(ng, k) = CN(np, k);
        if (nt == 2) {
            S->phip[ng] = emin;
            for (int d = 0; d < 3; d++) phd[d][ng] = emin;
            S->phig[ng] = 1.0 - S->phip[ng] - S->phiq[ng] - S->phir[ng] - S->phis[ng];
            for (int d = 0; d < 3; d++) { ud[d][ng] = S->up[ng]; vd[d][ng] = S->vp[ng]; wd[d][ng] = S->wp[ng]; }
        } else if (nt == 3) {
            S->phip[ng] = emin;
            for (int d = 0; d < 3; d++) phd[d][ng] = phd[d][np];
            S->phig[ng] = 1.0 - S->phip[ng] - S->phiq[ng] - S->phir[ng] - S->phis[ng];
            for (int d = 0; d < 3; d++) { ud[d][ng] = ud[d][np]; vd[d][ng] = vd[d][np]; wd[d][ng] = wd[d][np]; }
        } else if (nt == 5) {
            for (int d = 0; d < 3; d++) phd[d][ng] = phd[d][np];
            for (int d = 0; d < 3; d++) { ud[d][ng] = -ud[d][np]; vd[d][ng] = -vd[d][np]; wd[d][ng] = -wd[d][np]; }
        }
        for (int d = 0; d < 3; d++) {
            int k = 11 + 4 * d;
            CN(ng, k) = phd[d][ng] * rho[d];
            CN(ng, k + 1) = phd[d][ng] * rho[d] * ud[d][ng];
            CN(ng, k + 2) = phd[d][ng] * rho[d] * vd[d][ng];
            CN(ng, k + 3) = phd[d][ng] * rho[d] * wd[d][ng];
        }
    }
    int neles = S->neles;
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= neles; i++) {
        if (S->iblank[i] != 1) continue;
        for (int k = 11; k <= 22; k++) RHS(i, k) = 0.0;
        for (int f = 0; f < 4; f++) {
            int neigh = S->nc[f][i];
            double scx = S->sc[3 * f][i], scy = S->sc[3 * f + 1][i], scz = S->sc[3 * f + 2][i];
            double area = sqrt(scx * scx + scy * scy + scz * scz);
            double enx = scx / area, eny = scy / area, enz = scz / area;
            int nt = 0;
            if (neigh > neles) nt = S->ntype[neigh - neles];
            if (nt == 5) continue;
            for (int d = 0; d < 3; d++) {
                double qnl = ud[d][i] * enx + vd[d][i] * eny + wd[d][i] * enz;
                double qnr = ud[d][neigh] * enx + vd[d][neigh] * eny + wd[d][neigh] * enz;
                double phih = (phd[d][i] + phd[d][neigh]) * 0.5;
                double roh = (rho[d] + rho[d]) * 0.5;
                double uh = (ud[d][i] + ud[d][neigh]) * 0.5;
                double vh = (vd[d][i] + vd[d][neigh]) * 0.5;
                double wh = (wd[d][i] + wd[d][neigh]) * 0.5;
                double qh = (qnl + qnr) * 0.5;
                int k = 11 + 4 * d;
                RHS(i, k) = RHS(i, k) + (phih * roh * qh) * area;
                RHS(i, k + 1) = RHS(i, k + 1) + (phih * roh * qh * uh) * area;
                RHS(i, k + 2) = RHS(i, k + 2) + (phih * roh * qh * vh) * area;
                RHS(i, k + 3) = RHS(i, k + 3) + (phih * roh * qh * wh) * area;
            }
        }
    }
    source_qrs(S);
}

/* Interphase sources, src/sr_source.F90:42-178 */
static void source(or_case *S) {
    const or_params *p = &S->p;
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) {
        if (S->iblank[i] != 1) continue;
        double voli = S->vol[i];
        double tg = S->tg[i], phig = S->phig[i], rog = S->rog[i], rop = S->rop[i], phip = S->phip[i];
        double ug = S->ug[i], vg = S->vg[i], wg = S->wg[i], up = S->up[i], vp = S->vp[i], wp = S->wp[i];
        double amug = p->as * sqrt(tg) / (1.0 + p->ts / tg);
        double drag = 0.44 * phig * (phig - 1.0) * rog *
                      sqrt(sq(ug - up) + sq(vg - vp) + sq(wg - wp)) * S->dl[i];
        double fdgx = drag * (ug - up), fdgy = drag * (vg - vp), fdgz = drag * (wg - wp);
        double enu = 2.0;
        double qsource = 6.0 * phip * amug * p->cpg * enu * (S->tp[i] - tg) / (p->prg * sq(S->dl[i]));
        double delpstar = 2.0 * (phig * rog * phip * rop) / (phig * rop + phip * rog) *
                          (sq(ug - up) + sq(vg - vp) + sq(wg - wp));
        double pint = S->pg[i] - mn2(delpstar, 0.01 * S->pg[i]);
        double den = phig * rog + (1.0 - phig) * rop;
        double uint = (phig * rog * ug + (1.0 - phig) * rop * up) / den;
        double vint = (phig * rog * vg + (1.0 - phig) * rop * vp) / den;
        double wint = (phig * rog * wg + (1.0 - phig) * rop * wp) / den;
        int n1 = S->nc[0][i], n2 = S->nc[1][i], n3 = S->nc[2][i], n4 = S->nc[3][i];
        double xi = S->xcel[i], yi = S->ycel[i], zi = S->zcel[i];
        double xa = S->xcel[n1] - xi, xb = S->xcel[n2] - xi, xc = S->xcel[n3] - xi, xd = S->xcel[n4] - xi;
        double ya = S->ycel[n1] - yi, yb = S->ycel[n2] - yi, yc = S->ycel[n3] - yi, yd = S->ycel[n4] - yi;
        double za = S->zcel[n1] - zi, zb = S->zcel[n2] - zi, zc = S->zcel[n3] - zi, zd = S->zcel[n4] - zi;
        double pa = S->phig[n1] - phig, pb = S->phig[n2] - phig, pc = S->phig[n3] - phig, pd = S->phig[n4] - phig;
        double wt1 = sqrt(sq(xa) + sq(ya) + sq(za));
        double wt2 = sqrt(sq(xb) + sq(yb) + sq(zb));
        double wt3 = sqrt(sq(xc) + sq(yc) + sq(zc));
        double wt4 = sqrt(sq(xd) + sq(yd) + sq(zd));
        double a1 = sq(xa) / wt1 + sq(xb) / wt2 + sq(xc) / wt3 + sq(xd) / wt4;
        double a2 = sq(ya) / wt1 + sq(yb) / wt2 + sq(yc) / wt3 + sq(yd) / wt4;
        double a3 = sq(za) / wt1 + sq(zb) / wt2 + sq(zc) / wt3 + sq(zd) / wt4;
        double b1 = xa * ya / wt1 + xb * yb / wt2 + xc * yc / wt3 + xd * yd / wt4;
        double b2 = xa * za / wt1 + xb * zb / wt2 + xc * zc / wt3 + xd * zd / wt4;
        double b3 = ya * za / wt1 + yb * zb / wt2 + yc * zc / wt3 + yd * zd / wt4;
        double c1 = pa * xa / wt1 + pb * xb / wt2 + pc * xc / wt3 + pd * xd / wt4;
        double c2 = pa * ya / wt1 + pb * yb / wt2 + pc * yc / wt3 + pd * yd / wt4;
        double c3 = pa * za / wt1 + pb * zb / wt2 + pc * zc / wt3 + pd * zd / wt4;
        double dnr = det(a1, b1, b2, b1, a2, b3, b2, b3, a3);
        double dpx = det(c1, c2, c3, b1, a2, b3, b2, b3, a3) / dnr;
        double dpy = det(a1, b1, b2, c1, c2, c3, b2, b3, a3) / dnr;
        double dpz = det(a1, b1, b2, b1, a2, b3, c1, c2, c3) / dnr;
        double g = S->gravity;
        double en = pint * (uint * dpx + vint * dpy + wint * dpz) + uint * fdgx + vint * fdgy +
                    wint * fdgz + qsource;
        RHS(i, 2) = RHS(i, 2) - (fdgx + pint * dpx + phig * rog * g) * voli - S->vis[0][i];
        RHS(i, 3) = RHS(i, 3) - (fdgy + pint * dpy) * voli - S->vis[1][i];
        RHS(i, 4) = RHS(i, 4) - (fdgz + pint * dpz) * voli - S->vis[2][i];
        RHS(i, 5) = RHS(i, 5) - en * voli - S->vis[3][i];
        RHS(i, 7) = RHS(i, 7) + (fdgx + pint * dpx - phip * rop * g) * voli - S->vis[4][i];
        RHS(i, 8) = RHS(i, 8) + (fdgy + pint * dpy) * voli - S->vis[5][i];
        RHS(i, 9) = RHS(i, 9) + (fdgz + pint * dpz) * voli - S->vis[6][i];
        RHS(i, 10) = RHS(i, 10) + en * voli - S->vis[7][i];
    }
}

/* Jameson central flux, src/sr_jameson.F90:43-282 (two-phase equations).
 * Cell values on both sides of each face, with no reconstruction and no
 * phase blending: the face flux is the mean of the two sides' physical
 * fluxes times the area; a wall face (neighbour ghost of type 5) adds the
 * phase pressures only (:185-191).  The densities are the primitive arrays'
 * (:139,:145); the sound speeds the reference forms (:197,:202,:207,:212)
 * enter no flux and are left out.  The reference does not ship a run of
 * it: parity is against this restatement only. */
static void jameson_faces(or_case *S) {
    const or_params *p = &S->p;
    double rrg = S->rrg, gamag = p->gamag, gamap = p->gamap, pinf = p->pinf, cpp = p->cpp;
    int neles = S->neles, nghosts = S->nghosts;
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= neles; i++) {
        if (S->iblank[i] != 1) continue;
        for (int k = 1; k <= 10; k++) RHS(i, k) = 0.0;
        for (int f = 0; f < 4; f++) {
            int neigh = S->nc[f][i];
            double scx = S->sc[3 * f][i], scy = S->sc[3 * f + 1][i], scz = S->sc[3 * f + 2][i];
            double area = sqrt(scx * scx + scy * scy + scz * scz);
            double enx = scx / area, eny = scy / area, enz = scz / area;
            int nt = 0;
            if (neigh > neles && neigh <= neles + nghosts) nt = S->ntype[neigh - neles];
            double rogL = S->rog[i], ugL = S->ug[i], vgL = S->vg[i], wgL = S->wg[i], tgL = S->tg[i],
                   phigL = S->phig[i], ropL = S->rop[i], upL = S->up[i], vpL = S->vp[i], wpL = S->wp[i],
                   tpL = S->tp[i], pgL = S->pg[i], ppL = S->pp[i];
            double rogR = S->rog[neigh], ugR = S->ug[neigh], vgR = S->vg[neigh], wgR = S->wg[neigh],
                   tgR = S->tg[neigh], phigR = S->phig[neigh], ropR = S->rop[neigh], upR = S->up[neigh],
                   vpR = S->vp[neigh], wpR = S->wp[neigh], tpR = S->tp[neigh], pgR = S->pg[neigh],
                   ppR = S->pp[neigh];
            double phipL = 1.0 - phigL, phipR = 1.0 - phigR;
            if (nt == 5) {
                RHS(i, 2) = RHS(i, 2) + phigL * pgL * enx * area;
                RHS(i, 3) = RHS(i, 3) + phigL * pgL * eny * area;
                RHS(i, 4) = RHS(i, 4) + phigL * pgL * enz * area;
                RHS(i, 7) = RHS(i, 7) + phipL * ppL * enx * area;
                RHS(i, 8) = RHS(i, 8) + phipL * ppL * eny * area;
                RHS(i, 9) = RHS(i, 9) + phipL * ppL * enz * area;
                continue;
            }
            double egL = rrg * tgL / (gamag - 1.0) + 0.5 * (sq(ugL) + sq(vgL) + sq(wgL));
            double hgL = egL + pgL / rogL;
            double qgL = ugL * enx + vgL * eny + wgL * enz;
            double egR = rrg * tgR / (gamag - 1.0) + 0.5 * (sq(ugR) + sq(vgR) + sq(wgR));
            double hgR = egR + pgR / rogR;
            double qgR = ugR * enx + vgR * eny + wgR * enz;
            double epL = (cpp * tpL) / gamap + pinf / ropL + 0.5 * (sq(upL) + sq(vpL) + sq(wpL));
            double hpL = epL + ppL / ropL;
            double qpL = upL * enx + vpL * eny + wpL * enz;
            double epR = (cpp * tpR) / gamap + pinf / ropR + 0.5 * (sq(upR) + sq(vpR) + sq(wpR));
            double hpR = epR + ppR / ropR;
            double qpR = upR * enx + vpR * eny + wpR * enz;
            double fl[10], fr[10];
            fl[0] = phigL * rogL * qgL;
            fl[1] = phigL * rogL * qgL * ugL + phigL * pgL * enx;
            fl[2] = phigL * rogL * qgL * vgL + phigL * pgL * eny;
            fl[3] = phigL * rogL * qgL * wgL + phigL * pgL * enz;
            fl[4] = phigL * rogL * qgL * hgL;
            fl[5] = phipL * ropL * qpL;
            fl[6] = phipL * ropL * qpL * upL + phipL * ppL * enx;
            fl[7] = phipL * ropL * qpL * vpL + phipL * ppL * eny;
            fl[8] = phipL * ropL * qpL * wpL + phipL * ppL * enz;
            fl[9] = phipL * ropL * qpL * hpL;
            fr[0] = phigR * rogR * qgR;
            fr[1] = phigR * rogR * qgR * ugR + phigR * pgR * enx;
            fr[2] = phigR * rogR * qgR * vgR + phigR * pgR * eny;
            fr[3] = phigR * rogR * qgR * wgR + phigR * pgR * enz;
            fr[4] = phigR * rogR * qgR * hgR;
            fr[5] = phipR * ropR * qpR;
            fr[6] = phipR * ropR * qpR * upR + phipR * ppR * enx;
            fr[7] = phipR * ropR * qpR * vpR + phipR * ppR * eny;
            fr[8] = phipR * ropR * qpR * wpR + phipR * ppR * enz;
            fr[9] = phipR * ropR * qpR * hpR;
            /* :252-261 */
            for (int k = 1; k <= 10; k++) RHS(i, k) = RHS(i, k) + (fl[k - 1] + fr[k - 1]) * 0.5 * area;
        }
    }
}

/* CallFluxSolver, src/mod_Fluxmodule.F90:7-21: myflux 1 = HLLC-Zien
 * (src/sr_hllczien.F90:29-506), 2 = HLLC-Batten (src/sr_hllcbatten.F90:
 * 29-560), 3 = Jameson (src/sr_jameson.F90:1-288: primitiveplusbc, no
 * gradients or limiter, the central flux, source); or_create rejects any
 * other value */
void or_flux(or_case *S) {
    or_primitiveplusbc(S);
    if (S->p.myflux == 3) {
        jameson_faces(S);
        source(S);
        if (S->p.five_phase) jameson_qrs(S);    /* src/mod_Fluxmodule.F90:18-20 */
        return;
    }
    if (S->p.myorder == 2) { or_derivative(S); or_venkat(S); }
    hllc_faces(S, S->p.myflux == 1);
    source(S);
    if (S->p.five_phase) jameson_qrs(S);    /* src/mod_Fluxmodule.F90:18-20 */
}

/* ------------------------------------------------------------------ */
/* Face-centred viscous fluxes, src/sr_viscousgp.F90:37-1138 (AMUP constant) */
static const int VIS_FACE[4][3] = {{2, 3, 4}, {1, 3, 4}, {1, 2, 4}, {1, 2, 3}};

void or_viscous(or_case *S) {
    const or_params *p = &S->p;
    for (int i = 1; i <= S->neles; i++) {
        if (S->iblank[i] != 1) continue;
        for (int k = 0; k < 8; k++) S->vis[k][i] = 0.0;
    }
    bc_fill(S, 1);
    if (p->inviscid) return;
    double *fld[8] = {S->ug, S->vg, S->wg, S->tg, S->up, S->vp, S->wp, S->tp};
    double c23 = S->c23;
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= S->neles; i++) {
        if (S->iblank[i] != 1) continue;
        for (int f = 0; f < 4; f++) {
            double scx = S->sc[3 * f][i], scy = S->sc[3 * f + 1][i], scz = S->sc[3 * f + 2][i];
            int a = S->nod[VIS_FACE[f][0] - 1][i], b = S->nod[VIS_FACE[f][1] - 1][i],
                c = S->nod[VIS_FACE[f][2] - 1][i];
            double xf = (S->x[a] + S->x[b] + S->x[c]) / 3.0;
            double yf = (S->y[a] + S->y[b] + S->y[c]) / 3.0;
            double zf = (S->z[a] + S->z[b] + S->z[c]) / 3.0;
            int neigh = S->nc[f][i];
            double ff[8];
            for (int v = 0; v < 8; v++) ff[v] = (fld[v][i] + fld[v][neigh]) * 0.5;
            double phigf = (S->phig[i] + S->phig[neigh]) * 0.5;
            double tgf = ff[3];
            double amug = p->as * sqrt(tgf) / (1.0 + p->ts / tgf);
            double akg = amug * p->cpg / p->prg;
            double phipf = (S->phip[i] + S->phip[neigh]) * 0.5;
            double amup = 0.001;
            double akp = amup * p->cpp / S->prp;
            int m[8], nm;
            m[0] = S->nc[0][i]; m[1] = S->nc[1][i]; m[2] = S->nc[2][i]; m[3] = S->nc[3][i];
            if (neigh > S->neles) {
                m[4] = i; nm = 5;
            } else {
                m[4] = S->nc[0][neigh]; m[5] = S->nc[1][neigh]; m[6] = S->nc[2][neigh];
                m[7] = S->nc[3][neigh]; nm = 8;
            }
            double dx[8], dy[8], dz[8];
            for (int k = 0; k < nm; k++) {
                dx[k] = S->xcel[m[k]] - xf; dy[k] = S->ycel[m[k]] - yf; dz[k] = S->zcel[m[k]] - zf;
            }
            double a11 = 0, a22 = 0, a33 = 0, a12 = 0, a13 = 0, a23 = 0;
            a11 = sq(dx[0]); a22 = sq(dy[0]); a33 = sq(dz[0]);
            a12 = dx[0] * dy[0]; a13 = dx[0] * dz[0]; a23 = dy[0] * dz[0];
            for (int k = 1; k < nm; k++) {
                a11 = a11 + sq(dx[k]); a22 = a22 + sq(dy[k]); a33 = a33 + sq(dz[k]);
                a12 = a12 + dx[k] * dy[k]; a13 = a13 + dx[k] * dz[k]; a23 = a23 + dy[k] * dz[k];
            }
            double dnr = det(a11, a12, a13, a12, a22, a23, a13, a23, a33);
            double gr[8][3];
            for (int v = 0; v < 8; v++) {
                double d0 = fld[v][m[0]] - ff[v];
                double b1 = d0 * dx[0], b2 = d0 * dy[0], b3 = d0 * dz[0];
                for (int k = 1; k < nm; k++) {
                    double dk = fld[v][m[k]] - ff[v];
                    b1 = b1 + dk * dx[k]; b2 = b2 + dk * dy[k]; b3 = b3 + dk * dz[k];
                }
                gr[v][0] = det(b1, b2, b3, a12, a22, a23, a13, a23, a33) / dnr;
                gr[v][1] = det(a11, a12, a13, b1, b2, b3, a13, a23, a33) / dnr;
                gr[v][2] = det(a11, a12, a13, a12, a22, a23, b1, b2, b3) / dnr;
            }
            double ugf = ff[0], vgf = ff[1], wgf = ff[2], upf = ff[4], vpf = ff[5], wpf = ff[6];
            double dugx = gr[0][0], dugy = gr[0][1], dugz = gr[0][2];
            double dvgx = gr[1][0], dvgy = gr[1][1], dvgz = gr[1][2];
            double dwgx = gr[2][0], dwgy = gr[2][1], dwgz = gr[2][2];
            double dtgx = gr[3][0], dtgy = gr[3][1], dtgz = gr[3][2];
            double dupx = gr[4][0], dupy = gr[4][1], dupz = gr[4][2];
            double dvpx = gr[5][0], dvpy = gr[5][1], dvpz = gr[5][2];
            double dwpx = gr[6][0], dwpy = gr[6][1], dwpz = gr[6][2];
            double dtpx = gr[7][0], dtpy = gr[7][1], dtpz = gr[7][2];
            double delvg = dugx + dvgy + dwgz;
            double txxg = amug * (2.0 * dugx - c23 * delvg);
            double tyyg = amug * (2.0 * dvgy - c23 * delvg);
            double tzzg = amug * (2.0 * dwgz - c23 * delvg);
            double txyg = amug * (dvgx + dugy);
            double txzg = amug * (dwgx + dugz);
            double tyzg = amug * (dvgz + dwgy);
            double qxxg = ugf * txxg + vgf * txyg + wgf * txzg + akg * dtgx;
            double qyyg = ugf * txyg + vgf * tyyg + wgf * tyzg + akg * dtgy;
            double qzzg = ugf * txzg + vgf * tyzg + wgf * tzzg + akg * dtgz;
            double delvp = dupx + dvpy + dwpz;
            double txxp = amup * (2.0 * dupx - c23 * delvp);
            double tyyp = amup * (2.0 * dvpy - c23 * delvp);
            double tzzp = amup * (2.0 * dwpz - c23 * delvp);
            double txyp = amup * (dvpx + dupy);
            double txzp = amup * (dwpx + dupz);
            double tyzp = amup * (dvpz + dwpy);
            double qxxp = upf * txxp + vpf * txyp + wpf * txzp + akp * dtpx;
            double qyyp = upf * txyp + vpf * tyyp + wpf * tyzp + akp * dtpy;
            double qzzp = upf * txzp + vpf * tyzp + wpf * tzzp + akp * dtpz;
            S->vis[0][i] = S->vis[0][i] + phigf * (txxg * scx + txyg * scy + txzg * scz);
            S->vis[1][i] = S->vis[1][i] + phigf * (txyg * scx + tyyg * scy + tyzg * scz);
            S->vis[2][i] = S->vis[2][i] + phigf * (txzg * scx + tyzg * scy + tzzg * scz);
            S->vis[3][i] = S->vis[3][i] + phigf * (qxxg * scx + qyyg * scy + qzzg * scz);
            S->vis[4][i] = S->vis[4][i] + phipf * (txxp * scx + txyp * scy + txzp * scz);
            S->vis[5][i] = S->vis[5][i] + phipf * (txyp * scx + tyyp * scy + tyzp * scz);
            S->vis[6][i] = S->vis[6][i] + phipf * (txzp * scx + tyzp * scy + tzzp * scz);
            S->vis[7][i] = S->vis[7][i] + phipf * (qxxp * scx + qyyp * scy + qzzp * scz);
        }
    }
}

/* ------------------------------------------------------------------ */
/* RK stages, src/sr_RK.F90:19-164 (rk_scheme 0) or Shu-Osher SSP-RK3 */
static void stage(or_case *S, int st) {
    int ne = S->neles;
#pragma omp parallel for num_threads(g_threads) if (PAR(S)) schedule(static)
    for (int i = 1; i <= ne; i++) {
        if (S->iblank[i] != 1) continue;
        double dtbyvol = S->dt / S->vol[i];
        for (int j = 1; j <= S->neq; j++) {
            double r = RHS(i, j) - D24(i, j);
            if (S->p.rk_scheme == 0) {
                double upd = CN(i, j) - (11.0 / 20.0) * dtbyvol * r;
                if (st == 1) {
                    CN(i, j) = CU(i, j) - (11.0 / 20.0) * dtbyvol * r;
                    CN1(i, j) = CN(i, j);
                } else if (st == 2) {
                    CN(i, j) = (3.0 / 8.0) * CU(i, j) + (5.0 / 8.0) * upd;
                } else if (st == 3) {
                    CN(i, j) = (4.0 / 9.0) * CU(i, j) + (5.0 / 9.0) * upd;
                } else {
                    CN(i, j) = (111.0 / 1331.0) * CU(i, j) + (260.0 / 1331.0) * CN1(i, j) +
                               (960.0 / 1331.0) * upd;
                }
            } else {
                double upd = CN(i, j) - dtbyvol * r;
                if (st == 1) CN(i, j) = CU(i, j) - dtbyvol * r;
                else if (st == 2) CN(i, j) = 0.75 * CU(i, j) + 0.25 * upd;
                else CN(i, j) = (1.0 / 3.0) * CU(i, j) + (2.0 / 3.0) * upd;
            }
        }
    }
}

static void overset_apply(or_case *S);

static void rk(or_case *S) {
    or_viscous(S);
    int nst = S->p.rk_scheme == 0 ? 4 : 3;
    for (int st = 1; st <= nst; st++) {
        or_flux(S);
        stage(S, st);
        if (S->nfringe) overset_apply(S);
    }
}

void or_set_dt(or_case *S, double dt) { S->dt = dt; }

/* One time step, src/main.F90:515-641 */
static void one_step(or_case *S, double *diff4, double *velmag) {
    const or_params *p = &S->p;
    S->total++;
    or_primitive(S);
    S->dtmin = 1.0e8;
    /* min over cells skipping NaN: exact in any order, so chunks are
     * reduced per thread and combined */
    double dtmin = 1.0e8;
#pragma omp parallel num_threads(g_threads) if (PAR(S))
    {
        double loc = 1.0e8;
#pragma omp for schedule(static)
        for (int i = 1; i <= S->neles; i++) {
            S->ag[i] = sqrt((p->gamag * S->pg[i]) / S->rog[i]);
            S->ap[i] = sqrt((p->gamap * (S->pp[i] + p->pinf)) / S->rop[i]);
            double qgi = sqrt(sq(S->ug[i]) + sq(S->vg[i]) + sq(S->wg[i]));
            double qpi = sqrt(sq(S->up[i]) + sq(S->vp[i]) + sq(S->wp[i]));
            loc = mn2(loc, S->dl[i] / (mx2(S->ag[i], S->ap[i]) + mx2(qgi, qpi)));
        }
#pragma omp critical
        dtmin = mn2(dtmin, loc);
    }
    S->dtmin = dtmin;
    S->dt = S->dtmin * p->cfl;
    S->time = S->time + S->dt;
    or_smooth(S);
    if (p->five_phase) dissipation_qrs(S);   /* src/main.F90:570-572 */
    rk(S);
    or_primitive(S);
    double dp = 0, du = 0, dv = 0, dw = 0;
    for (int i = 1; i <= S->neles; i++) {
        dp = mx2(dp, fabs(CN(i, 1) - CU(i, 1)));
        du = mx2(du, fabs(CN(i, 2) - CU(i, 2)));
        dv = mx2(dv, fabs(CN(i, 3) - CU(i, 3)));
        dw = mx2(dw, fabs(CN(i, 4) - CU(i, 4)));
    }
    memcpy(S->cu, S->cn, sizeof(double) * (size_t)S->ntot * S->neq);
    if (diff4) { diff4[0] = dp; diff4[1] = du; diff4[2] = dv; diff4[3] = dw; }
    if (velmag) *velmag = sqrt(sq(S->ug[1]) + sq(S->vg[1]) + sq(S->wg[1]));
}

int or_run(or_case *S, int32_t nsteps, double *time_out, double *velmag_out,
           double *diff_out) {
    g_nan_mode = S->p.nan_mode;
    for (int s = 0; s < nsteps; s++) {
        double d4[4], vm;
        one_step(S, d4, &vm);
        if (time_out) time_out[s] = S->time;
        if (velmag_out) velmag_out[s] = vm;
        if (diff_out) memcpy(diff_out + 4 * (size_t)s, d4, sizeof d4);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
double or_time(const or_case *S) { return S->time; }
double or_last_dt(const or_case *S) { return S->dt; }
int32_t or_ntot(const or_case *S) { return S->ntot; }
void or_get_cu(const or_case *S, double *out) {
    memcpy(out, S->cu, sizeof(double) * (size_t)S->ntot * S->neq);
}
void or_get_cn(const or_case *S, double *out) {
    memcpy(out, S->cn, sizeof(double) * (size_t)S->ntot * S->neq);
}
/* ug,vg,wg,pg,pp,tg,phig,up,vp,wp,phip,tp,rop,rog,ag,ap */
void or_get_prims(const or_case *S, double *out) {
    const double *a[16] = {S->ug, S->vg, S->wg, S->pg, S->pp, S->tg, S->phig, S->up,
                           S->vp, S->wp, S->phip, S->tp, S->rop, S->rog, S->ag, S->ap};
    for (int v = 0; v < 16; v++)
        memcpy(out + (size_t)v * S->ntot, a[v] + 1, sizeof(double) * S->ntot);
}
/* xcel,ycel,zcel,vol,dl,dd, sc1x..sc4z, then nc1..nc4 as doubles */
void or_get_geometry(const or_case *S, double *out) {
    const double *a[18] = {S->xcel, S->ycel, S->zcel, S->vol, S->dl, S->dd,
                           S->sc[0], S->sc[1], S->sc[2], S->sc[3], S->sc[4], S->sc[5],
                           S->sc[6], S->sc[7], S->sc[8], S->sc[9], S->sc[10], S->sc[11]};
    for (int v = 0; v < 18; v++)
        memcpy(out + (size_t)v * S->ntot, a[v] + 1, sizeof(double) * S->ntot);
    for (int k = 0; k < 4; k++)
        for (int i = 1; i <= S->ntot; i++) out[(size_t)(18 + k) * S->ntot + i - 1] = S->nc[k][i];
}
void or_get_ghost_restart(const or_case *S, double *out) {
    const double *a[6] = {S->ug, S->vg, S->wg, S->pg, S->tg, S->rog};
    for (int v = 0; v < 6; v++)
        for (int i = 1; i <= S->nghosts; i++) out[(size_t)v * S->nghosts + i - 1] = a[v][S->nghost[i]];
}
void or_get_rhs(const or_case *S, double *out) {
    memcpy(out, S->rhs, sizeof(double) * (size_t)S->neles * S->neq);
}
void or_get_d24(const or_case *S, double *out) {
    memcpy(out, S->d24, sizeof(double) * (size_t)S->neles * S->neq);
}
void or_get_vis(const or_case *S, double *out) {
    for (int v = 0; v < 8; v++)
        memcpy(out + (size_t)v * S->neles, S->vis[v] + 1, sizeof(double) * S->neles);
}
void or_get_grad(const or_case *S, double *out) {
    for (int v = 0; v < NGRAD; v++)
        memcpy(out + (size_t)v * S->ntot, S->g[v] + 1, sizeof(double) * S->ntot);
    memcpy(out + (size_t)NGRAD * S->ntot, S->phi + 1, sizeof(double) * S->ntot);
}

/* ------------------------------------------------------------------ */
/* Overset fringe interpolation.  New work: the reference only freezes
 * cells with iblank != 1 (src/sr_RK.F90:31; its hole cutting comes from
 * TIOGA, outside the path).  Test infrastructure: the library's own
 * hp_overset_build (csrc/hp_overset.cpp) and the device interpolation are
 * checked against this restatement of the same rules.
 *
 * Fringe: background (block 0) field cells next to a hole cell (iblank 0),
 * component (block 1) field cells next to a ghost of type outer_type, then
 * `layers - 1` further layers of field cells of the same block next to the
 * previous layer; fringe cells get iblank -1.
 * Donor cell D of a fringe cell with centroid x: the lowest-id field cell of
 * the other block whose tet contains x (barycentric coordinates >= -1e-10);
 * if none does, the field cell of that block with the nearest centroid.
 * Weights: barycentric coordinates of x in a tet spanned by four centroids
 * among D, its field neighbours and theirs (two rings, face order): of the
 * tets that contain x (coordinates >= -1e-12), the one whose vertices are
 * closest to x (least sum of squared distances); if none contains x, the one
 * whose smallest coordinate is largest; D alone (weight 1) without any tet.
 * Every RK stage then sets cn of each fringe cell to sum_k w_k cn(donor_k). */
static double ov_bary(const double p0[3], const double p1[3], const double p2[3], const double p3[3],
                      const double x[3], double lam[4]) {
    double a[3], b[3], c[3], d[3];
    for (int k = 0; k < 3; k++) {
        a[k] = p1[k] - p0[k]; b[k] = p2[k] - p0[k]; c[k] = p3[k] - p0[k]; d[k] = x[k] - p0[k];
    }
    double v = det(a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]);
    if (v == 0.0) return 0.0;
    double l1 = det(d[0], d[1], d[2], b[0], b[1], b[2], c[0], c[1], c[2]) / v;
    double l2 = det(a[0], a[1], a[2], d[0], d[1], d[2], c[0], c[1], c[2]) / v;
    double l3 = det(a[0], a[1], a[2], b[0], b[1], b[2], d[0], d[1], d[2]) / v;
    lam[0] = 1.0 - l1 - l2 - l3; lam[1] = l1; lam[2] = l2; lam[3] = l3;
    return v;
}

static void ov_centroid(const double *x, const double *y, const double *z, const int32_t *r, double c[3]) {
    c[0] = 0.25 * (x[r[0] - 1] + x[r[1] - 1] + x[r[2] - 1] + x[r[3] - 1]);
    c[1] = 0.25 * (y[r[0] - 1] + y[r[1] - 1] + y[r[2] - 1] + y[r[3] - 1]);
    c[2] = 0.25 * (z[r[0] - 1] + z[r[1] - 1] + z[r[2] - 1] + z[r[3] - 1]);
}

int or_overset_build(int32_t nodes, int32_t neles, int32_t nghosts, const double *x, const double *y,
                     const double *z, const int32_t *elem, const int32_t *ghost, const int32_t *block,
                     int32_t layers, int32_t outer_type, int32_t *iblank_out, int32_t *nfringe,
                     int32_t *fringe, int32_t *donor, double *weight, int32_t *nfallback) {
    (void)nodes;
    const int ntot = neles + nghosts;
    int *gtype = ialloc(ntot + 2), *mark = ialloc(neles + 1);
    for (int g = 0; g < nghosts; g++) {
        int id = ghost[4 * g + 1];
        if (id >= 1 && id <= ntot) gtype[id] = ghost[4 * g + 2];
    }
#define ROW(e) (elem + 9 * (size_t)((e) - 1))
    for (int e = 1; e <= neles; e++) {
        const int32_t *r = ROW(e);
        if (r[8] != 1) continue;
        for (int k = 0; k < 4; k++) {
            int n = r[4 + k];
            if ((block[e - 1] == 0 && n <= neles && ROW(n)[8] == 0) ||
                (block[e - 1] == 1 && n > neles && gtype[n] == outer_type)) { mark[e] = 1; break; }
        }
    }
    for (int l = 2; l <= layers; l++)
        for (int e = 1; e <= neles; e++) {
            const int32_t *r = ROW(e);
            if (r[8] != 1 || mark[e]) continue;
            for (int k = 0; k < 4; k++) {
                int n = r[4 + k];
                if (n <= neles && mark[n] == l - 1 && block[n - 1] == block[e - 1]) { mark[e] = l; break; }
            }
        }
    int nf = 0, nfb = 0;
    for (int e = 1; e <= neles; e++) {
        iblank_out[e - 1] = mark[e] ? -1 : ROW(e)[8];
        if (mark[e]) fringe[nf++] = e;
    }
    for (int f = 0; f < nf; f++) {
        const int e = fringe[f], B = 1 - block[e - 1];
        double xp[3];
        ov_centroid(x, y, z, ROW(e), xp);
        int D = 0;
        for (int t = 1; t <= neles && !D; t++) {
            if (iblank_out[t - 1] != 1 || block[t - 1] != B) continue;
            const int32_t *r = ROW(t);
            double p[4][3], lam[4];
            for (int k = 0; k < 4; k++) { p[k][0] = x[r[k] - 1]; p[k][1] = y[r[k] - 1]; p[k][2] = z[r[k] - 1]; }
            if (ov_bary(p[0], p[1], p[2], p[3], xp, lam) == 0.0) continue;
            if (lam[0] >= -1e-10 && lam[1] >= -1e-10 && lam[2] >= -1e-10 && lam[3] >= -1e-10) D = t;
        }
        if (!D) {
            double best = 0.0;
            for (int t = 1; t <= neles; t++) {
                if (iblank_out[t - 1] != 1 || block[t - 1] != B) continue;
                double c[3];
                ov_centroid(x, y, z, ROW(t), c);
                double d2 = (c[0] - xp[0]) * (c[0] - xp[0]) + (c[1] - xp[1]) * (c[1] - xp[1]) +
                            (c[2] - xp[2]) * (c[2] - xp[2]);
                if (!D || d2 < best) { best = d2; D = t; }
            }
            nfb++;
        }
        int *dn = donor + 4 * (size_t)f;
        double *w = weight + 4 * (size_t)f;
        dn[0] = dn[1] = dn[2] = dn[3] = D;
        w[0] = 1.0; w[1] = w[2] = w[3] = 0.0;
        if (!D) { dn[0] = dn[1] = dn[2] = dn[3] = e; continue; }   /* no field cell at all */
        /* candidates: D, its field neighbours, theirs (two rings, face order) */
        int cand[17], m = 0;
        cand[m++] = D;
        for (int ring = 0, lo = 0; ring < 2; ring++) {
            int hi = m;
            for (int a = lo; a < hi; a++)
                for (int k = 0; k < 4 && m < 17; k++) {
                    int n = ROW(cand[a])[4 + k];
                    if (n > neles || iblank_out[n - 1] != 1 || block[n - 1] != B) continue;
                    int seen = 0;
                    for (int q = 0; q < m; q++) seen |= (cand[q] == n);
                    if (!seen) cand[m++] = n;
                }
            lo = hi;
        }
        double cc[17][3];
        for (int a = 0; a < m; a++) ov_centroid(x, y, z, ROW(cand[a]), cc[a]);
        /* the containing tet (coordinates >= -1e-12) whose vertices are
         * closest to x (sum of squared distances); none containing x: the
         * tet whose smallest coordinate is largest */
        double best_in = 0.0, best_out = -1.0e300;
        int have_in = 0;
        for (int i = 0; i < m; i++)
            for (int j = i + 1; j < m; j++)
                for (int k = j + 1; k < m; k++)
                    for (int l = k + 1; l < m; l++) {
                        double lam[4];
                        if (ov_bary(cc[i], cc[j], cc[k], cc[l], xp, lam) == 0.0) continue;
                        double sc = mn4(lam[0], lam[1], lam[2], lam[3]);
                        const int id[4] = {i, j, k, l};
                        if (sc >= -1e-12) {
                            double s2 = 0.0;
                            for (int q = 0; q < 4; q++)
                                s2 = s2 + ((cc[id[q]][0] - xp[0]) * (cc[id[q]][0] - xp[0]) +
                                           (cc[id[q]][1] - xp[1]) * (cc[id[q]][1] - xp[1]) +
                                           (cc[id[q]][2] - xp[2]) * (cc[id[q]][2] - xp[2]));
                            if (!have_in || s2 < best_in) {
                                have_in = 1; best_in = s2;
                                for (int q = 0; q < 4; q++) { dn[q] = cand[id[q]]; w[q] = lam[q]; }
                            }
                        } else if (!have_in && sc > best_out) {
                            best_out = sc;
                            for (int q = 0; q < 4; q++) { dn[q] = cand[id[q]]; w[q] = lam[q]; }
                        }
                    }
    }
#undef ROW
    *nfringe = nf;
    if (nfallback) *nfallback = nfb;
    free(gtype); free(mark);
    return 0;
}

void or_set_overset(or_case *S, int32_t nfringe, const int32_t *fringe, const int32_t *donor,
                    const double *weight) {
    free(S->ofr); free(S->odon); free(S->ow);
    S->nfringe = nfringe;
    S->ofr = ialloc(nfringe + 1); S->odon = ialloc(4 * (size_t)nfringe + 1);
    S->ow = dalloc(4 * (size_t)nfringe + 1);
    memcpy(S->ofr, fringe, sizeof(int) * (size_t)nfringe);
    memcpy(S->odon, donor, sizeof(int) * 4 * (size_t)nfringe);
    memcpy(S->ow, weight, sizeof(double) * 4 * (size_t)nfringe);
}

static void overset_apply(or_case *S) {
    for (int f = 0; f < S->nfringe; f++) {
        const int i = S->ofr[f];
        const int *d = S->odon + 4 * (size_t)f;
        const double *w = S->ow + 4 * (size_t)f;
        for (int j = 1; j <= NEQ; j++)
            CN(i, j) = w[0] * CN(d[0], j) + w[1] * CN(d[1], j) + w[2] * CN(d[2], j) + w[3] * CN(d[3], j);
    }
}

/* ------------------------------------------------------------------ */
/* Overset hole cut.  New work: the reference takes its hole cut from
 * TIOGA, outside the path, and only freezes cells with iblank != 1
 * (src/sr_RK.F90:31).  Test infrastructure: the library's
 * hp_overset_hole_cut (csrc/hp_overset.cpp) and hp_overset_hole_cut_gpu
 * (csrc/hp_overset_gpu.cu) are checked against this brute-force
 * restatement of the rule.
 *
 * Wall surface: the faces of component (block 1) elements whose neighbour
 * is a ghost of type wall_type; face k of an element is the triangle of its
 * nodes other than node k, in the node order of src/sr_geometry.F90:149-158
 * ((2,3,4), (4,3,1), (2,4,1), (3,2,1)).  A background (block 0) field cell
 * (iblank 1) becomes a hole (iblank 0) when its centroid p
 *   - lies within `margin` of the surface: the squared distance to some wall
 *     triangle is <= margin*margin, or
 *   - is enclosed by it: the ray from p towards +x crosses an odd number of
 *     wall triangles.
 * A crossing is decided in the (y, z) projection.  Each edge function is
 * evaluated from the lexicographically lower end of its edge, so the two
 * triangles that share an edge see exactly opposite values; where an edge
 * function is zero it takes the sign it has once p moves by (0, eps, eps^2)
 * (simulation of simplicity), so a ray through an edge or a vertex counts
 * one triangle of those around it.  The crossing counts when the hit point
 * lies at x > p.x.  The surface must be closed, or open only across planes
 * parallel to the x axis (an extruded body between planes z = const).
 * Other cells keep their iblank. */
static double hc_dot(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static void hc_cross3(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

/* squared distance from p to the segment u-v */
static double hc_seg2(const double p[3], const double u[3], const double v[3]) {
    double w[3], d[3];
    for (int k = 0; k < 3; k++) { w[k] = v[k] - u[k]; d[k] = p[k] - u[k]; }
    double ww = hc_dot(w, w), t = hc_dot(d, w);
    if (t <= 0.0 || ww == 0.0) return hc_dot(d, d);
    if (t >= ww) {
        double q[3] = {p[0] - v[0], p[1] - v[1], p[2] - v[2]};
        return hc_dot(q, q);
    }
    double s = t / ww, q[3];
    for (int k = 0; k < 3; k++) q[k] = d[k] - s * w[k];
    return hc_dot(q, q);
}

/* squared distance from p to the triangle a, b, c */
static double hc_dist2(const double p[3], const double a[3], const double b[3], const double c[3]) {
    double ab[3], ac[3], n[3];
    for (int k = 0; k < 3; k++) { ab[k] = b[k] - a[k]; ac[k] = c[k] - a[k]; }
    hc_cross3(ab, ac, n);
    double nn = hc_dot(n, n);
    if (nn > 0.0) {
        const double *V[3] = {a, b, c};
        int in = 1;
        for (int q = 0; q < 3 && in; q++) {
            const double *u = V[q], *v = V[(q + 1) % 3];
            double e[3], d[3], x[3];
            for (int k = 0; k < 3; k++) { e[k] = v[k] - u[k]; d[k] = p[k] - u[k]; }
            hc_cross3(e, d, x);
            in = hc_dot(n, x) >= 0.0;
        }
        if (in) {
            double ap[3] = {p[0] - a[0], p[1] - a[1], p[2] - a[2]};
            double h = hc_dot(ap, n);
            return h * h / nn;
        }
    }
    double d0 = hc_seg2(p, a, b), d1 = hc_seg2(p, b, c), d2 = hc_seg2(p, c, a);
    return d0 < d1 ? (d0 < d2 ? d0 : d2) : (d1 < d2 ? d1 : d2);
}

/* sign (+1/-1) of the projected edge function of u->v at p (value in *val);
 * 0 when u and v coincide in projection */
static int hc_edge(const double u[3], const double v[3], const double p[3], double *val) {
    int swap = u[1] > v[1] || (u[1] == v[1] && u[2] > v[2]);
    const double *s = swap ? v : u, *t = swap ? u : v;
    double dy = t[1] - s[1], dz = t[2] - s[2];
    if (dy == 0.0 && dz == 0.0) { *val = 0.0; return 0; }
    double e = dy * (p[2] - s[2]) - dz * (p[1] - s[1]);
    int sg = e > 0.0 ? 1 : e < 0.0 ? -1 : (dz != 0.0 ? (dz > 0.0 ? -1 : 1) : 1);
    *val = swap ? -e : e;
    return swap ? -sg : sg;
}

/* 1 if the ray from p towards +x crosses the triangle a, b, c */
static int hc_ray(const double p[3], const double a[3], const double b[3], const double c[3]) {
    double ea, eb, ec;
    int sa = hc_edge(b, c, p, &ea), sb = hc_edge(c, a, p, &eb), sc = hc_edge(a, b, p, &ec);
    if (sa == 0 || sb == 0 || sc == 0 || sa != sb || sb != sc) return 0;
    double den = ea + eb + ec;
    double xh = den != 0.0 ? (ea * a[0] + eb * b[0] + ec * c[0]) / den : a[0];
    return xh > p[0];
}

int or_overset_hole_cut(int32_t nodes, int32_t neles, int32_t nghosts, const double *x, const double *y,
                        const double *z, const int32_t *elem, const int32_t *ghost, const int32_t *block,
                        int32_t wall_type, double margin, int32_t *iblank_out, int32_t *nholes) {
    (void)nodes;
    static const int FACE[4][3] = {{2, 3, 4}, {4, 3, 1}, {2, 4, 1}, {3, 2, 1}};
    const int ntot = neles + nghosts;
    int *gtype = ialloc(ntot + 2);
    for (int g = 0; g < nghosts; g++) {
        int id = ghost[4 * g + 1];
        if (id >= 1 && id <= ntot) gtype[id] = ghost[4 * g + 2];
    }
    int ntri = 0;
    for (int e = 1; e <= neles; e++)
        for (int k = 0; k < 4; k++) {
            int n = elem[9 * (size_t)(e - 1) + 4 + k];
            ntri += block[e - 1] == 1 && n > neles && gtype[n] == wall_type;
        }
    double *tri = dalloc(9 * (size_t)ntri + 1);
    int t = 0;
    for (int e = 1; e <= neles; e++)
        for (int k = 0; k < 4; k++) {
            const int32_t *r = elem + 9 * (size_t)(e - 1);
            int n = r[4 + k];
            if (!(block[e - 1] == 1 && n > neles && gtype[n] == wall_type)) continue;
            for (int v = 0; v < 3; v++) {
                int nd = r[FACE[k][v] - 1];
                tri[9 * (size_t)t + 3 * v + 0] = x[nd - 1];
                tri[9 * (size_t)t + 3 * v + 1] = y[nd - 1];
                tri[9 * (size_t)t + 3 * v + 2] = z[nd - 1];
            }
            t++;
        }
    const double m2 = margin * margin;
    int nh = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : nh)
    for (int e = 1; e <= neles; e++) {
        const int32_t *r = elem + 9 * (size_t)(e - 1);
        int ib = r[8];
        if (block[e - 1] == 0 && ib == 1) {
            double p[3];
            ov_centroid(x, y, z, r, p);
            int hole = 0, par = 0;
            for (int q = 0; q < ntri && !hole; q++) {
                const double *T = tri + 9 * (size_t)q;
                hole = hc_dist2(p, T, T + 3, T + 6) <= m2;
                par ^= hc_ray(p, T, T + 3, T + 6);
            }
            if (hole || par) { ib = 0; nh++; }
        }
        iblank_out[e - 1] = ib;
    }
    *nholes = nh;
    free(gtype); free(tri);
    return ntri > 0 ? 0 : -1;
}
