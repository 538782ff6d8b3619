/*
 * hydra_oracle.h -- CPU oracle for the two-phase residual/update step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a sequential FP64 restatement of the
 * reference solver's explicit time-step path (HydraPhase_60_FPC_5mill,
 * Fortran 90).  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load it, and only as the checker.
 * The product library never links or calls it.
 *
 * Parity pin: the oracle is checked against the reference's own shipped
 * outputs for the shipped case (Velocity.dat lines 131-140 and
 * restart_files/restart0000.in after 10 steps of flow.in) by
 * tests/test_oracle_pin.py.
 *
 * Indexing follows the reference: cells are 1-based, the conserved state is
 * column-major cn(ntot, neq) with ntot = neles + nghosts (one partition).
 */
#ifndef HYDRA_ORACLE_H
#define HYDRA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* flow.in fields in file order (src/sr_Read_flow.F90:19-268) plus the
 * switches this build adds on top of the reference scheme. */
typedef struct or_params {
    double pmax, pmin, tgmax, tgmin;
    double ugmax, ugmin, vgmax, vgmin, wgmax, wgmin;
    double upmax, upmin, vpmax, vpmin, wpmax, wpmin;
    double tpmax, tpmin;
    double pinf, gamap, gamag, cpp, cpg, amolg, prg, epslnmax;
    double epslnmin, epslninf, phipzero;
    double cfl;
    int32_t niter, itersub;
    int32_t istart;
    double diap;
    double surfacetension;
    int32_t myflux;
    int32_t myorder;
    double as, ts;
    /* --- additions (no reference counterpart; defaults reproduce it) --- */
    int32_t nan_mode;   /* 0: MIN/MAX skip a NaN argument (pinned default);
                           1: x86 MIN_EXPR/MAX_EXPR ordering */
    double venkat_k;    /* limiter eps^2 = (K*dl)^3; reference K = 0.3 */
    int32_t rk_scheme;  /* 0: reference 4-stage ESSPRK; 1: Shu-Osher SSP-RK3 */
    int32_t inviscid;   /* 1: skip the viscous face fluxes (vis* = 0) */
    double twall;       /* isothermal wall temperature for BC type 6 */
    double pad_[3];
    /* five-phase model (the reference's FIVE_PHASE build): three dispersed,
     * incompressible phases q, r, s with mass and momentum each, so
     * neq = 22.  flow.in groups 19-21 (src/sr_Read_flow.F90:214-250). */
    int32_t five_phase;
    double rhoq, rhor, rhos;            /* phase densities */
    double radq, radr, rads;            /* particle radii */
    double phiqinit, phirinit, phisinit;/* volume fractions of the uniform start */
} or_params;

typedef struct or_case or_case;

/* Mesh arrays exactly as the reference reads them (sr_geometry.F90:101-139):
 * x,y,z[nodes]; elem[neles*9] = nod1..4, nc1..4, iblank per element (row
 * order, 1-based ids); ghost[nghosts*4] = nparent, nghost, ntype, nside. */
or_case *or_create(const or_params *p, int32_t nodes, int32_t neles,
                   int32_t nghosts, const double *x, const double *y,
                   const double *z, const int32_t *elem,
                   const int32_t *ghost);
void or_destroy(or_case *c);

/* sr_init_cond.F90:177-226 (uniform state) followed by cn = cu. */
void or_init_uniform(or_case *c);
/* Restart-style state injection (main.F90:427-441): cu for elements
 * (column-major neles x neq) and ug,vg,wg,pg,tg,rog at the ghost ids
 * (nghosts each, in ghost-list order). ghost_prims may be NULL. */
void or_set_state(or_case *c, double time, const double *cu_elem,
                  const double *ghost_prims);

/* Run nsteps of main.F90:511-657.  Per-step diagnostics go to the optional
 * arrays (length nsteps): simulation time, |u_g(cell 1)| and the four
 * max-norm differences (diffp, diffu, diffv, diffw). */
int or_run(or_case *c, int32_t nsteps, double *time_out, double *velmag_out,
           double *diff_out);

/* Copy-out accessors. */
double or_time(const or_case *c);
int32_t or_ntot(const or_case *c);
void or_get_cu(const or_case *c, double *out);          /* ntot x 10 col-major */
void or_get_cn(const or_case *c, double *out);          /* ntot x 10 col-major */
void or_get_prims(const or_case *c, double *out);       /* 16 x ntot, see .c */
void or_get_geometry(const or_case *c, double *out);    /* 19 x ntot, see .c */
void or_get_ghost_restart(const or_case *c, double *out); /* 6 x nghosts */
void or_get_rhs(const or_case *c, double *out);         /* neles x 10 */
void or_get_d24(const or_case *c, double *out);         /* neles x 10 */
void or_get_vis(const or_case *c, double *out);         /* 8 x neles */
void or_get_grad(const or_case *c, double *out);        /* 33 x ntot + phi */
double or_last_dt(const or_case *c);

/* OpenMP threads for the cell loops of meshes without aliased ghost ids
 * (results are identical for any thread count). */
void or_set_threads(int n);

/* Individual phases of one step for unit checks of single kernels. */
void or_primitive(or_case *c);
void or_primitiveplusbc(or_case *c);
void or_derivative(or_case *c);
void or_venkat(or_case *c);
void or_smooth(or_case *c);
void or_viscous(or_case *c);
void or_flux(or_case *c);
void or_set_dt(or_case *c, double dt);

/* Overset fringe tables (rules in hydra_oracle.c); output arrays hold neles
 * entries (fringe), 4*neles (donor, weight) and neles (iblank_out). */
int or_overset_build(int32_t nodes, int32_t neles, int32_t nghosts, const double *x, const double *y,
                     const double *z, const int32_t *elem, const int32_t *ghost, const int32_t *block,
                     int32_t layers, int32_t outer_type, int32_t *iblank_out, int32_t *nfringe,
                     int32_t *fringe, int32_t *donor, double *weight, int32_t *nfallback);
void or_set_overset(or_case *c, int32_t nfringe, const int32_t *fringe, const int32_t *donor,
                    const double *weight);
/* Hole cut of an overset mesh (rule in hydra_oracle.c): iblank_out[neles]
 * is 0 on background field cells within `margin` of, or enclosed by, the
 * wall surface of the component block; -1 if there is no wall face. */
int or_overset_hole_cut(int32_t nodes, int32_t neles, int32_t nghosts, const double *x, const double *y,
                        const double *z, const int32_t *elem, const int32_t *ghost, const int32_t *block,
                        int32_t wall_type, double margin, int32_t *iblank_out, int32_t *nholes);

#ifdef __cplusplus
}
#endif
#endif
