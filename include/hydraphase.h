/*
 * hydraphase.h -- C ABI of the B200 residual-and-update engine for the
 * two-phase six-equation solver (reference: GauthamBijoy23/Multiphase-code,
 * project HydraPhase_60_FPC_5mill, Fortran 90 + OpenACC).
 *
 * The reference has no library API: its time loop (src/main.F90:511-657)
 * calls argument-less subroutines that share module globals
 * (src/mod_GlobalVariables.F90).  This header replaces that loop.  A Fortran
 * host keeps its own Read_flow, mesh reader and restart/Tecplot writers and
 * calls these entry points through ISO_C_BINDING interfaces (one bind(C)
 * interface per function below); plain pointers and sizes only, 1-based cell ids as the
 * reference stores them, column-major conserved state.
 *
 * Conventions: every entry point returns 0 on success and a negative
 * HP_E_* code on failure (never exits or stops); hp_last_error() gives the
 * message.  One host thread per handle; each handle owns one CUDA stream and
 * all of its device memory.
 */
#ifndef HYDRAPHASE_H
#define HYDRAPHASE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    HP_OK = 0,
    HP_E_ARG = -1,        /* bad argument / malformed mesh or parameters */
    HP_E_CUDA = -2,       /* CUDA runtime failure */
    HP_E_NOMEM = -3,      /* device allocation failed or over the HBM budget */
    HP_E_IO = -4,         /* file could not be opened / parsed */
    HP_E_STATE = -5,      /* call out of order (e.g. step before set_state) */
    HP_E_UNSUPPORTED = -6 /* feature outside this build (proc_bc partition ghosts) */
};

/* Arithmetic of the hot kernels. */
enum {
    HP_PREC_FP64_PARITY = 0, /* FP64, no FMA contraction: bit-parity path */
    HP_PREC_FP64 = 1,        /* FP64 with FMA */
    HP_PREC_MIXED = 2,       /* FP32 gradients/limiter/fluxes, FP64 state,
                                EOS recovery and reductions */
    HP_PREC_FP32 = 3         /* everything FP32, state path included: the
                                precision-stress reference (ghost fill and
                                diagnostics stay FP64) */
};

/* flow.in in file order (src/sr_Read_flow.F90:19-268) plus the switches of
 * this build.  Field meanings and units are those of flow.in. */
typedef struct hp_params {
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
    int32_t myflux;          /* 1 = HLLC-Zien, 2 = HLLC-Batten, 3 = Jameson central flux */
    int32_t myorder;         /* 1 or 2 */
    double as, ts;           /* Sutherland constants */
    /* --- additions; zero-initialised values reproduce the reference --- */
    int32_t face_mode;       /* FP32-arithmetic variants: 0 = fluxes evaluated
                                once per face where the mesh allows, stored as
                                face records and gathered per cell in face
                                order; 1 = once from each side (four lanes per
                                cell); 2 = once per face, added to per-cell sums
                                colour by colour (no atomics, fixed order);
                                3 = once per face with atomic adds (the last
                                bits vary from run to run); hydraphase.tune
                                picks it */
    double venkat_k;         /* limiter eps^2 = (K*dl)^3; 0 selects 0.3 */
    int32_t rk_scheme;       /* 0: reference 4-stage ESSPRK; 1: SSP-RK3 */
    int32_t inviscid;        /* 1: viscous face fluxes off */
    double twall;            /* isothermal wall temperature (BC type 6) */
    int32_t precision;       /* HP_PREC_* */
    int32_t renumber;        /* 1: space-filling-curve cell order on device */
    int32_t block_size;      /* threads per block of the one-thread-per-cell
                                kernels: 0 (= 256) or a multiple of 32 in
                                [64, 512]; hydraphase.tune picks it */
    int32_t use_graph;       /* 1: capture each step in a CUDA graph; 2: one
                                fused cooperative kernel per step (precision
                                HP_PREC_FP64_PARITY on plain meshes: not aliased,
                                two-phase, no overset fringe or partition halo;
                                every other handle runs as with 1); 0: launch
                                each kernel */
    double pad_[4];
    /* --- five-phase model (the reference's FIVE_PHASE build): three
     * dispersed, incompressible phases q, r, s with mass and momentum each,
     * so 22 conserved variables (src/main.F90:114-124); flow.in groups
     * 19-21 (src/sr_Read_flow.F90:214-250), read when present --------- */
    int32_t five_phase;      /* 1: 22 conserved variables (cu(1:22)) */
    double rhoq, rhor, rhos; /* dispersed-phase densities */
    double radq, radr, rads; /* particle radii */
    double phiginit, phipinit, phiqinit, phirinit, phisinit;  /* start fractions */
    /* FP32-arithmetic precisions (mixed, fp32): the cells within this many
     * layers of a wall ghost (types 5 and 6) take their viscous terms,
     * fluxes, sources and RK update from the FP64 kernels (0: none).  Not
     * with aliased ghost ids.  The FP64 precisions ignore it. */
    int32_t wall_fp64_layers;
} hp_params;

/* Mesh as the reference reads it (src/sr_geometry.F90:101-139):
 *   x, y, z[nodes]                   node coordinates
 *   elem[neles*9] row-major          nod1..nod4, nc1..nc4, iblank (1-based)
 *   ghost[nghosts*4] row-major       nparent, nghost, ntype, nside
 * Partition ghosts (proc_bc) must be zero: a part of a partitioned mesh is an
 * ordinary mesh whose halo cells are elements (see hp_set_halo). */
typedef struct hp_mesh {
    int32_t nodes, neles, nghosts, pghosts;
    const double *x, *y, *z;
    const int32_t *elem;
    const int32_t *ghost;
} hp_mesh;

/* Per-step diagnostics (src/main.F90:646-654). */
typedef struct hp_diag {
    double time;      /* simulation time after the step */
    double dt;        /* time step used */
    double velmag;    /* |u_g| of cell 1 (Velocity.dat) */
    double diff[4];   /* max |cn - cu| of variables 1..4 (diffp,diffu,diffv,diffw) */
    double nan_cells; /* elements whose state is NaN after the step */
} hp_diag;

typedef struct hp_handle hp_handle;

/* --- lifecycle --------------------------------------------------------- */
/* Replaces the setup half of src/main.F90:47-499: computes the geometry of
 * src/sr_geometry.F90:147-347 (bit-identical to the reference), builds the
 * device layout, and allocates all device memory on the current device. */
int hp_create(const hp_mesh *mesh, const hp_params *params, hp_handle **out);
/* A batch: ncase meshes (same parameters) in one handle.  No counterpart in
 * the reference.  Their cell and ghost lists are concatenated on the device,
 * so every kernel of a step sweeps all cases in one launch; each case keeps
 * its own dt, time, residuals and diagnostics, and its results are those
 * it would have alone.  Meshes whose ghost ids alias element ids
 * (HP_E_UNSUPPORTED) and partition ghosts cannot be batched.  hp_create is
 * hp_create_batch with ncase = 1. */
int hp_create_batch(const hp_mesh *meshes, int32_t ncase, const hp_params *params, hp_handle **out);
int hp_case_count(const hp_handle *h, int32_t *ncase);
int hp_destroy(hp_handle *h);
const char *hp_last_error(const hp_handle *h);
/* Message of the last failed hp_create (no handle exists then). */
const char *hp_create_error(void);

/* src/sr_init_cond.F90:177-226 (uniform state) and cn = cu. */
int hp_init_uniform(hp_handle *h);
/* Restart injection, src/main.F90:427-441: cu_elem is cu(1:neles,1:10)
 * column-major; ghost_prims (may be NULL) is ug,vg,wg,pg,tg,rog at the ghost
 * ids in ghost-list order (6 x nghosts).  Host pointers. */
int hp_set_state(hp_handle *h, double time, const double *cu_elem,
                 const double *ghost_prims);
/* The same for case c of a batch (hp_set_state is case 0).  Every case of a
 * batch is set before its first step (HP_E_STATE afterwards). */
int hp_set_state_case(hp_handle *h, int32_t c, double time, const double *cu_elem,
                      const double *ghost_prims);

/* nsteps of src/main.F90:515-654 for every case of the handle.  diag may be
 * NULL or hold ncase * nsteps entries (case c's steps at c * nsteps).
 * Asynchronous with respect to the host unless diag != NULL. */
int hp_step(hp_handle *h, int32_t nsteps, hp_diag *diag);
/* Blocks until the handle's stream is idle. */
int hp_sync(hp_handle *h);
/* nsteps without diagnostics; *device_ms is the device time of those steps
 * measured with CUDA events on the handle's stream. */
int hp_step_timed(hp_handle *h, int32_t nsteps, double *device_ms);
/* nsteps launched eagerly with a CUDA event between every two kernels;
 * accumulates device time and launch counts per kernel kind (nkinds >= 16:
 * prim_start, step_begin, smooth1, smooth2, bc_visc, visc, prim_stage, bc,
 * grad, flux, prim_end, step_end, serial, overset, halo, qrs). */
int hp_profile_steps(hp_handle *h, int32_t nsteps, double *ms_per_kind,
                     int64_t *launches_per_kind, int32_t nkinds);

/* State read-back in the restart layout (src/main.F90:817-824). */
int hp_get_state(hp_handle *h, double *time, double *cu_elem,
                 double *ghost_prims);
int hp_get_state_case(hp_handle *h, int32_t c, double *time, double *cu_elem,
                      double *ghost_prims);
/* Cell primitives after the last step (ug,vg,wg,tg,pg,pp,phig,phip,up,vp,wp,
 * tp,rog,rop; 14 x neles, reference cell order) of case 0. */
int hp_get_prims(hp_handle *h, double *prims);

/* --- device-resident access (for callers that keep data in HBM) --------- */
/* Device pointer of the conserved state cu (10 x ld, internal cell order)
 * and the leading dimension; valid until hp_destroy. */
int hp_device_state(hp_handle *h, double **cu_dev, int64_t *ld);
/* Number of kernels one step launches and the device bytes the handle
 * holds. */
int hp_info(const hp_handle *h, int64_t *kernels_per_step, int64_t *device_bytes,
            int64_t *aliased);

/* --- overset meshes -------------------------------------------------------- */
/* New work: the reference only freezes cells with iblank != 1
 * (src/sr_RK.F90:31); its hole cut and donor search come from TIOGA, outside
 * the solver.  An overset mesh here is one element list of two blocks
 * (block[e] = 0 background, 1 component), with the caller's hole cut as
 * iblank = 0 on background cells.  hp_overset_build marks the fringe
 * (background field cells next to holes, component field cells next to
 * ghosts of type outer_type, `layers` layers deep; iblank_out = -1 there,
 * the input iblank elsewhere) and finds, for each fringe cell, four donor
 * cells of the other block and barycentric weights.  Create the handle with
 * iblank_out in the mesh, then hp_set_overset: after every RK stage each
 * fringe cell's state becomes sum_k weight_k * state(donor_k). */
typedef struct hp_overset {
    int32_t nfringe;
    int32_t *fringe;    /* [nfringe] element ids (1-based), ascending */
    int32_t *donor;     /* [4 * nfringe] element ids (1-based), row-major */
    double *weight;     /* [4 * nfringe] */
    int32_t nfallback;  /* fringe cells inside no donor-block cell (nearest used) */
} hp_overset;
int hp_overset_build(const hp_mesh *mesh, const int32_t *block, int32_t layers, int32_t outer_type,
                     int32_t *iblank_out, hp_overset *out);
/* The same tables, bit for bit, with the donor search, the nearest-centroid
 * fallback and the weights on the current CUDA device (the host marks the
 * fringe and sizes the search grids).  Allocates temporary device memory;
 * HP_E_CUDA if a device call fails. */
int hp_overset_build_gpu(const hp_mesh *mesh, const int32_t *block, int32_t layers, int32_t outer_type,
                         int32_t *iblank_out, hp_overset *out);
/* Hole cut, the step before hp_overset_build (new work: the reference takes
 * it from TIOGA).  The wall surface is the set of faces of component
 * (block 1) elements whose neighbour is a ghost of type wall_type (face k:
 * the element's nodes other than node k).  A background (block 0) cell with
 * iblank 1 becomes a hole, iblank_out = 0, when its centroid lies within
 * `margin` (>= 0) of a wall triangle or is enclosed by the surface (the ray
 * from it towards +x crosses an odd number of wall triangles; edges and
 * vertices counted once); every other cell keeps the mesh's iblank.  The
 * surface must be closed, or open only across planes parallel to the x axis
 * (a body extruded between planes z = const).  *nholes (may be NULL) = cells
 * cut.  HP_E_ARG on bad arguments or when no face has type wall_type.  The
 * _gpu form tests the cells on the current CUDA device (temporary device
 * memory; HP_E_CUDA if a device call fails) and returns the same iblank. */
int hp_overset_hole_cut(const hp_mesh *mesh, const int32_t *block, int32_t wall_type, double margin,
                        int32_t *iblank_out, int32_t *nholes);
int hp_overset_hole_cut_gpu(const hp_mesh *mesh, const int32_t *block, int32_t wall_type, double margin,
                            int32_t *iblank_out, int32_t *nholes);
void hp_free_overset(hp_overset *ov);
/* Single-case handles only; replaces any earlier table. */
int hp_set_overset(hp_handle *h, const hp_overset *ov);

/* --- partitioned meshes ------------------------------------------------------ */
/* The reference runs one partition per MPI rank, with one layer of partition
 * ghosts whose conserved state is exchanged after every RK stage
 * (src/sr_mpiexchangecn.F90:1-96, called from src/sr_RK.F90) and an
 * MPI_Allreduce of the time step (src/main.F90:552).  Here a part is an
 * ordinary mesh: its own cells, then two layers of the neighbouring parts'
 * cells as elements with their nodes (iblank HP_IBLANK_HALO1: gradients and
 * limiter evaluated, no RK update; HP_IBLANK_HALO2: frozen), with the
 * bounding-box nodes of the whole mesh appended.  Every owned cell then sees
 * the inputs it has in the whole mesh, and the parts reproduce the
 * single-mesh run bit for bit.  hydraphase.partition builds the parts. */
enum { HP_IBLANK_HALO1 = 2, HP_IBLANK_HALO2 = 3 };
/* Parts on one device, as the cases of a batch: after every RK stage, halo
 * element dst_elem[t] of case dst_case[t] takes the conserved state of element
 * src_elem[t] of case src_case[t] (1-based elements, 0-based cases; a
 * destination is no source), and every case takes one dt, the minimum over
 * the parts.  n = 0 removes the table.  Set before the first step. */
int hp_set_halo(hp_handle *h, int32_t n, const int32_t *dst_case, const int32_t *dst_elem,
                const int32_t *src_case, const int32_t *src_elem);
/* Parts on several GPUs, one single-case handle per process.  The library
 * calls fn(user, point, stream) on the thread that enqueues the steps, with
 * the handle's cudaStream_t:
 *   HP_X_DT    before each step forms its dt: the part's partial minimum
 *              (*hp_dtmin_ptr: the bit pattern of a positive double, so the
 *              minimum over parts is the unsigned minimum) is complete in
 *              stream order; the callback enqueues its replacement by the
 *              minimum over all parts (an allreduce(MIN) on the stream);
 *   HP_X_HALO  after each RK stage: the callback enqueues hp_halo_pack, the
 *              exchange between parts and hp_halo_unpack on the stream.
 * Steps of a handle with a callback are not captured in CUDA graphs.  fn =
 * NULL removes it. */
enum { HP_X_DT = 0, HP_X_HALO = 1 };
typedef void (*hp_exchange_fn)(void *user, int32_t point, void *stream);
int hp_set_exchange(hp_handle *h, hp_exchange_fn fn, void *user);
/* Cells this part sends (send_elem, its own elements) and receives
 * (recv_elem, its halo elements), 1-based, each list in the order of the
 * exchange buffers. */
int hp_set_halo_lists(hp_handle *h, int32_t nsend, const int32_t *send_elem, int32_t nrecv,
                      const int32_t *recv_elem);
/* Enqueued on the handle's stream: buf[10 * t + k] = cn(send_elem[t], k+1)
 * for the 10 conserved variables, and cn(recv_elem[t], k+1) =
 * buf[10 * t + k] (cell major: one peer's cells are one contiguous block).
 * Device buffers of 10 * nsend and 10 * nrecv doubles. */
int hp_halo_pack(hp_handle *h, double *buf);
int hp_halo_unpack(hp_handle *h, const double *buf);
/* Device address of case 0's partial dt minimum (uint64 bit pattern). */
int hp_dtmin_ptr(hp_handle *h, uint64_t **bits);

/* --- output ------------------------------------------------------------------ */
/* The Tecplot file of src/main.F90:956-1268 (two-phase build): node
 * coordinates, the 13 cell-centred fields (U V W PG PP TG UP VP WP PHIG TP
 * ROG ROP, fields[13][neles], reference element order) and the
 * connectivity; values as Fortran ES16.8.  Host only. */
int hp_write_tecplot(const char *path, const hp_mesh *mesh, const double *fields);
/* Asynchronous output of case c, with no counterpart in the reference (which
 * stops its time loop to write): a snapshot of the state after the steps
 * enqueued so far is taken on the device, copied to pinned memory on a side
 * stream, and written by a host thread to restart_path (the restart format
 * of hp_write_restart; may be NULL) and tecplot_path (hp_write_tecplot's
 * file, fields computed on the device from cu; may be NULL), while later
 * steps run.  For Tecplot, `mesh` is the case's mesh and must stay valid
 * until hp_output_wait returns.  Two requests may be in flight; a third
 * waits for the older one.  hp_output_wait blocks until the request's files
 * are written and returns its status (HP_E_IO on a write failure); a ticket
 * is valid until it is waited for or its slot is reused. */
int hp_output_async(hp_handle *h, int32_t c, const hp_mesh *mesh, const char *restart_path,
                    const char *tecplot_path, int32_t *ticket);
int hp_output_wait(hp_handle *h, int32_t ticket);

/* --- serving many cases ---------------------------------------------------- */
/* No counterpart in the reference, which runs one case per process.  Device
 * bytes hp_create would allocate for this mesh and precision (admission
 * against an HBM budget before creating). */
int hp_estimate_bytes(const hp_mesh *mesh, const hp_params *params, int64_t *bytes);
/* Host threads of the set-up loops (geometry, least-squares tables, cell
 * order) that hp_create runs on the calling thread; 0 = one per core.  A
 * server that sets up several cases at once on worker threads gives each
 * worker a share of the cores, so the workers do not oversubscribe the host
 * (and starve the thread that feeds the GPU). */
int hp_set_host_threads(int32_t n);
int hp_estimate_batch_bytes(const hp_mesh *meshes, int32_t ncase, const hp_params *params,
                            int64_t *bytes);
/* *busy = 1 while steps queued on the handle's stream are still running,
 * 0 once they are done; never blocks.  Lets one host thread drive many
 * handles whose streams overlap on the device. */
int hp_poll(hp_handle *h, int32_t *busy);

/* --- allocation-free time step ------------------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (a Fortran/OpenACC host whose device arrays and memory budget belong
 * to its compiler runtime, or a framework whose pool allocator owns the whole
 * GPU): the time step dt = cfl * min(dl / (max(ag,ap) + max(|ug|,|up|)))
 * of a conserved state, as hp_step computes it at the start of a step
 * (primitive recovery + reduction of src/main.F90:529-556), from buffers the
 * caller owns.  Inputs: cn_dev, 10 columns of leading dimension ld
 * (column-major cn(1:ncells,1:10), any cell order), dl_dev[ncells] (minimum
 * edge length per cell, as src/sr_geometry.F90:210-217 defines it); output:
 * dt_dev[0].  Device pointers; the work is queued on `stream` (a
 * cudaStream_t, NULL for the default stream) and the call returns without
 * waiting.  The call allocates nothing: its only scratch, one partial minimum
 * per 256 cells, is a static device array sized for HP_NOALLOC_MAX_CELLS
 * cells that each GPU using the library keeps until exit; larger ncells is
 * rejected with HP_E_ARG.  All calls share that array, so calls that overlap
 * on the GPU race.  The first call on each device looks up the array's device
 * address; make it before any stream capture.  The lookup is repeated when
 * the device's context changes (after cudaDeviceReset, or a runtime that
 * shuts the device down and opens it again), so the call stays valid across
 * such a reset.  If an earlier CUDA call of the caller left an error pending,
 * the call returns HP_E_CUDA without launching and leaves that error for the
 * caller to read. */
#define HP_NOALLOC_MAX_CELLS (1 << 24)
int hp_dt_noalloc(const double *cn_dev, int64_t ld, const double *dl_dev,
                  int32_t ncells, const hp_params *params, double *dt_dev,
                  void *stream);

/* --- reference file formats (drop-in inputs/outputs) -------------------- */
/* flow.in parser, src/sr_Read_flow.F90:19-268. */
int hp_read_flow(const char *path, hp_params *out);
/* Mesh files of one rank: geometry_files/{grid_procNNNN.dat, bc_procNNNN.in,
 * proc_bcNNNN.in}.  Arrays are malloc'ed; free with hp_free_mesh. */
int hp_read_mesh(const char *case_dir, int32_t rank, hp_mesh *out);
void hp_free_mesh(hp_mesh *m);
/* Restart file, src/main.F90:427-441 / 812-828. */
int hp_read_restart(const char *path, int32_t neles, int32_t nghosts,
                    double *time, double *cu_elem, double *ghost_prims);
int hp_write_restart(const char *path, int32_t neles, int32_t nghosts,
                     double time, const double *cu_elem, const double *ghost_prims);

#ifdef __cplusplus
}
#endif
#endif
