// Precision variant "fp64": flux/gradient arithmetic in double.
#define HP_NS v_fp64
#define HP_R double
// geometry-only least-squares terms: loaded from the set-up tables
#define HP_LSQ_TABLE 1
// division form and blocks per SM of the 4-lane kernels (measured per variant)
#ifndef HP_DIV_FAST
#define HP_DIV_FAST 1
#endif
// fast division in gradients, fluxes and JST; the viscous kernel spills with
// its second (fallback) body and is faster with hardware division
#ifndef HP_FAST_MASK
#define HP_FAST_MASK 11
#endif
// the four-lane gradient kernel stages its cell geometry, its fields' values
// at the cell and its neighbours and the limiter's inputs in shared memory
// (asynchronous copies issued when it starts); the flux kernel prefetches
// what its sources and RK update read the same way
#ifndef HP_GRAD4_STAGE
#define HP_GRAD4_STAGE 1
#endif
#ifndef HP_FLUX4_PREFETCH
#define HP_FLUX4_PREFETCH 1
#endif
#ifndef HP_GRAD4_MINB
#define HP_GRAD4_MINB 5
#endif
#ifndef HP_FLUX4_MINB
#define HP_FLUX4_MINB 4
#endif
#ifndef HP_VISC4_MINB
#define HP_VISC4_MINB 3
#endif
#include "hp_kernels.cuh"

namespace hp {
const Variant variant_fp64 = {"fp64", sizeof(double), &v_fp64::enqueue_start, &v_fp64::enqueue_step, (HP_FACE_VISC && sizeof(HP_R) != sizeof(double)) ? 1 : 0,
    &v_fp64::fused_grid, &v_fp64::enqueue_fused};

// The FP64 (FMA) kernels over the wall-layer cell lists, for the steps of the
// FP32-arithmetic variants (same compile flags as theirs: -fmad=true).
namespace v_fp64 {
static void wall_visc(const DevMesh& m, const DevState<double>& s, const DevParams& P, cudaStream_t st) {
    if (m.nwall > 0) k_visc8<1><<<grid_for(8ll * m.nwall, 128), 128, 0, st>>>(m, s, P);
}
// With the layer-first cell order (m.wprefix) the lists are the leading
// cells, and the gradient and flux kernels run their whole-mesh form over a
// view of the mesh that ends after them: the same per-cell arithmetic, with
// the coalesced staging of the whole-mesh launches.  (The viscous kernel
// tells boundary faces by m.neles, so it keeps the list.)
static DevMesh prefix_view(const DevMesh& m, int n) {
    DevMesh v = m;
    v.neles = n;
    return v;
}
static void wall_grad(const DevMesh& m, const DevState<double>& s, const DevParams& P, cudaStream_t st) {
    if (m.ngwall <= 0) return;
    if (m.wprefix) k_grad4<0><<<grid_for(4ll * m.ngwall, 128), 128, 0, st>>>(prefix_view(m, m.ngwall), s, P);
    else k_grad4<1><<<grid_for(4ll * m.ngwall, 128), 128, 0, st>>>(m, s, P);
}
template <int Z>
static void wall_flux_z(const DevMesh& m, const DevState<double>& s, const DevParams& P, cudaStream_t st,
                        int stage) {
    const unsigned g = grid_for(4ll * m.nwall, 128);
    if (m.wprefix) k_flux4<Z, 0><<<g, 128, 0, st>>>(prefix_view(m, m.nwall), s, P, stage);
    else k_flux4<Z, 1><<<g, 128, 0, st>>>(m, s, P, stage);
}
static void wall_flux(const DevMesh& m, const DevState<double>& s, const DevParams& P, cudaStream_t st,
                      int stage) {
    if (m.nwall <= 0) return;
    if (P.myflux == 1) wall_flux_z<1>(m, s, P, st, stage);
    else if (P.myflux == 3) wall_flux_z<2>(m, s, P, st, stage);
    else wall_flux_z<0>(m, s, P, st, stage);
}
}  // namespace v_fp64
const WallFp64 wall_fp64 = {&v_fp64::wall_visc, &v_fp64::wall_grad, &v_fp64::wall_flux};
}
