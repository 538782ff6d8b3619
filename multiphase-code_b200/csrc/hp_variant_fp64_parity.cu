// Precision variant "fp64_parity": flux/gradient arithmetic in double.
#define HP_NS v_fp64_parity
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
// the fused step kernel (one cooperative launch per step)
#define HP_FUSED_STEP 1
#include "hp_kernels.cuh"

namespace hp {
const Variant variant_fp64_parity = {"fp64_parity", sizeof(double), &v_fp64_parity::enqueue_start, &v_fp64_parity::enqueue_step, (HP_FACE_VISC && sizeof(HP_R) != sizeof(double)) ? 1 : 0,
    &v_fp64_parity::fused_grid, &v_fp64_parity::enqueue_fused};
}
