// Precision variant "mixed": flux/gradient arithmetic in float.
#define HP_NS v_mixed
#define HP_R float
// geometry-only least-squares terms: recomputed in FP32
#define HP_LSQ_TABLE 0
// division form and blocks per SM of the 4-lane kernels (measured per variant)
#ifndef HP_DIV_FAST
#define HP_DIV_FAST 0
#endif
#ifndef HP_GRAD4_MINB
#define HP_GRAD4_MINB 6
#endif
#ifndef HP_FLUX4_MINB
#define HP_FLUX4_MINB 5
#endif
#ifndef HP_VISC4_MINB
#define HP_VISC4_MINB 4
#endif
#include "hp_kernels.cuh"

namespace hp {
const Variant variant_mixed = {"mixed", sizeof(float), &v_mixed::enqueue_start, &v_mixed::enqueue_step, (HP_FACE_VISC && sizeof(HP_R) != sizeof(double)) ? 1 : 0,
    &v_mixed::fused_grid, &v_mixed::enqueue_fused};
}
