// Precision variant "fp32": every kernel computes in float, the state path
// included (EOS recovery, RK update, JST, dt); the state is kept as
// float-rounded values.  The precision-stress reference point: it shows what
// the steps the mixed variant keeps in FP64 would lose.
#define HP_NS v_fp32
#define HP_R float
#define HP_S float
// geometry-only least-squares terms: recomputed in FP32
#define HP_LSQ_TABLE 0
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
const Variant variant_fp32 = {"fp32", sizeof(float), &v_fp32::enqueue_start, &v_fp32::enqueue_step, (HP_FACE_VISC && sizeof(HP_R) != sizeof(double)) ? 1 : 0,
    &v_fp32::fused_grid, &v_fp32::enqueue_fused};
}
