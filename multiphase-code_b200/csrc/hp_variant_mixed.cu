// Precision variant "mixed": flux/gradient arithmetic in float.
#define HP_NS v_mixed
#define HP_R float
// geometry-only least-squares terms: recomputed in FP32
#define HP_LSQ_TABLE 0
#include "hp_kernels.cuh"

namespace hp {
const Variant variant_mixed = {"mixed", sizeof(float), &v_mixed::enqueue_start, &v_mixed::enqueue_step, 0};
}
