// Precision variant "fp64": flux/gradient arithmetic in double.
#define HP_NS v_fp64
#define HP_R double
// geometry-only least-squares terms: loaded from the set-up tables
#define HP_LSQ_TABLE 1
#include "hp_kernels.cuh"

namespace hp {
const Variant variant_fp64 = {"fp64", sizeof(double), &v_fp64::enqueue_start, &v_fp64::enqueue_step, 0};
}
