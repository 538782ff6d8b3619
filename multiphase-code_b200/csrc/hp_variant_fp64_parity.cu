// Precision variant "fp64_parity": flux/gradient arithmetic in double.
#define HP_NS v_fp64_parity
#define HP_R double
// geometry-only least-squares terms: loaded from the set-up tables
#define HP_LSQ_TABLE 1
#include "hp_kernels.cuh"

namespace hp {
const Variant variant_fp64_parity = {"fp64_parity", sizeof(double), &v_fp64_parity::enqueue_start, &v_fp64_parity::enqueue_step, 0};
}
