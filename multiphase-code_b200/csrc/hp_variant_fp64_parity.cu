// Precision variant "fp64_parity": flux/gradient arithmetic in double.
#define HP_NS v_fp64_parity
#define HP_R double
#include "hp_kernels.cuh"

namespace hp {
const Variant variant_fp64_parity = {"fp64_parity", sizeof(double), &v_fp64_parity::enqueue_start, &v_fp64_parity::enqueue_step, 0};
}
