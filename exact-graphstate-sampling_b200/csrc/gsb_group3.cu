// Instantiations of the complex64 FP32 fused passes with three CTAs per SM (autotuner candidates, gsb_group.cuh).
#include "gsb_group.cuh"
#include "gsb_pick.h"

namespace gsb {

void *pick_group3(int d, int tr) {
    if (tr) return d == 2 ? (void *)k_group<float2, float, 2, 1, 3> : (void *)k_group<float2, float, 1, 1, 3>;
    return d == 3 ? (void *)k_group<float2, float, 3, 0, 3> : (void *)k_group<float2, float, 2, 0, 3>;
}

}  // namespace gsb
