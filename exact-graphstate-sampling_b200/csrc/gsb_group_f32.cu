// Instantiations of the complex64 FP32 fused passes, two CTAs per SM, one barrier per tile (gsb_group.cuh).
#include "gsb_group.cuh"
#include "gsb_pick.h"

namespace gsb {

void *pick_group_f32(int d, int tr) {
    if (tr) return d == 2 ? (void *)k_group<float2, float, 2, 1> : (void *)k_group<float2, float, 1, 1>;
    return d == 3 ? (void *)k_group<float2, float, 3, 0> : (void *)k_group<float2, float, 2, 0>;
}

}  // namespace gsb
