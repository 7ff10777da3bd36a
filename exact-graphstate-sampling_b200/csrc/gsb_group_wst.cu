// Instantiations of the warp-specialised complex64 FP32 fused sampling passes: written steps and the next step's
// branch norms (tiles of 2^9 classes or more, gsb_group.cuh).
#include "gsb_group.cuh"
#include "gsb_pick.h"

namespace gsb {

void *pick_group_ws_trailing(int d) {
    return d == 2 ? (void *)k_group<float2, float, 2, 1, 2, true> : (void *)k_group<float2, float, 1, 1, 2, true>;
}

}  // namespace gsb
