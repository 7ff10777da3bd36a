// Instantiations of the warp-specialised complex64 FP32 fused chain passes (tiles of 2^9 classes or more,
// gsb_group.cuh); the sampling ones (a trailing step) are in gsb_group_wst.cu.
#include "gsb_group.cuh"
#include "gsb_pick.h"

namespace gsb {

void *pick_group_ws(int d, int tr) {
    if (tr) return pick_group_ws_trailing(d);
    return d == 3 ? (void *)k_group<float2, float, 3, 0, 2, true> : (void *)k_group<float2, float, 2, 0, 2, true>;
}

}  // namespace gsb
