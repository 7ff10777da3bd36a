// The complex64 FP32 fused-pass kernels (k_group<float2, float, ...>) are instantiated in translation units of their
// own, so the library's objects compile in parallel; these return their addresses for cudaLaunchKernel.
#pragma once

namespace gsb {

void *pick_group_f32(int d, int tr);   // two CTAs per SM, one barrier per tile (gsb_group_f32.cu)
void *pick_group_ws(int d, int tr);    // warp-specialised, tiles of 2^9 classes or more (gsb_group_ws.cu)
void *pick_group_ws_trailing(int d);  // the same with a trailing step, tr = 1 (gsb_group_wst.cu)
void *pick_group3(int d, int tr);      // three CTAs per SM (gsb_group3.cu)

}  // namespace gsb
