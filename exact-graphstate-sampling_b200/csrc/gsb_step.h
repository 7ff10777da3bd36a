// Step descriptor shared by the translation units that run DP steps on the device (executor, adjoint sweep).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gsb {

struct StepArgs {
    uint64_t tk[40];        // Tkeep (entries >= nk are 0)
    uint64_t tq[4];         // distinct coset offsets, ascending
    uint64_t g, rhoc;
    double Mr[2][2], Mi[2][2];
    double Mr32[2][2], Mi32[2][2];   // the same rounded to float values for the FP32 kernels (the engine's apply_coeffs)
    int nk, k, ntq, m;
    int tau0[4], tau1[4], par[4];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace gsb
