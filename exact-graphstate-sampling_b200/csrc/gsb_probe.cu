// L2 copy-bandwidth probe: the denominator of the L2 roofline for work whose tables stay in L2 (the batched launch's
// team tables).  One launch copies an L2-resident buffer onto another `reps` times, so launch overhead does not
// count; loads and stores bypass L1 (ld.global.cg / st.global.cg), so every byte is an L2 transaction.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "gsb.h"
#include "gsb_common.h"

namespace {

__global__ void __launch_bounds__(512) k_l2_copy(const float4 *__restrict__ src, float4 *__restrict__ dst, size_t n,
                                                 int reps) {
    // four independent 16-byte loads in flight per thread, so the probe is not bound by L2 latency itself
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int r = 0; r < reps; r++) {
        size_t i = t0;
        for (; i + 3 * stride < n; i += 4 * stride) {
            const float4 a = __ldcg(src + i), b = __ldcg(src + i + stride), c = __ldcg(src + i + 2 * stride),
                         d = __ldcg(src + i + 3 * stride);
            __stcg(dst + i, a);
            __stcg(dst + i + stride, b);
            __stcg(dst + i + 2 * stride, c);
            __stcg(dst + i + 3 * stride, d);
        }
        for (; i < n; i += stride) __stcg(dst + i, __ldcg(src + i));
    }
}

int probe_fail(int code, const std::string &m) { return gsb::fail(code, m); }

}  // namespace

extern "C" int gsb_probe_l2_copy(int device, uint64_t bytes, int reps, float *gbs) {
    if (!gbs) return probe_fail(GSB_E_USAGE, "null argument");
    if (bytes < (1u << 20) || bytes > (64ull << 20) || bytes % 16 || reps < 1 || reps > 100000)
        return probe_fail(GSB_E_USAGE, "bytes must be a multiple of 16 in [1 MiB, 64 MiB], reps in [1, 100000]");
    int ndev = 0, prev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return probe_fail(GSB_E_CUDA, "no such CUDA device");
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    float4 *src = nullptr, *dst = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = 0;
    float ms = 0;
    const size_t n = (size_t)(bytes / 16);
    if (cudaMalloc(&src, bytes) != cudaSuccess || cudaMalloc(&dst, bytes) != cudaSuccess) {
        rc = probe_fail(GSB_E_ALLOC, "probe buffers");
    } else if (cudaMemset(src, 0, bytes) != cudaSuccess || cudaMemset(dst, 0, bytes) != cudaSuccess ||
               cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = probe_fail(GSB_E_CUDA, "probe set-up");
    } else {
        const int grid = 2 * (sms > 0 ? sms : 148);
        k_l2_copy<<<grid, 512>>>(src, dst, n, 2);   // warm-up: both buffers into L2
        cudaEventRecord(e0);
        k_l2_copy<<<grid, 512>>>(src, dst, n, reps);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0)
            rc = probe_fail(GSB_E_CUDA, std::string("probe launch: ") + cudaGetErrorString(cudaGetLastError()));
        else
            *gbs = (float)(2.0 * (double)bytes * reps / (ms * 1e-3) / 1e9);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(src);
    cudaFree(dst);
    cudaSetDevice(prev);
    return rc;
}
