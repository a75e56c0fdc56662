// FP64 fused multiply-add throughput of the device, measured by the library
// itself: the denominator of the FP64 compute roof the flux pass is held
// against (the pass is bound by FP64 issue, not by HBM).
//
// Every thread runs CHAINS independent FMA chains x <- x*a + b for `iters`
// rounds of UNROLL steps; enough resident warps keep the FP64 pipe full.
// One FMA counts as two flops.
#include <cuda_runtime.h>

#include "mfcfd_b200.h"

namespace {

constexpr int CHAINS = 8;
constexpr int UNROLL = 16;
constexpr int PEAK_BLOCK = 256;

__global__ void __launch_bounds__(PEAK_BLOCK) k_fp64_fma(double *out, int iters, double a, double b) {
    double x[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) x[c] = 1e-3 * (threadIdx.x + c);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
#pragma unroll
            for (int c = 0; c < CHAINS; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps every chain live
}

}  // namespace

extern "C" int mfcfd_measure_fp64_peak(double *tflops) {
    if (!tflops) return MFCFD_ERR_ARG;
    *tflops = 0.0;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MFCFD_ERR_NODEV;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return MFCFD_ERR_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fp64_fma, PEAK_BLOCK, 0) !=
        cudaSuccess)
        return MFCFD_ERR_CUDA;
    const int grid = sms * (per_sm > 0 ? per_sm : 1);
    const int iters = 4096;
    double *out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = MFCFD_OK;
    float best = 0.f;
    if (cudaMalloc(&out, sizeof(double) * (size_t)grid * PEAK_BLOCK) != cudaSuccess)
        return MFCFD_ERR_OOM;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        st = MFCFD_ERR_CUDA;
        goto done;
    }
    // one warm-up launch, then the best of five timed launches
    for (int rep = 0; rep < 6; ++rep) {
        cudaEventRecord(e0, 0);
        k_fp64_fma<<<grid, PEAK_BLOCK>>>(out, iters, 0.9999999, 1e-7);
        cudaEventRecord(e1, 0);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            st = MFCFD_ERR_CUDA;
            goto done;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && (best == 0.f || ms < best)) best = ms;
    }
    {
        const double flops = 2.0 * CHAINS * UNROLL * (double)iters * grid * PEAK_BLOCK;
        *tflops = flops / (best * 1e-3) / 1e12;
    }
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(out);
    return st;
}
