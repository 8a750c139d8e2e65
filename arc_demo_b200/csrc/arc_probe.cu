// arc_probe.cu - FP32 FMA throughput probe: the roofline denominator of the
// step kernels, which are bound by FP32 CUDA-core issue (no tensor cores:
// nothing in the XPBD step is a dense contraction).
#include <cuda_runtime.h>
#include "../../include/arc_sim.h"

namespace {

// 8 independent FMA chains per thread, each 2 FLOP per iteration
__global__ void __launch_bounds__(256) k_fma(float* out, int iters, float a, float b)
{
    float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
        x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
    if (x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7 == 1234.5f)
        out[threadIdx.x] = x0;
}

}  // namespace

extern "C" int arc_probe_fp32_peak(double* flops_per_s, double* seconds)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        return ARC_ERR_CUDA;
    float* out = nullptr;
    if (cudaMalloc(&out, 256 * sizeof(float)) != cudaSuccess)
        return ARC_ERR_CUDA;
    const int blocks = sms * 8, threads = 256, iters = 1 << 16;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);  // warm-up
    cudaEventRecord(e0);
    for (int r = 0; r < 5; ++r)
        k_fma<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess)
        return ARC_ERR_CUDA;
    const double flop = 5.0 * blocks * threads * (double)iters * 8 * 2;
    if (flops_per_s)
        *flops_per_s = flop / (ms * 1e-3);
    if (seconds)
        *seconds = ms * 1e-3;
    return ARC_OK;
}
