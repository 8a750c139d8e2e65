// arc_step_warps64.cu - the warp-per-leg step in FP64: the reference's own
// precision (csrc/arc_math.h:3-4), for callers that need its results to
// within FMA contraction rather than to FP32 rounding.
//
// The same group step as the FP32 kernel (arc_step_warps.cuh, compiled here
// with F = double): a CTA of four warps steps 32 worlds, warp k running leg
// k of each. Its bodies, anchors and contact records take twice the shared
// memory of the FP32 step (109 KB per CTA), so two CTAs share an SM, and
// each thread may use up to 255 registers. The whole control step runs in
// one launch (no substep tiles).
#define ARC_WARPS_FP64
#include "arc_step_warps.cuh"

namespace arc {

namespace {

struct Smem64 {
    wl::Smem step;
    int next;  // the next group from the work queue
};

__global__ void __launch_bounds__(wl::kThreads, 2)
k_step_warps64(const __grid_constant__ DevModel<double> M, Worlds<double> W, Actuation A, double* __restrict__ spill,
               int spill_per_lane, int lane_cap, const int* __restrict__ ids, int n_items, int* queue)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem64& sm = *reinterpret_cast<Smem64*>(smem_raw);
    const int tid = threadIdx.x, leg = tid / wl::kWorlds, j = tid % wl::kWorlds;
    const int n_groups = (n_items + wl::kWorlds - 1) / wl::kWorlds;
    // with a queue every group, the first included, is taken from it
    int first = blockIdx.x;
    if (queue) {
        if (tid == 0)
            sm.next = atomicAdd(queue, 1);
        __syncthreads();
        first = sm.next;
    }
#pragma unroll 1
    for (int group = first; group < n_groups;) {
        wl::step_group(sm.step, M, W, A, spill, spill_per_lane, lane_cap, ids, n_items, group, tid, leg, j, 0,
                       M.substeps, nullptr);
        if (!queue)
            break;
        __syncthreads();
        if (tid == 0)
            sm.next = atomicAdd(queue, 1);
        __syncthreads();
        group = sm.next;
    }
    if (queue) {
        // the last CTA to leave zeroes the queue for the next launch
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            if (atomicAdd(queue + 1, 1) == (int)gridDim.x - 1) {
                queue[0] = 0;
                queue[1] = 0;
                __threadfence();
            }
        }
    }
}

}  // namespace

cudaError_t launch_step_warps64(const DevModel<double>& M, const Worlds<double>& W, const Actuation& A,
                                double* spill, int spill_per_lane, int lane_cap, const int* ids, int n_items,
                                int* queue, cudaStream_t stream)
{
    if (W.n <= 0 || n_items <= 0)
        return cudaSuccess;
    if (!M.leaper)
        return cudaErrorInvalidValue;
    const int smem = (int)sizeof(Smem64);
    // per device: the shared-memory attribute, and how many CTAs are resident
    // at once (the work queue's wave)
    static std::atomic<unsigned long long> configured{0};
    static int resident[64] = {};
    cudaError_t e = once_per_device(configured, [&](int dev) {
        cudaError_t r = cudaFuncSetAttribute(k_step_warps64, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int sms = 0, per_sm = 0;
        if (r == cudaSuccess)
            r = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (r == cudaSuccess)
            r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_warps64, wl::kThreads, smem);
        if (r == cudaSuccess)
            resident[dev] = sms * (per_sm > 0 ? per_sm : 1);
        return r;
    });
    if (e != cudaSuccess)
        return e;
    const int groups = (n_items + wl::kWorlds - 1) / wl::kWorlds;
    int grid = groups;
    if (queue) {
        int dev = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess)
            return e;
        grid = groups < resident[dev] ? groups : resident[dev];  // one wave of resident CTAs
    }
    k_step_warps64<<<grid, wl::kThreads, smem, stream>>>(M, W, A, spill, spill_per_lane, lane_cap, ids, n_items,
                                                         queue);
    return cudaGetLastError();
}

}  // namespace arc
