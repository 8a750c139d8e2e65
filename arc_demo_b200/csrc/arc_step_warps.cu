// arc_step_warps.cu - the warp-per-leg step kernel (FP32): CTAs of four
// warps step groups of 32 worlds (arc_step_warps.cuh), one group each or, with
// a work queue, as many as the queue hands them.
#include "arc_step_warps.cuh"

namespace arc {
namespace wl {
namespace {

// Work items are worlds (ids[item], or item itself without ids), 32 to a
// group; CTA b steps group b. With a queue (two ints, zero before the
// launch), CTAs take groups from it until none is left, and the last CTA to
// leave zeroes the queue again for the next launch.
__global__ void __launch_bounds__(kThreads, 4)
k_step_warps(const __grid_constant__ DevModel<F> M, Worlds<F> W, Actuation A, F* __restrict__ spill, int spill_per_lane,
             int lane_cap, const int* __restrict__ ids, int n_items, int* queue, int sub0, int sub1,
             F* __restrict__ tile_q)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
    __shared__ int s_next;
    const int tid = threadIdx.x, leg = tid / kWorlds, j = tid % kWorlds;
    const int n_groups = (n_items + kWorlds - 1) / kWorlds;
    // with a queue every group, the first included, is taken from it: a CTA
    // that becomes resident only when others leave finds the queue empty
    // instead of holding back a group of its own
    int first = blockIdx.x;
    if (queue) {
        if (tid == 0)
            s_next = atomicAdd(queue, 1);
        __syncthreads();
        first = s_next;
    }
#pragma unroll 1
    for (int group = first; group < n_groups;) {
        step_group(sm, M, W, A, spill, spill_per_lane, lane_cap, ids, n_items, group, tid, leg, j, sub0, sub1, tile_q);
        if (!queue)
            break;
        if (tid == 0)
            s_next = atomicAdd(queue, 1);
        __syncthreads();
        group = s_next;
    }
    if (queue) {
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
}  // namespace wl

size_t warps_smem_bytes() { return sizeof(wl::Smem); }

cudaError_t launch_step_warps(const DevModel<float>& M, const Worlds<float>& W, const Actuation& A, float* spill,
                              int spill_per_lane, int lane_cap, const int* ids, int n_items, int* queue,
                              cudaStream_t stream, int tile, float* tile_q)
{
    if (W.n <= 0 || n_items <= 0)
        return cudaSuccess;
    if (!M.leaper)
        return cudaErrorInvalidValue;
    const int smem = (int)sizeof(wl::Smem);
    // per device: the shared-memory attribute, and how many CTAs are resident
    // at once (the work queue's wave)
    static std::atomic<unsigned long long> configured{0};
    static int resident[64] = {};
    cudaError_t e = once_per_device(configured, [&](int dev) {
        cudaError_t r = cudaFuncSetAttribute(wl::k_step_warps, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             smem > 48 * 1024 ? smem : 48 * 1024);
        int sms = 0, per_sm = 0;
        if (r == cudaSuccess)
            r = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (r == cudaSuccess)
            r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wl::k_step_warps, wl::kThreads, smem);
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
    if (tile <= 0 || tile >= M.substeps || !tile_q)
        tile = M.substeps;
    for (int sub0 = 0; sub0 < M.substeps; sub0 += tile) {
        const int sub1 = sub0 + tile < M.substeps ? sub0 + tile : M.substeps;
        wl::k_step_warps<<<grid, wl::kThreads, smem, stream>>>(M, W, A, spill, spill_per_lane, lane_cap, ids, n_items,
                                                               queue, sub0, sub1, tile_q);
        if ((e = cudaGetLastError()) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

}  // namespace arc
