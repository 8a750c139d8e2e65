// arc_kernels.cuh - launchers of every kernel of the library.
#pragma once

#include <atomic>

#include <cuda_runtime.h>
#include "arc_device.cuh"

namespace arc {

// Kernel attributes belong to a device: a launcher's `setup(dev)` runs once
// for each device it is used on (two first calls racing may both run it,
// which is harmless: it only sets attributes and reads properties).
template <class Setup> cudaError_t once_per_device(std::atomic<unsigned long long>& done, Setup&& setup)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (dev < 0 || dev >= 64)
        return cudaErrorInvalidDevice;
    const unsigned long long bit = 1ull << dev;
    if (done.load(std::memory_order_acquire) & bit)
        return cudaSuccess;
    e = setup(dev);
    if (e == cudaSuccess)
        done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// FP64 data of the reset path (csrc/arc_sim.c:88-110, csrc/arc_phys.c:749-782):
// forward-kinematics frames, default stance, limits.
struct ResetModel {
    int nb, nj, ns;
    int parent[kMaxJoints], child[kMaxJoints];
    V3<double> r1[kMaxJoints], r2[kMaxJoints], a1[kMaxJoints];
    Q4<double> q_rel0[kMaxJoints];
    double default_angles[kMaxJoints], lo[kMaxJoints], hi[kMaxJoints];
    double stand_height, footprint;
};

// ----- stepping
template <class R>
cudaError_t launch_step_plain(const DevModel<R>& M, const Worlds<R>& W, const Actuation& A, const int* ids,
                              int n_ids, cudaStream_t stream);

// Leg-parallel step: four lanes per world, state staged in shared memory.
// worlds_per_cta in {1, 2, 4, 8, 16, 32, 64} (a warp steps eight worlds;
// CTAs of 1, 2 or 4 worlds are part of a warp).
// spill: per world and lane, spill_per_lane contact records of 8 R beyond
// the on-chip ones; lane_cap bounds the contacts one lane can record.
template <class R>
cudaError_t launch_step_fast(const DevModel<R>& M, const Worlds<R>& W, const Actuation& A, R* spill,
                             int spill_per_lane, int lane_cap, int worlds_per_cta, cudaStream_t stream);

template <class R> size_t fast_smem_bytes(int stride, int worlds_per_cta);

// Warp-per-leg step (FP32, arc_task.cu): a CTA of four warps steps 32
// worlds, warp k runs leg k of every world; same spill layout as
// launch_step_fast. Steps the
// n_items worlds ids[0..n_items) (ids NULL: worlds 0..n_items-1). With a
// queue (two device ints, zero between launches) one wave of resident CTAs
// takes groups of 32 worlds from it until none is left. tile in
// 1 .. substeps - 1 (with tile_q: 13 x 4 floats per world): the control step
// as launches of `tile` substeps each, the same worlds bit for bit.
cudaError_t launch_step_warps(const DevModel<float>& M, const Worlds<float>& W, const Actuation& A, float* spill,
                              int spill_per_lane, int lane_cap, const int* ids, int n_items, int* queue,
                              cudaStream_t stream, int tile = 0, float* tile_q = nullptr);
// The same step in FP64 (arc_step_warps64.cu): two CTAs per SM (its bodies
// take twice the shared memory), the whole control step in one launch.
cudaError_t launch_step_warps64(const DevModel<double>& M, const Worlds<double>& W, const Actuation& A,
                                double* spill, int spill_per_lane, int lane_cap, const int* ids, int n_items,
                                int* queue, cudaStream_t stream);
constexpr int kFastOnChipContacts = 2;
constexpr int kWarpsOnChipContacts = 1;  // keeps four CTAs of the warp-per-leg kernel per SM
// the fewest on-chip records of any kernel: a spill area of lane_cap minus
// this many records per lane serves every kernel
constexpr int kMinOnChipContacts = kWarpsOnChipContacts;
constexpr int kFastMaxSubsteps = 1023;  // touch counters of the leg-parallel kernel

// ----- outputs of the reference ABI (double precision, any pointer may be null)
// rows in world order, or with ids the n_items worlds ids[0..n_items) in list order
template <class R>
cudaError_t launch_observe(const DevModel<R>& M, const Worlds<R>& W, double* root, double* rot, double* joints,
                           double* contacts, int* flags, cudaStream_t stream, const int* ids = nullptr,
                           int n_items = 0);
template <class R>
cudaError_t launch_heights(const Worlds<R>& W, const double* offsets, int k, double* out, cudaStream_t stream);
template <class R>
cudaError_t launch_terrain_at(const Worlds<R>& W, const int* ids, const double* xy, int m, double* out,
                              cudaStream_t stream);

// ----- snapshots: nb*13 + ns*8 + nj*4 + 2 doubles per world
template <class R>
cudaError_t launch_get_state(const DevModel<R>& M, const Worlds<R>& W, const int* ids, int n_ids, double* out,
                             cudaStream_t stream);
template <class R>
cudaError_t launch_set_state(const DevModel<R>& M, const Worlds<R>& W, const int* ids, int n_ids, const double* in,
                             cudaStream_t stream);

// ----- resets (FP64): seeded terrain + noisy stance (csrc/arc_sim.c:88-121)
// The reset kernels' RNG skip table; once per device, before any reset.
cudaError_t init_reset_tables(cudaStream_t stream);
template <class R>
cudaError_t launch_reset(const ResetModel& RM, const Worlds<R>& W, TerrainGeom<R>* tg, TerrainGeomD* tgd,
                         const int* ids, int n_ids, const unsigned* seeds, const double* difficulty,
                         const int* grid_of, double cell, cudaStream_t stream);

// Writes one world's terrain from FP64 heights already on the device.
template <class R>
cudaError_t launch_set_terrain(const Worlds<R>& W, TerrainGeom<R>* tg, TerrainGeomD* tgd, int id, int nx, int ny,
                               double cell, double outside, const double* heights, cudaStream_t stream);

}  // namespace arc
