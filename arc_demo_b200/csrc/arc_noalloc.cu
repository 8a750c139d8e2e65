// arc_noalloc.cu - a control step of quadruped worlds held in caller memory,
// with no device allocation by the library.
//
// Who needs it: callers that cannot call cudaMalloc. A host that owns all
// device memory through its own pre-allocated arena (a simulator or game
// runtime embedding this step) must not have a library allocate behind its
// back; a latency-critical control loop cannot afford cudaMalloc/cudaFree,
// which may synchronise the whole device. arc_sim_create allocates every
// buffer a simulation needs, so such callers cannot use it.
//
// What it does: the caller passes the worlds' state (the snapshot layout of
// arc_sim_get_state, FP64, on the device), their terrain heights and the
// drive targets. The entry point converts the state into the leg-parallel
// kernel's FP32 records, runs that kernel unchanged, and converts back. The
// records, terrain geometry and contact spill area the kernel needs live in
// one file-scope static device array, g_noalloc_scratch, of fixed size
// (kNoAllocMaxWorlds worlds), which every GPU that loads the library holds
// until the process exits.
#include <cstdio>
#include <mutex>

#include "arc_model.h"
#include "../../include/arc_sim.h"

namespace arc {
namespace {

constexpr int kNoAllocMaxWorlds = 1024;
constexpr int kNoAllocGridMax = kGridMax;
// FP32 record of the quadruped: 13 bodies x 13 + 21 spheres x 6 + 12 joints x 4
// = 343 floats, padded to 16 bytes
constexpr int kRecStride = 344;
constexpr int kSnap = 13 * 13 + 21 * 8 + 12 * 4 + 2;  // 387 doubles per world
// contact records one lane may spill beyond its two on-chip ones: the
// quadruped's bound for cells of at least 0.4 m (the reference's default
// cell, arc/task.py:22-23) is 29 records per lane
constexpr int kSpillPerLane = 28;
constexpr double kMinCell = 0.4;

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kOffRec = 0;
constexpr size_t kOffSph = align256(kOffRec + sizeof(float) * kNoAllocMaxWorlds * kRecStride);
constexpr size_t kOffUnstable = align256(kOffSph + sizeof(uint32_t) * kNoAllocMaxWorlds * 21);
constexpr size_t kOffTime = align256(kOffUnstable + sizeof(int) * kNoAllocMaxWorlds);
constexpr size_t kOffToff = align256(kOffTime + sizeof(double) * kNoAllocMaxWorlds);
constexpr size_t kOffTg = align256(kOffToff + sizeof(long long) * kNoAllocMaxWorlds);
constexpr size_t kOffTgd = align256(kOffTg + sizeof(TerrainGeom<float>) * kNoAllocMaxWorlds);
constexpr size_t kOffSpill = align256(kOffTgd + sizeof(TerrainGeomD) * kNoAllocMaxWorlds);
constexpr size_t kOffEnd = align256(kOffSpill + sizeof(float) * (size_t)kNoAllocMaxWorlds * 4 * kSpillPerLane * 8);
#ifdef ARC_DEVICE_CHECKS
// the checked build also records each world's grid, against which its
// kernels test every terrain column they read
constexpr size_t kOffGridOf = kOffEnd;
constexpr size_t kScratchBytes = align256(kOffGridOf + sizeof(int) * kNoAllocMaxWorlds);
#else
constexpr size_t kScratchBytes = kOffEnd;  // ~4.9 MB
#endif

// Shared by every call on a device and kept between calls: calls whose
// work overlaps on the GPU race on it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// snapshot (FP64, caller memory) -> FP32 records, flags and terrain geometry (scratch)
__global__ void k_noalloc_in(unsigned char* scratch, const double* __restrict__ state, int n, int grid, double cell,
                             double outside)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    float* rec = reinterpret_cast<float*>(scratch + kOffRec) + (size_t)i * kRecStride;
    uint32_t* sph = reinterpret_cast<uint32_t*>(scratch + kOffSph) + (size_t)i * 21;
    const double* p = state + (size_t)i * kSnap;
    for (int k = 0; k < 13 * 13; ++k)
        rec[k] = (float)p[k];
    p += 13 * 13;
    float* sr = rec + 13 * 13;
    for (int s = 0; s < 21; ++s, p += 8) {
        for (int c = 0; c < 6; ++c)
            sr[s * 6 + c] = (float)p[1 + c];
        sph[s] = ((uint32_t)p[7] & 0xffffu) | ((uint32_t)(p[0] != 0.0) << 16);
    }
    float* jr = sr + 21 * 6;
    for (int j = 0; j < 12 * 4; ++j)
        jr[j] = (float)p[j];
    p += 12 * 4;
    rec[kRecStride - 1] = 0.0f;
    reinterpret_cast<int*>(scratch + kOffUnstable)[i] = p[0] != 0.0;
    reinterpret_cast<double*>(scratch + kOffTime)[i] = p[1];
    reinterpret_cast<long long*>(scratch + kOffToff)[i] = (long long)i * grid * grid;
    const TerrainGeomD g{grid, grid, cell, -0.5 * grid * cell, -0.5 * grid * cell, outside};
    reinterpret_cast<TerrainGeomD*>(scratch + kOffTgd)[i] = g;
    reinterpret_cast<TerrainGeom<float>*>(scratch + kOffTg)[i] =
        TerrainGeom<float>{grid, grid, (float)g.cell, (float)g.ox, (float)g.oy, (float)g.outside};
#ifdef ARC_DEVICE_CHECKS
    reinterpret_cast<int*>(scratch + kOffGridOf)[i] = grid;
#endif
}

// FP32 records (scratch) -> snapshot (FP64, caller memory)
__global__ void k_noalloc_out(const unsigned char* scratch, double* __restrict__ state, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float* rec = reinterpret_cast<const float*>(scratch + kOffRec) + (size_t)i * kRecStride;
    const uint32_t* sph = reinterpret_cast<const uint32_t*>(scratch + kOffSph) + (size_t)i * 21;
    double* p = state + (size_t)i * kSnap;
    for (int k = 0; k < 13 * 13; ++k)
        p[k] = (double)rec[k];
    p += 13 * 13;
    const float* sr = rec + 13 * 13;
    for (int s = 0; s < 21; ++s, p += 8) {
        p[0] = (double)((sph[s] >> 16) & 1u);
        for (int c = 0; c < 6; ++c)
            p[1 + c] = (double)sr[s * 6 + c];
        p[7] = (double)(sph[s] & 0xffffu);
    }
    const float* jr = sr + 21 * 6;
    for (int j = 0; j < 12 * 4; ++j)
        p[j] = (double)jr[j];
    p += 12 * 4;
    p[0] = (double)reinterpret_cast<const int*>(scratch + kOffUnstable)[i];
    p[1] = reinterpret_cast<const double*>(scratch + kOffTime)[i];
}

// Device address of g_noalloc_scratch for each device, looked up once per
// device with that device current (host code cannot use the symbol itself).
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

unsigned char* scratch_for_current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return nullptr;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "arc_step_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return nullptr;
        }
        g_scratch_ptr[dev] = static_cast<unsigned char*>(ptr);
    }
    return g_scratch_ptr[dev];
}

// the quadruped's model constants, built once on the host (no device memory)
std::once_flag g_model_once;
ModelHost g_model;

}  // namespace
}  // namespace arc

using namespace arc;

extern "C" int arc_step_noalloc(double* d_state, const float* d_heights, int grid, double cell, double outside,
                                const double* d_targets, int n_worlds, double dt, int substeps, void* stream)
{
    if (n_worlds < 0 || n_worlds > kNoAllocMaxWorlds) {
        std::fprintf(stderr, "arc_step_noalloc: %d worlds; at most %d per call\n", n_worlds, kNoAllocMaxWorlds);
        return ARC_ERR_ARG;
    }
    if (grid < 1 || grid > kNoAllocGridMax || !(cell >= kMinCell) || substeps < 1 || substeps > kFastMaxSubsteps ||
        !(dt > 0.0)) {
        std::fprintf(stderr, "arc_step_noalloc: need 1 <= grid <= %d, cell >= %.1f m, 1 <= substeps <= %d, dt > 0\n",
                     kNoAllocGridMax, kMinCell, kFastMaxSubsteps);
        return ARC_ERR_ARG;
    }
    if (n_worlds == 0)
        return ARC_OK;
    if (!d_state || !d_heights || !d_targets)
        return ARC_ERR_ARG;
    unsigned char* scratch = scratch_for_current_device();
    if (!scratch)
        return ARC_ERR_CUDA;
    std::call_once(g_model_once, [] { build_leaper(g_model); });
    // the most contact records one lane can make in a substep on these
    // columns; the spill area holds all but the kernel's on-chip ones
    const int lane_cap = lane_contact_bound(g_model, cell);
    if (lane_cap > kSpillPerLane + kFastOnChipContacts) {
        std::fprintf(stderr, "arc_step_noalloc: %d contacts per lane on %.3f m cells exceed the static spill area (%d)\n",
                     lane_cap, cell, kSpillPerLane + kFastOnChipContacts);
        return ARC_ERR_ARG;
    }
    const DevModel<float> M = make_dev_model<float>(g_model, dt, substeps, 0.6);

    Worlds<float> W;
    W.rec = reinterpret_cast<float*>(scratch + kOffRec);
    W.stride = kRecStride;
    W.off_sphere = 13 * kBodyRec;
    W.off_joint = W.off_sphere + 21 * kSphereRec;
    W.sph = reinterpret_cast<uint32_t*>(scratch + kOffSph);
    W.unstable = reinterpret_cast<int*>(scratch + kOffUnstable);
    W.time = reinterpret_cast<double*>(scratch + kOffTime);
    W.th = const_cast<float*>(d_heights);
    W.toff = reinterpret_cast<const long long*>(scratch + kOffToff);
    W.tg = reinterpret_cast<const TerrainGeom<float>*>(scratch + kOffTg);
    W.tgd = reinterpret_cast<const TerrainGeomD*>(scratch + kOffTgd);
    W.n = n_worlds;
#ifdef ARC_DEVICE_CHECKS
    W.grid_of = reinterpret_cast<const int*>(scratch + kOffGridOf);
#endif

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int threads = 128, blocks = (n_worlds + threads - 1) / threads;
    k_noalloc_in<<<blocks, threads, 0, st>>>(scratch, d_state, n_worlds, grid, cell, outside);
    if (cudaGetLastError() != cudaSuccess)
        return ARC_ERR_CUDA;
    Actuation A{d_targets, nullptr};
    // a lane keeps kFastOnChipContacts (2) records on chip and spills the
    // rest, at most lane_cap - 2 <= kSpillPerLane of them
    if (launch_step_fast<float>(M, W, A, reinterpret_cast<float*>(scratch + kOffSpill), kSpillPerLane, lane_cap, 8,
                                st) != cudaSuccess)
        return ARC_ERR_CUDA;
    k_noalloc_out<<<blocks, threads, 0, st>>>(scratch, d_state, n_worlds);
    return cudaGetLastError() == cudaSuccess ? ARC_OK : ARC_ERR_CUDA;
}
