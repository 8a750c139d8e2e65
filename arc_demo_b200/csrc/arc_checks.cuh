// arc_checks.cuh - index checks of the checked build (-DARC_DEVICE_CHECKS).
//
// A second build of the library (libarcsim_checked.so) checks the kernels'
// data-dependent indexes at the sites below against the slice of memory
// each belongs to: a terrain cell against its world's share of the terrain
// pool, a contact record against its lane's share of the spill buffer. A
// failed check counts, keeps the first site and index, and skips the access
// (a read yields a neutral value, a write is dropped); nothing traps or
// waits. arc_device_checks() reads the count and the first failure and
// clears them. In the regular build every check is `true` and compiles away.
#pragma once

namespace arc {

enum CheckSite : int {
    kCheckTerrainRead = 1,    // a sphere's terrain column (step kernels)
    kCheckSpillWrite = 2,     // a contact record beyond the on-chip ones
    kCheckSpillRead = 3,      // ... read back by the velocity pass
    kCheckHeightsRead = 4,    // an observation height or a terrain lookup (task, observe)
    kCheckTerrainWrite = 5,   // a reset's new terrain
};

}  // namespace arc

#if defined(ARC_DEVICE_CHECKS) && defined(__CUDACC__)
#include <cuda_runtime.h>

namespace arc {

// defined in arc_sim.cu: collects one reader per translation unit
int register_device_checks(int (*read)(unsigned long long* record, bool clear));

// each translation unit keeps its own record (internal linkage)
static __device__ unsigned long long g_check[3];  // failures, first site, first index

static int read_device_checks(unsigned long long* record, bool clear)
{
    if (cudaMemcpyFromSymbol(record, g_check, sizeof(g_check)) != cudaSuccess)
        return -1;
    if (clear) {
        const unsigned long long zero[3] = {0, 0, 0};
        if (cudaMemcpyToSymbol(g_check, zero, sizeof(zero)) != cudaSuccess)
            return -1;
    }
    return 0;
}

static const int g_check_registered = register_device_checks(&read_device_checks);

static __device__ __forceinline__ bool in_bounds(long long i, long long n, int site)
{
    if (i >= 0 && i < n)
        return true;
    if (atomicAdd(&g_check[0], 1ull) == 0) {
        g_check[1] = (unsigned long long)site;
        g_check[2] = (unsigned long long)i;
    }
    return false;
}

}  // namespace arc

#ifdef __CUDA_ARCH__
#define ARC_IN_BOUNDS(i, n, site) ::arc::in_bounds((long long)(i), (long long)(n), (site))
#else
#define ARC_IN_BOUNDS(i, n, site) true  // the host pass of host-device helpers
#endif
#else
#define ARC_IN_BOUNDS(i, n, site) true
#endif
