// arc_device.cuh - device data layout of a batch of worlds.
//
// HBM layout (one arc_sim owns all of it):
//   rec      [N][stride] R   per-world record, contiguous so a CTA can stage
//                           a world with vector loads:
//                             bodies  nb x (x3 q4 v3 w3)         13 R each
//                             spheres ns x (anchor3 anchor_n3)   6 R each
//                             joints  nj x (target angle rate torque)
//                           stride is padded to a multiple of 16 bytes
//   sph      [N][ns] u32     touch count (low 16 bits) | anchored << 16
//   unstable [N] i32, time [N] f64
//   terrain  heights pool (R), per-world offset and geometry, so worlds may
//            have different grid sizes
// The model (robot constants, identical for every world) travels as a
// __grid_constant__ kernel parameter and is staged into shared memory by
// kernels whose lanes read different entries.
#pragma once

#include "arc_solver.cuh"

namespace arc {

constexpr int kMaxBodies = 16;   // csrc/arc_phys.h:19-23
constexpr int kMaxJoints = 16;
constexpr int kMaxSpheres = 48;
constexpr int kMaxContacts = 128;
constexpr int kGridMax = 64;     // csrc/arc_terrain.h:10
constexpr int kBodyRec = 13;
constexpr int kSphereRec = 6;
constexpr int kJointRec = 4;
constexpr int kContactRec = 8;
constexpr int kNumLegs = 4;      // csrc/arc_robot.h:19-20
constexpr int kNumJoints = 12;

template <class R> struct DevModel {
    int nb, nj, ns, n_channels;
    int substeps;
    double step_dt;  // dt of one control step (world time advance)
    int leaper;  // topology of csrc/arc_robot.c: torso + 4 legs of 3 joints
    BodyK<R> body[kMaxBodies];
    JointK<R> joint[kMaxJoints];
    SphereK<R> sphere[kMaxSpheres];
    int channel[kMaxSpheres];  // observe contact channel (csrc/arc_sim.c:47-50)
    StepK<R> step;
    R lo[kMaxJoints], hi[kMaxJoints];   // target clamp (csrc/arc_sim.c:132-134)
    double default_angles[kMaxJoints];  // actuation: default + scale * clip(a)
    double action_scale;
};

template <class R> struct TerrainGeom {
    int nx, ny;
    R cell, ox, oy, outside;
};

struct TerrainGeomD {
    int nx, ny;
    double cell, ox, oy, outside;
};

template <class R> struct Worlds {
    R* rec;
    int stride;          // in R
    int off_sphere, off_joint;
    uint32_t* sph;
    int* unstable;
    double* time;
    R* th;               // terrain heights pool
    const long long* toff;
    const TerrainGeom<R>* tg;
    const TerrainGeomD* tgd;
    int n;
    // the last substep's contact list per world (csrc/arc_phys.h:100-112),
    // written by the step kernels when not NULL: kMaxContacts records of
    // kContactRec R (body, local3, n3, unused) and the count
    R* lastc = nullptr;
    int* lastn = nullptr;
#ifdef ARC_DEVICE_CHECKS
    const int* grid_of = nullptr;  // terrain capacity of each world: grid_of[i]^2 columns
#endif
};

// Columns of world i's slice of the terrain pool (checked build; -1: unknown)
template <class R> ARC_HD long long terrain_cap(const Worlds<R>& W, int i)
{
#ifdef ARC_DEVICE_CHECKS
    return W.grid_of ? (long long)W.grid_of[i] * W.grid_of[i] : -1;
#else
    return -1;
#endif
}

// Whether column c lies in world i's slice of the terrain pool: always in
// the regular build, checked (and recorded under `site` when not) in the
// checked build.
template <class R> ARC_HD bool terrain_column_ok(const Worlds<R>& W, int i, long long c, int site)
{
#ifdef ARC_DEVICE_CHECKS
    const long long cap = terrain_cap(W, i);
    return cap < 0 || ARC_IN_BOUNDS(c, cap, site);
#else
    (void)W, (void)i, (void)c, (void)site;
    return true;
#endif
}

template <class R> ARC_HD TerrainView<R> terrain_of(const Worlds<R>& W, int i)
{
    TerrainGeom<R> g = W.tg[i];
    TerrainView<R> v{W.th + W.toff[i], g.nx, g.ny, g.cell, g.ox, g.oy, g.outside};
#ifdef ARC_DEVICE_CHECKS
    v.cap = terrain_cap(W, i);
#endif
    return v;
}

// How a step kernel gets its drive targets.
//   targets64: N x nj FP64 targets (the reference ABI, csrc/arc_sim.c:123-138)
//   actions32: N x nj FP32 policy actions; target = default + scale * clip(a, -1, 1)
//              in FP64 (arc/task.py:159-160), then clamped
struct Actuation {
    const double* targets64;
    const float* actions32;
};

template <class R>
ARC_HD R actuate(const DevModel<R>& M, const Actuation& A, int i, int j)
{
    double t;
    if (A.actions32) {
        double a = (double)A.actions32[(size_t)i * M.nj + j];
        a = a < -1.0 ? -1.0 : (a > 1.0 ? 1.0 : a);
        t = M.default_angles[j] + M.action_scale * a;
    } else {
        t = A.targets64[(size_t)i * M.nj + j];
    }
    // csrc/arc_sim.c:132-134 clamps to the limits; a joint whose limits are
    // off (lo > hi, csrc/arc_phys.c:140-141) takes the target as given
    return M.lo[j] <= M.hi[j] ? r_clamp((R)t, M.lo[j], M.hi[j]) : (R)t;
}

// Contacts that do not fit in a kernel's on-chip list go to this per-world
// scratch area in HBM, kMaxContacts records per world.
template <class R> struct ContactSpill {
    ContactRec<R>* rec;  // [N][kMaxContacts]
    int* body;           // [N][kMaxContacts]
};

// Error flags a kernel can raise (host reads them after a sync).
enum : int {
    kErrNone = 0,
    kErrModel = 1,  // model topology not supported by this kernel
};

}  // namespace arc
