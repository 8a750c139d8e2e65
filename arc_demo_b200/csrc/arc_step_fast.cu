// arc_step_fast.cu - the leg-parallel step kernel.
//
// Four lanes step one world, one lane per leg; a warp steps eight worlds.
// The world's record is staged from HBM into shared memory with 16-byte
// vector copies (one contiguous block per CTA), stepped there, and written
// back once per control step.
//
// Why four lanes: 66% of the reference's arithmetic is the serial
// Gauss-Seidel chain of 12 joint solves per substep (csrc/arc_phys.c:729-730).
// In the leaper (csrc/arc_robot.c:145-195) joint 3k+c links, for leg k,
// torso -> coxa -> femur -> tibia, so the solves of one leg touch only that
// leg's bodies, except joint 3k, which also moves the torso. Running the
// joints in the reference order 0..11 is therefore the same computation as
// this six-slot wavefront, in which lane k runs joint 3k+(s-k) at slot s:
//
//   slot 0: J0            slot 3: J5 J7 J9
//   slot 1: J1 J3         slot 4: J8 J10
//   slot 2: J2 J4 J6      slot 5: J11
//
// Every pair of solves that this reorders touches disjoint bodies, so each
// body sees exactly the reference's sequence of updates (bitwise, up to FMA
// contraction). The same holds for the velocity pass (csrc/arc_phys.c:734-735).
// Sphere contacts and the contact velocity pass change only the sphere's own
// body (csrc/arc_phys.c:488-626), so each lane handles its leg's spheres
// (lane 0 also the torso sphere), in the reference's per-body order.
//
// Contacts: each lane keeps its first kOnChip contact records in shared
// memory and the rest in a per-world HBM spill area; the reference's cap of
// 128 per world (csrc/arc_phys.c:493) is applied in the reference's order
// (sphere order, which is lane-major) with a 4-lane prefix sum.
#include "arc_kernels.cuh"

namespace arc {

namespace fast {

constexpr int kLanes = 4;     // lanes per world (legs)
constexpr int kDer = 22;      // per-body derived data: rot 9, iiw 6, x_prev 3, q_prev 4
constexpr int kOnChip = kFastOnChipContacts;  // contact records per lane in shared memory
constexpr int kCRec = 8;      // local 3, n 3, body, pad
constexpr int kSlots = 6;     // joint wavefront length
constexpr int kLaneSpheres = 6;

template <class R> struct SmemModel {
    BodyK<R> body[13];
    JointK<R> joint[12];
    SphereK<R> sphere[21];
};

__host__ __device__ constexpr size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

// body handled by `leg` at iteration it of the per-body phases
__device__ __forceinline__ int body_of(int leg, int it) { return it == 0 ? (leg == 0 ? 0 : -1) : 3 * leg + it; }
// sphere handled by `leg` at iteration it of the collision phase
__device__ __forceinline__ int sphere_of(int leg, int it) { return it == 0 ? (leg == 0 ? 0 : -1) : 5 * leg + it; }

template <class R> struct Stage {
    R* rec;   // the world's record (bodies x q v w, spheres, joints)
    R* der;   // derived per-body data
    __device__ __forceinline__ void load_pose(int b, Pose<R>& P) const
    {
        const R* r = rec + b * kBodyRec;
        const R* d = der + b * kDer;
        P.x = V3<R>{r[0], r[1], r[2]};
        P.q = Q4<R>{r[3], r[4], r[5], r[6]};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                P.rot.m[a][c] = d[a * 3 + c];
        P.iiw = S3<R>{d[9], d[10], d[11], d[12], d[13], d[14]};
    }
    __device__ __forceinline__ void store_pose(int b, const Pose<R>& P) const
    {
        R* r = rec + b * kBodyRec;
        R* d = der + b * kDer;
        r[0] = P.x.x; r[1] = P.x.y; r[2] = P.x.z;
        r[3] = P.q.w; r[4] = P.q.x; r[5] = P.q.y; r[6] = P.q.z;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                d[a * 3 + c] = P.rot.m[a][c];
        d[9] = P.iiw.xx; d[10] = P.iiw.xy; d[11] = P.iiw.xz;
        d[12] = P.iiw.yy; d[13] = P.iiw.yz; d[14] = P.iiw.zz;
    }
    __device__ __forceinline__ V3<R> v(int b) const { const R* r = rec + b * kBodyRec; return V3<R>{r[7], r[8], r[9]}; }
    __device__ __forceinline__ V3<R> w(int b) const { const R* r = rec + b * kBodyRec; return V3<R>{r[10], r[11], r[12]}; }
    __device__ __forceinline__ void set_v(int b, V3<R> a) const { R* r = rec + b * kBodyRec; r[7] = a.x; r[8] = a.y; r[9] = a.z; }
    __device__ __forceinline__ void set_w(int b, V3<R> a) const { R* r = rec + b * kBodyRec; r[10] = a.x; r[11] = a.y; r[12] = a.z; }
    __device__ __forceinline__ V3<R> xp(int b) const { const R* d = der + b * kDer; return V3<R>{d[15], d[16], d[17]}; }
    __device__ __forceinline__ Q4<R> qp(int b) const { const R* d = der + b * kDer; return Q4<R>{d[18], d[19], d[20], d[21]}; }
    __device__ __forceinline__ void set_prev(int b, V3<R> x, Q4<R> q) const
    {
        R* d = der + b * kDer;
        d[15] = x.x; d[16] = x.y; d[17] = x.z;
        d[18] = q.w; d[19] = q.x; d[20] = q.y; d[21] = q.z;
    }
    __device__ __forceinline__ const R* rot(int b) const { return der + b * kDer; }
    __device__ __forceinline__ S3<R> iiw(int b) const
    {
        const R* d = der + b * kDer;
        return S3<R>{d[9], d[10], d[11], d[12], d[13], d[14]};
    }
    __device__ __forceinline__ M3<R> rotm(int b) const
    {
        const R* d = der + b * kDer;
        M3<R> m;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                m.m[a][c] = d[a * 3 + c];
        return m;
    }
};

template <class R> __host__ __device__ size_t smem_bytes(int stride, int wpc)
{
    size_t b = align16(sizeof(SmemModel<R>));
    b += align16(sizeof(R) * (size_t)wpc * stride);
    b += align16(sizeof(R) * (size_t)wpc * 13 * kDer);
    b += align16(sizeof(R) * (size_t)wpc * 12);
    b += align16(sizeof(R) * (size_t)wpc * kLanes * kOnChip * kCRec);
    return b;
}

template <class R, int WPC>
__global__ void __launch_bounds__(WPC * kLanes)
k_step_fast(const __grid_constant__ DevModel<R> M, Worlds<R> W, Actuation A, R* __restrict__ spill, int spill_per_lane,
            int lane_cap)
{
    extern __shared__ __align__(16) unsigned char smem[];
    SmemModel<R>& sm = *reinterpret_cast<SmemModel<R>*>(smem);
    R* s_rec = reinterpret_cast<R*>(smem + align16(sizeof(SmemModel<R>)));
    R* s_der = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(s_rec) + align16(sizeof(R) * WPC * W.stride));
    R* s_tacc = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(s_der) + align16(sizeof(R) * WPC * 13 * kDer));
    R* s_con = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(s_tacc) + align16(sizeof(R) * WPC * 12));

    const int tid = threadIdx.x, wl = tid / kLanes, leg = tid % kLanes;
    // the lanes of a warp that exist: CTAs of 1, 2 or 4 worlds are 4, 8 or 16 threads
    constexpr unsigned kMask = WPC * kLanes >= 32 ? 0xffffffffu : (1u << (WPC * kLanes)) - 1u;
    const int w0 = blockIdx.x * WPC;
    const int nw = min(WPC, W.n - w0);
    const int world = w0 + wl;
    const bool valid = wl < nw;

    // model constants to shared memory (lanes read different entries)
    for (int k = tid; k < 13; k += blockDim.x)
        sm.body[k] = M.body[k];
    for (int k = tid; k < 12; k += blockDim.x)
        sm.joint[k] = M.joint[k];
    for (int k = tid; k < 21; k += blockDim.x)
        sm.sphere[k] = M.sphere[k];
    // the CTA's world records are one contiguous block: 16-byte copies
    {
        using V = typename std::conditional<sizeof(R) == 4, float4, double2>::type;
        constexpr int per = 16 / sizeof(R);
        const int nvec = nw * W.stride / per;
        const V* src = reinterpret_cast<const V*>(W.rec + (size_t)w0 * W.stride);
        V* dst = reinterpret_cast<V*>(s_rec);
        for (int k = tid; k < nvec; k += blockDim.x)
            dst[k] = src[k];
    }
    __syncthreads();

    const Stage<R> S{s_rec + wl * W.stride, s_der + wl * 13 * kDer};
    R* jr = S.rec + W.off_joint;
    R* sr = S.rec + W.off_sphere;
    R* tacc = s_tacc + wl * 12;
    R* con = s_con + (size_t)tid * kOnChip * kCRec;
    R* spl = spill + ((size_t)(valid ? world : 0) * kLanes + leg) * (size_t)spill_per_lane * kCRec;

    // actuation (csrc/arc_sim.c:132-136): this lane's three joints
    if (valid) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int j = 3 * leg + c;
            jr[j * kJointRec] = actuate(M, A, world, j);
            tacc[j] = R(0);
        }
    }
    const bool active = valid && W.unstable[world] == 0;

    // per-sphere state of this lane: anchored bits, touch counts packed
    // 10 bits each (the host runs this kernel only for <= 1023 substeps)
    uint32_t anch = 0;
    unsigned long long touches = 0;
    const uint32_t* sph = W.sph + (size_t)(valid ? world : 0) * 21;
#pragma unroll
    for (int it = 0; it < kLaneSpheres; ++it) {
        const int s = sphere_of(leg, it);
        if (valid && s >= 0)
            anch |= ((sph[s] >> 16) & 1u) << it;
    }
    const TerrainView<R> T = terrain_of(W, valid ? world : 0);
    const StepK<R>& st = M.step;

    // csrc/arc_phys.c:713-714
#pragma unroll 1
    for (int it = 0; it < 4; ++it) {
        const int b = body_of(leg, it);
        if (active && b >= 0) {
            Pose<R> P;
            const R* r = S.rec + b * kBodyRec;
            P.x = V3<R>{r[0], r[1], r[2]};
            P.q = Q4<R>{r[3], r[4], r[5], r[6]};
            body_sync(P, sm.body[b]);
            S.store_pose(b, P);
        }
    }
    __syncwarp(kMask);

    for (int sub = 0; sub < M.substeps; ++sub) {
        // integrate (csrc/arc_phys.c:658-672)
#pragma unroll 1
        for (int it = 0; it < 4; ++it) {
            const int b = body_of(leg, it);
            if (active && b >= 0) {
                Pose<R> P;
                S.load_pose(b, P);
                V3<R> v = S.v(b), w = S.w(b), xp;
                Q4<R> qp;
                integrate_body(P, v, w, xp, qp, sm.body[b], st);
                S.store_pose(b, P);
                S.set_v(b, v);
                S.set_w(b, w);
                S.set_prev(b, xp, qp);
            }
        }
        __syncwarp(kMask);

        // joint positions: the six-slot wavefront
        for (int slot = 0; slot < kSlots; ++slot) {
            const int li = slot - leg;
            if (active && li >= 0 && li < 3) {
                const int j = 3 * leg + li;
                const JointK<R>& jk = sm.joint[j];
                const int p = jk.parent, c = jk.child;
                Pose<R> Pp, Pc;
                S.load_pose(p, Pp);
                S.load_pose(c, Pc);
                R ta = tacc[j];
                joint_positions<R, true>(Pp, sm.body[p], Pc, sm.body[c], jk, joint_step_k(jk, st), jr[j * kJointRec],
                                         ta, st.hh);
                tacc[j] = ta;
                S.store_pose(p, Pp);
                S.store_pose(c, Pc);
            }
            __syncwarp(kMask);
        }

        // sphere contacts (csrc/arc_phys.c:731-732)
        int nc = 0;
        {
            int cur = -1;
            Pose<R> P;
            V3<R> xp{};
            Q4<R> qp{};
#pragma unroll 1
            for (int it = 0; it < kLaneSpheres; ++it) {
                const int s = sphere_of(leg, it);
                if (active && s >= 0) {
                    const SphereK<R>& sk = sm.sphere[s];
                    const int b = sk.body;
                    if (b != cur) {
                        if (cur >= 0)
                            S.store_pose(cur, P);
                        S.load_pose(b, P);
                        xp = S.xp(b);
                        qp = S.qp(b);
                        cur = b;
                    }
                    R* a = sr + s * kSphereRec;
                    SphereState<R> ss{V3<R>{a[0], a[1], a[2]}, V3<R>{a[3], a[4], a[5]}, (int)((anch >> it) & 1u)};
                    const int t = collide_sphere(P, sm.body[b], xp, qp, sk, ss, T, st, [&](V3<R> local, V3<R> n) {
                        R* dst = nc < kOnChip ? con + nc * kCRec
                                 : (nc < lane_cap && ARC_IN_BOUNDS(nc - kOnChip, spill_per_lane, kCheckSpillWrite))
                                     ? spl + (size_t)(nc - kOnChip) * kCRec
                                     : nullptr;
                        if (dst) {
                            dst[0] = local.x; dst[1] = local.y; dst[2] = local.z;
                            dst[3] = n.x; dst[4] = n.y; dst[5] = n.z;
                            dst[6] = (R)b;
                        }
                        ++nc;
                    });
                    touches += (unsigned long long)t << (10 * it);
                    anch = (anch & ~(1u << it)) | ((uint32_t)(ss.anchored != 0) << it);
                    a[0] = ss.anchor.x; a[1] = ss.anchor.y; a[2] = ss.anchor.z;
                    a[3] = ss.anchor_n.x; a[4] = ss.anchor_n.y; a[5] = ss.anchor_n.z;
                }
            }
            if (cur >= 0)
                S.store_pose(cur, P);
        }
        __syncwarp(kMask);

        // velocities from positions (csrc/arc_phys.c:674-687)
#pragma unroll 1
        for (int it = 0; it < 4; ++it) {
            const int b = body_of(leg, it);
            if (active && b >= 0) {
                R* r = S.rec + b * kBodyRec;
                Q4<R> q{r[3], r[4], r[5], r[6]};
                V3<R> x{r[0], r[1], r[2]}, v, w;
                update_velocity(q, x, v, w, S.xp(b), S.qp(b), st);
                r[3] = q.w; r[4] = q.x; r[5] = q.y; r[6] = q.z;
                S.set_v(b, v);
                S.set_w(b, w);
            }
        }
        __syncwarp(kMask);

        // drive damping: the same wavefront
        for (int slot = 0; slot < kSlots; ++slot) {
            const int li = slot - leg;
            if (active && li >= 0 && li < 3) {
                const int j = 3 * leg + li;
                const JointK<R>& jk = sm.joint[j];
                const int p = jk.parent, c = jk.child;
                V3<R> wp = S.w(p), wc = S.w(c);
                R ta = tacc[j];
                joint_velocities<R, true>(S.rotm(p), S.iiw(p), wp, S.iiw(c), wc, jk, joint_step_k(jk, st), st.h, ta);
                tacc[j] = ta;
                S.set_w(p, wp);
                S.set_w(c, wc);
            }
            __syncwarp(kMask);
        }

        // contact velocities, in the reference's order and under its cap:
        // base = number of this world's contacts recorded by lower lanes
        int base;
        {
            int x = nc;
            int y = __shfl_up_sync(kMask, x, 1, kLanes);
            if (leg >= 1)
                x += y;
            y = __shfl_up_sync(kMask, x, 2, kLanes);
            if (leg >= 2)
                x += y;
            base = x - nc;
        }
        if (active) {
            const int ncl = nc < lane_cap ? nc : lane_cap;
            // the last substep's list (lane-major is the reference's order)
            R* lastc = W.lastc && sub == M.substeps - 1 ? W.lastc + (size_t)world * kMaxContacts * kContactRec
                                                        : nullptr;
            if (lastc && leg == kLanes - 1)
                W.lastn[world] = base + ncl < kMaxContacts ? base + ncl : kMaxContacts;
            for (int c = 0; c < ncl && base + c < kMaxContacts; ++c) {
                if (c >= kOnChip && !ARC_IN_BOUNDS(c - kOnChip, spill_per_lane, kCheckSpillRead))
                    continue;
                const R* src = c < kOnChip ? con + c * kCRec : spl + (size_t)(c - kOnChip) * kCRec;
                ContactRec<R> cr{V3<R>{src[0], src[1], src[2]}, V3<R>{src[3], src[4], src[5]}};
                const int b = (int)src[6];
                if (lastc) {
                    R* d = lastc + (size_t)(base + c) * kContactRec;
                    d[0] = (R)b;
                    for (int f = 0; f < 6; ++f)
                        d[1 + f] = src[f];
                }
                V3<R> v = S.v(b), w = S.w(b);
                contact_velocity(S.rotm(b), S.iiw(b), sm.body[b].inv_mass, v, w, cr);
                S.set_v(b, v);
                S.set_w(b, w);
            }
        }
        __syncwarp(kMask);
    }

    // epilogue (csrc/arc_phys.c:739-746)
    bool bad = false;
    if (active) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int j = 3 * leg + c;
            const JointK<R>& jk = sm.joint[j];
            const R* rp = S.rec + jk.parent * kBodyRec;
            const R* rc = S.rec + jk.child * kBodyRec;
            Q4<R> qp{rp[3], rp[4], rp[5], rp[6]}, qc{rc[3], rc[4], rc[5], rc[6]};
            jr[j * kJointRec + 1] = joint_angle(qp, qc, jk);
            jr[j * kJointRec + 2] = joint_rate(qp, S.w(jk.parent), S.w(jk.child), jk);
            jr[j * kJointRec + 3] = tacc[j] / R(M.substeps);
        }
#pragma unroll
        for (int it = 0; it < 4; ++it) {
            const int b = body_of(leg, it);
            if (b >= 0) {
                const R* r = S.rec + b * kBodyRec;
                bad |= body_unstable(V3<R>{r[0], r[1], r[2]}, S.v(b), S.w(b));
            }
        }
    }
    int badi = bad ? 1 : 0;
    badi |= __shfl_xor_sync(kMask, badi, 1, kLanes);
    badi |= __shfl_xor_sync(kMask, badi, 2, kLanes);
    if (active) {
        uint32_t* sphw = W.sph + (size_t)world * 21;
#pragma unroll
        for (int it = 0; it < kLaneSpheres; ++it) {
            const int s = sphere_of(leg, it);
            if (s >= 0)
                sphw[s] = (uint32_t)((touches >> (10 * it)) & 1023u) | (((anch >> it) & 1u) << 16);
        }
        if (leg == 0) {
            W.time[world] += M.step_dt;
            if (badi)
                W.unstable[world] = 1;
        }
    }
    __syncthreads();
    {
        using V = typename std::conditional<sizeof(R) == 4, float4, double2>::type;
        constexpr int per = 16 / sizeof(R);
        const int nvec = nw * W.stride / per;
        V* dst = reinterpret_cast<V*>(W.rec + (size_t)w0 * W.stride);
        const V* src = reinterpret_cast<const V*>(s_rec);
        for (int k = tid; k < nvec; k += blockDim.x)
            dst[k] = src[k];
    }
}

}  // namespace fast

template <class R> size_t fast_smem_bytes(int stride, int worlds_per_cta)
{
    return fast::smem_bytes<R>(stride, worlds_per_cta);
}

template <class R, int WPC>
static cudaError_t launch_fast_wpc(const DevModel<R>& M, const Worlds<R>& W, const Actuation& A, R* spill,
                                   int spill_per_lane, int lane_cap, cudaStream_t stream)
{
    const size_t smem = fast::smem_bytes<R>(W.stride, WPC);
    static std::atomic<unsigned long long> configured{0};
    cudaError_t e = once_per_device(configured, [&](int) {
        return cudaFuncSetAttribute(fast::k_step_fast<R, WPC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem > 48 * 1024 ? (int)smem : 48 * 1024);
    });
    if (e != cudaSuccess)
        return e;
    const int grid = (W.n + WPC - 1) / WPC;
    fast::k_step_fast<R, WPC><<<grid, WPC * fast::kLanes, smem, stream>>>(M, W, A, spill, spill_per_lane, lane_cap);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_step_fast(const DevModel<R>& M, const Worlds<R>& W, const Actuation& A, R* spill,
                             int spill_per_lane, int lane_cap, int worlds_per_cta, cudaStream_t stream)
{
    if (W.n <= 0)
        return cudaSuccess;
    if (!M.leaper)
        return cudaErrorInvalidValue;
    switch (worlds_per_cta) {
    case 1: return launch_fast_wpc<R, 1>(M, W, A, spill, spill_per_lane, lane_cap, stream);
    case 2: return launch_fast_wpc<R, 2>(M, W, A, spill, spill_per_lane, lane_cap, stream);
    case 4: return launch_fast_wpc<R, 4>(M, W, A, spill, spill_per_lane, lane_cap, stream);
    case 8: return launch_fast_wpc<R, 8>(M, W, A, spill, spill_per_lane, lane_cap, stream);
    case 16: return launch_fast_wpc<R, 16>(M, W, A, spill, spill_per_lane, lane_cap, stream);
    case 32: return launch_fast_wpc<R, 32>(M, W, A, spill, spill_per_lane, lane_cap, stream);
    case 64: return launch_fast_wpc<R, 64>(M, W, A, spill, spill_per_lane, lane_cap, stream);
    default: return cudaErrorInvalidValue;
    }
}

template cudaError_t launch_step_fast<float>(const DevModel<float>&, const Worlds<float>&, const Actuation&, float*,
                                             int, int, int, cudaStream_t);
template cudaError_t launch_step_fast<double>(const DevModel<double>&, const Worlds<double>&, const Actuation&,
                                              double*, int, int, int, cudaStream_t);
template size_t fast_smem_bytes<float>(int, int);
template size_t fast_smem_bytes<double>(int, int);

}  // namespace arc
