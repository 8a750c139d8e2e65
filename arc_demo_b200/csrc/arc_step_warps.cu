// arc_step_warps.cu - the warp-per-leg step kernel (FP32).
//
// A CTA of four warps steps 32 worlds: lane j of warp k is leg k of world j.
// The joint solves follow the same six-slot wavefront as the leg-parallel
// kernel (warp k runs joint 3k+(s-k) at slot s; see arc_step_fast.cu for why
// that is the reference's Gauss-Seidel order, csrc/arc_phys.c:729-735), but
// now a whole warp is either working or waiting at the slot barrier: waiting
// warps issue nothing and the scheduler fills their slots with other CTAs.
// Every lane of an active warp runs the same joint, so each joint is solved
// by code specialised for its bodies: joint 3k couples the torso and the
// coxa, both with equal principal moments, whose world inverse inertia is
// d*I (csrc/arc_phys.c:70-75); joint 3k+1 the coxa and the femur; joint 3k+2
// the femur and the tibia. The specialised arithmetic equals the general
// 3x3 arithmetic on a diagonal matrix term by term (the skipped products
// are exact zeros).
//
// State placement: each lane keeps its leg's three body poses (x, q, the
// rotation and world inverse inertia) in registers; velocities, previous
// poses and sphere anchors of its leg in shared memory ([field][lane],
// conflict-free); the torso of each world in shared memory, written only by
// the warp whose slot owns it.
#include "arc_kernels.cuh"

namespace arc {
namespace wl {

constexpr int kWarps = 4;            // one per leg
constexpr int kWorlds = 32;          // one per lane
constexpr int kThreads = kWarps * kWorlds;
constexpr int kOnChip = kFastOnChipContacts;

using F = float;
using V = V3<F>;
using Q = Q4<F>;

// world inverse inertia: d*I for a body with equal moments, else symmetric
template <bool ISO> struct Iw;
template <> struct Iw<true> {
    F d;
    __device__ __forceinline__ V mul(V v) const { return V{v.x * d, v.y * d, v.z * d}; }
    __device__ __forceinline__ void sync(const M3<F>&, const BodyK<F>& k) { d = k.inv_inertia.x; }
    __device__ __forceinline__ void add_to(S3<F>& K) const
    {
        K.xx += d;
        K.yy += d;
        K.zz += d;
    }
    // csrc/arc_phys.c:284-300 with a = d*I
    __device__ __forceinline__ void add_point_mass(S3<F>& K, F inv_mass, V r) const
    {
        const F x = r.x, y = r.y, z = r.z;
        K.xx += inv_mass + d * z * z + d * y * y;
        K.yy += inv_mass + d * x * x + d * z * z;
        K.zz += inv_mass + d * y * y + d * x * x;
        K.xy += -(d * x * y);
        K.xz += -(d * x * z);
        K.yz += -(d * y * z);
    }
    __device__ __forceinline__ S3<F> s3() const { return S3<F>{d, F(0), F(0), d, F(0), d}; }
};
template <> struct Iw<false> {
    S3<F> m;
    __device__ __forceinline__ V mul(V v) const { return arc::mul(m, v); }
    __device__ __forceinline__ void sync(const M3<F>& r, const BodyK<F>& k)
    {
        // the anisotropic branch of body_sync (csrc/arc_phys.c:76-81)
        const V d = k.inv_inertia;
        V r0{r.m[0][0] * d.x, r.m[0][1] * d.y, r.m[0][2] * d.z};
        V r1{r.m[1][0] * d.x, r.m[1][1] * d.y, r.m[1][2] * d.z};
        V r2{r.m[2][0] * d.x, r.m[2][1] * d.y, r.m[2][2] * d.z};
        m.xx = r0.x * r.m[0][0] + r0.y * r.m[0][1] + r0.z * r.m[0][2];
        m.xy = r0.x * r.m[1][0] + r0.y * r.m[1][1] + r0.z * r.m[1][2];
        m.xz = r0.x * r.m[2][0] + r0.y * r.m[2][1] + r0.z * r.m[2][2];
        m.yy = r1.x * r.m[1][0] + r1.y * r.m[1][1] + r1.z * r.m[1][2];
        m.yz = r1.x * r.m[2][0] + r1.y * r.m[2][1] + r1.z * r.m[2][2];
        m.zz = r2.x * r.m[2][0] + r2.y * r.m[2][1] + r2.z * r.m[2][2];
    }
    __device__ __forceinline__ void add_to(S3<F>& K) const
    {
        K.xx += m.xx; K.xy += m.xy; K.xz += m.xz;
        K.yy += m.yy; K.yz += m.yz; K.zz += m.zz;
    }
    __device__ __forceinline__ void add_point_mass(S3<F>& K, F inv_mass, V r) const
    {
        arc::add_point_mass(K, m, inv_mass, r);
    }
    __device__ __forceinline__ S3<F> s3() const { return m; }
};

template <bool ISO> struct Body {
    V x;
    Q q;
    M3<F> rot;
    Iw<ISO> iw;
    __device__ __forceinline__ void sync(const BodyK<F>& k)
    {
        rot = m3_from_quat(q);
        iw.sync(rot, k);
    }
};

// ---------------------------------------------------------------------------
// solver primitives on specialised bodies (csrc/arc_phys.c:182-371)

template <bool I> __device__ __forceinline__ F w_pos(const Body<I>& b, const BodyK<F>& k, V r, V n)
{
    V rn = cross(r, n);
    return k.inv_mass + dot(rn, b.iw.mul(rn));
}

template <bool I> __device__ __forceinline__ void pos_impulse(Body<I>& b, const BodyK<F>& k, V r, V p)
{
    b.x = madd(b.x, p, k.inv_mass);
    b.q = q_turn(b.q, b.iw.mul(cross(r, p)));
    b.sync(k);
}

template <bool I> __device__ __forceinline__ void rot_impulse(Body<I>& b, const BodyK<F>& k, V p)
{
    b.q = q_turn(b.q, b.iw.mul(p));
    b.sync(k);
}

template <bool I> __device__ __forceinline__ F solve_pos_static(Body<I>& b, const BodyK<F>& k, V r, V d)
{
    F c = len(d);
    if (c < F(1e-12))
        return F(0);
    V n = scale(d, F(1) / c);
    F denom = w_pos(b, k, r, n);
    if (denom <= F(0))
        return F(0);
    F dl = c / denom;
    pos_impulse(b, k, r, scale(n, dl));
    return dl;
}

template <bool IP, bool IC>
__device__ __forceinline__ void solve_point(Body<IP>& b1, const BodyK<F>& k1, V r1, Body<IC>& b2, const BodyK<F>& k2,
                                            V r2, V d)
{
    if (len2(d) < F(1e-24))
        return;
    S3<F> K{F(0), F(0), F(0), F(0), F(0), F(0)};
    b1.iw.add_point_mass(K, k1.inv_mass, r1);
    b2.iw.add_point_mass(K, k2.inv_mass, r2);
    V p;
    if (!solve3_sym(K, d, p))
        return;
    pos_impulse(b1, k1, r1, p);
    pos_impulse(b2, k2, r2, -p);
}

template <bool IP, bool IC>
__device__ __forceinline__ void solve_rot_block(Body<IP>& b1, const BodyK<F>& k1, Body<IC>& b2, const BodyK<F>& k2,
                                                V rot)
{
    if (len2(rot) < F(1e-24))
        return;
    S3<F> K{F(0), F(0), F(0), F(0), F(0), F(0)};
    b1.iw.add_to(K);
    b2.iw.add_to(K);
    V p;
    if (!solve3_sym(K, rot, p))
        return;
    rot_impulse(b1, k1, p);
    rot_impulse(b2, k2, -p);
}

template <bool IP, bool IC>
__device__ __forceinline__ V solve_rot(Body<IP>& b1, const BodyK<F>& k1, Body<IC>& b2, const BodyK<F>& k2, V rot,
                                       F alpha_hh, F max_dl)
{
    F theta = len(rot);
    if (theta < F(1e-12))
        return V{F(0), F(0), F(0)};
    V n = scale(rot, F(1) / theta);
    F denom = dot(n, b1.iw.mul(n)) + dot(n, b2.iw.mul(n)) + alpha_hh;
    if (denom <= F(0))
        return V{F(0), F(0), F(0)};
    F dl = theta / denom;
    if (dl > max_dl)
        dl = max_dl;
    V p = scale(n, dl);
    rot_impulse(b1, k1, p);
    rot_impulse(b2, k2, -p);
    return p;
}

// csrc/arc_phys.c:413-457 for a joint with a parent body
template <bool IP, bool IC>
__device__ __forceinline__ void joint_positions(Body<IP>& bp, const BodyK<F>& kp, Body<IC>& bc, const BodyK<F>& kc,
                                                const JointK<F>& j, F target, F& torque_acc, F hh)
{
    V a1;
    F s, c;
    if (j.kp > F(0)) {
        a1 = mul(bp.rot, j.a1);
        V b1 = mul(bp.rot, j.b1), b2 = mul(bc.rot, j.b2);
        s = dot(cross(b1, b2), a1);
        c = dot(b1, b2);
        F phi = r_atan2(s, c);
        V p = solve_rot(bp, kp, bc, kc, scale(a1, phi - target), j.alpha_hh, j.max_dl);
        torque_acc -= dot(p, a1) / hh;
    }
    if (j.lo <= j.hi) {
        a1 = mul(bp.rot, j.a1);
        V b1 = mul(bp.rot, j.b1), b2 = mul(bc.rot, j.b2);
        s = dot(cross(b1, b2), a1);
        c = dot(b1, b2);
        if (j.hi - j.lo > F(kPi) || s * j.lim[0] - c * j.lim[1] < F(0) || j.lim[3] * c - j.lim[2] * s < F(0)) {
            F phi = r_atan2(s, c);
            if (phi < j.lo)
                solve_rot_block(bp, kp, bc, kc, scale(a1, phi - j.lo));
            else if (phi > j.hi)
                solve_rot_block(bp, kp, bc, kc, scale(a1, phi - j.hi));
        }
    }
    a1 = mul(bp.rot, j.a1);
    solve_rot_block(bp, kp, bc, kc, cross(a1, mul(bc.rot, j.a2)));
    V r1 = mul(bp.rot, j.r1);
    V r2 = mul(bc.rot, j.r2);
    solve_point(bp, kp, r1, bc, kc, r2, (bc.x + r2) - (bp.x + r1));
}

// csrc/arc_phys.c:459-481
template <bool IP, bool IC>
__device__ __forceinline__ void joint_velocities(const Body<IP>& bp, V& wp, const Body<IC>& bc, V& wc,
                                                 const JointK<F>& j, F h, F& torque_acc)
{
    if (j.kd <= F(0))
        return;
    V a = mul(bp.rot, j.a1);
    F rel = dot(wc - wp, a);
    F wsum = dot(a, bp.iw.mul(a)) + dot(a, bc.iw.mul(a));
    if (wsum <= F(0))
        return;
    F impulse = -j.kd * rel * h;
    F cap = r_min(r_fabs(rel) / wsum, j.max_th);
    impulse = r_clamp(impulse, -cap, cap);
    wp = wp - bp.iw.mul(scale(a, impulse));
    wc = wc + bc.iw.mul(scale(a, impulse));
    torque_acc += impulse / h;
}

// csrc/arc_phys.c:658-672 for one body; xp/qp receive the substep-start pose
template <bool I>
__device__ __forceinline__ void integrate(Body<I>& b, V& v, V& w, V& xp, Q& qp, const BodyK<F>& k, const StepK<F>& s)
{
    xp = b.x;
    qp = b.q;
    v = madd(v, s.gravity, s.h);
    b.x = madd(b.x, v, s.h);
    if (!I)
        w = mul(b.rot, gyroscopic(k, tmul(b.rot, w), s.h));
    b.q = q_turn(b.q, scale(w, s.h));
    b.sync(k);
}

// csrc/arc_phys.c:512-539
template <bool I>
__device__ __forceinline__ void friction(Body<I>& b, const BodyK<F>& k, V xprev, Q qprev, const SphereK<F>& sk,
                                         SphereState<F>& ss, V n, F ln, const StepK<F>& st)
{
    V c = b.x + mul(b.rot, sk.pos);
    V p = madd(c, n, -sk.radius);
    F frac = F(1);
    if (!ss.anchored || dot(n, ss.anchor_n) < F(0.9)) {
        V c0 = xprev + qrotate(qprev, sk.pos);
        ss.anchor = madd(c0, n, -sk.radius);
        ss.anchor_n = n;
        ss.anchored = 1;
    }
    V e = p - ss.anchor;
    e = madd(e, n, -dot(e, n));
    F l = len(e);
    if (l < F(1e-12))
        return;
    V r = p - b.x;
    F wt = w_pos(b, k, r, scale(e, F(1) / l));
    F lt = l / wt;
    if (lt > st.mu_s * ln) {
        frac = r_min(st.mu_d * ln / lt, F(1));
        ss.anchor = madd(ss.anchor, e, F(1) - frac);
    }
    solve_pos_static(b, k, r, scale(e, -frac));
}

// csrc/arc_phys.c:542-610; record(local, n) receives each contact
template <bool I, class Rec>
__device__ __forceinline__ int collide(Body<I>& b, const BodyK<F>& k, V xprev, Q qprev, const SphereK<F>& sk,
                                       SphereState<F>& ss, const TerrainView<F>& t, const StepK<F>& st, Rec&& record)
{
    F rad = sk.radius, ln = F(0);
    V c = b.x + mul(b.rot, sk.pos), n_max{F(0), F(0), F(1)};
    F depth_max = F(0);
    int touched = 0;
    if (!(r_fabs(c.x) < F(1e6) && r_fabs(c.y) < F(1e6))) {
        ss.anchored = 0;
        return 0;
    }
    const int ix0 = (int)r_floor((c.x - rad - t.ox) / t.cell);
    const int ix1 = (int)r_floor((c.x + rad - t.ox) / t.cell);
    const int iy0 = (int)r_floor((c.y - rad - t.oy) / t.cell);
    const int iy1 = (int)r_floor((c.y + rad - t.oy) / t.cell);
    for (int iy = iy0; iy <= iy1; ++iy) {
        for (int ix = ix0; ix <= ix1; ++ix) {
            F top = terrain_cell(t, ix, iy);
            if (c.z - rad >= top)
                continue;
            F x0 = t.ox + F(ix) * t.cell, x1 = x0 + t.cell;
            F y0 = t.oy + F(iy) * t.cell, y1 = y0 + t.cell;
            int sx = c.x > x1 ? 1 : (c.x < x0 ? -1 : 0);
            int sy = c.y > y1 ? 1 : (c.y < y0 ? -1 : 0);
            if (sx && terrain_cell(t, ix + sx, iy) >= top)
                continue;
            if (sy && terrain_cell(t, ix, iy + sy) >= top)
                continue;
            if (sx && sy && terrain_cell(t, ix + sx, iy + sy) >= top)
                continue;
            V q{r_clamp(c.x, x0, x1), r_clamp(c.y, y0, y1), r_min(c.z, top)};
            V diff = c - q;
            F dist = len(diff), depth;
            V n;
            if (dist > F(1e-9)) {
                if (dist >= rad)
                    continue;
                n = scale(diff, F(1) / dist);
                depth = rad - dist;
            } else {
                n = V{F(0), F(0), F(1)};
                depth = top - c.z + rad;
            }
            V r = madd(c, n, -rad) - b.x;
            ln += solve_pos_static(b, k, r, scale(n, depth));
            record(tmul(b.rot, r), n);
            c = b.x + mul(b.rot, sk.pos);
            if (depth > depth_max) {
                depth_max = depth;
                n_max = n;
            }
            touched = 1;
        }
    }
    if (touched)
        friction(b, k, xprev, qprev, sk, ss, n_max, ln, st);
    else
        ss.anchored = 0;
    return touched;
}

// ---------------------------------------------------------------------------
// shared memory

constexpr int kTorso = 29;  // x3 q4 v3 w3 xp3 qp4 rot9 of each world's torso
// per lane (leg k of world j): v3 w3 xp3 qp4 of coxa, femur, tibia (39), anchors of
// its 5 spheres (30), and for warp 0 the torso sphere's anchor (6)
constexpr int kCold = 39 + 30 + 6;
constexpr int kCon = kOnChip * 7;  // on-chip contacts: local3 n3 body

struct Smem {
    BodyK<F> body[13];
    JointK<F> joint[12];
    SphereK<F> sphere[21];
    F torso[kTorso][kWorlds];
    F cold[kCold][kThreads];
    F con[kCon][kThreads];
    int nc[2][kWarps][kWorlds];
    int bad[kWarps][kWorlds];
};

// torso pose in shared memory of world j
__device__ __forceinline__ void load_torso(const Smem& sm, int j, Body<true>& b)
{
    b.x = V{sm.torso[0][j], sm.torso[1][j], sm.torso[2][j]};
    b.q = Q{sm.torso[3][j], sm.torso[4][j], sm.torso[5][j], sm.torso[6][j]};
#pragma unroll
    for (int a = 0; a < 9; ++a)
        (&b.rot.m[0][0])[a] = sm.torso[20 + a][j];
    b.iw.d = sm.body[0].inv_inertia.x;
}
__device__ __forceinline__ void store_torso(Smem& sm, int j, const Body<true>& b)
{
    sm.torso[0][j] = b.x.x; sm.torso[1][j] = b.x.y; sm.torso[2][j] = b.x.z;
    sm.torso[3][j] = b.q.w; sm.torso[4][j] = b.q.x; sm.torso[5][j] = b.q.y; sm.torso[6][j] = b.q.z;
#pragma unroll
    for (int a = 0; a < 9; ++a)
        sm.torso[20 + a][j] = (&b.rot.m[0][0])[a];
}
__device__ __forceinline__ V tget(const Smem& sm, int f, int j) { return V{sm.torso[f][j], sm.torso[f + 1][j], sm.torso[f + 2][j]}; }
__device__ __forceinline__ void tset(Smem& sm, int f, int j, V v)
{
    sm.torso[f][j] = v.x;
    sm.torso[f + 1][j] = v.y;
    sm.torso[f + 2][j] = v.z;
}
__device__ __forceinline__ V cget(const Smem& sm, int f, int t) { return V{sm.cold[f][t], sm.cold[f + 1][t], sm.cold[f + 2][t]}; }
__device__ __forceinline__ void cset(Smem& sm, int f, int t, V v)
{
    sm.cold[f][t] = v.x;
    sm.cold[f + 1][t] = v.y;
    sm.cold[f + 2][t] = v.z;
}
__device__ __forceinline__ Q cgetq(const Smem& sm, int f, int t)
{
    return Q{sm.cold[f][t], sm.cold[f + 1][t], sm.cold[f + 2][t], sm.cold[f + 3][t]};
}
__device__ __forceinline__ void csetq(Smem& sm, int f, int t, Q q)
{
    sm.cold[f][t] = q.w;
    sm.cold[f + 1][t] = q.x;
    sm.cold[f + 2][t] = q.y;
    sm.cold[f + 3][t] = q.z;
}
// cold-field offsets of leg body i (0 coxa, 1 femur, 2 tibia): v, w, xp, qp
__host__ __device__ constexpr int cv(int i) { return 13 * i; }
__host__ __device__ constexpr int cw(int i) { return 13 * i + 3; }
__host__ __device__ constexpr int cxp(int i) { return 13 * i + 6; }
__host__ __device__ constexpr int cqp(int i) { return 13 * i + 9; }
__host__ __device__ constexpr int canch(int s) { return 39 + 6 * s; }  // leg sphere s = 0..4, torso sphere 5

// named barriers between two warps (ids 1..8; 0 is __syncthreads). The
// producer's arrive orders its earlier shared-memory writes before the
// consumer's sync returns.
__device__ __forceinline__ void bar_arrive(int id) { asm volatile("bar.arrive %0, 64;" ::"r"(id) : "memory"); }
__device__ __forceinline__ void bar_sync(int id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }

// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kThreads, 3)
k_step_warps(const __grid_constant__ DevModel<F> M, Worlds<F> W, Actuation A, F* __restrict__ spill, int spill_per_lane,
             int lane_cap)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
    const int tid = threadIdx.x, leg = tid / kWorlds, j = tid % kWorlds;
    const int world = blockIdx.x * kWorlds + j;
    const bool valid = world < W.n;
    const int wi = valid ? world : 0;

    for (int k = tid; k < 13; k += kThreads)
        sm.body[k] = M.body[k];
    for (int k = tid; k < 12; k += kThreads)
        sm.joint[k] = M.joint[k];
    for (int k = tid; k < 21; k += kThreads)
        sm.sphere[k] = M.sphere[k];

    F* rec = W.rec + (size_t)wi * W.stride;
    F* sr = rec + W.off_sphere;
    F* jr = rec + W.off_joint;
    const int b_c = 1 + 3 * leg, b_f = 2 + 3 * leg, b_t = 3 + 3 * leg;  // coxa, femur, tibia
    const int j0 = 3 * leg;
    // actuation (csrc/arc_sim.c:132-136) and the leg's state
    F target[3], tacc[3] = {F(0), F(0), F(0)};
    if (valid) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            target[c] = actuate(M, A, world, j0 + c);
            jr[(j0 + c) * kJointRec] = target[c];
        }
    }
    const bool active = valid && W.unstable[wi] == 0;
    Body<true> co;
    Body<false> fe, ti;
    auto load_body = [&](int b, V& x, Q& q) {
        const F* r = rec + b * kBodyRec;
        x = V{r[0], r[1], r[2]};
        q = Q{r[3], r[4], r[5], r[6]};
        cset(sm, cv(b == b_c ? 0 : (b == b_f ? 1 : 2)), tid, V{r[7], r[8], r[9]});
        cset(sm, cw(b == b_c ? 0 : (b == b_f ? 1 : 2)), tid, V{r[10], r[11], r[12]});
    };
    load_body(b_c, co.x, co.q);
    load_body(b_f, fe.x, fe.q);
    load_body(b_t, ti.x, ti.q);
    uint32_t anch = 0;
    const uint32_t* sphr = W.sph + (size_t)wi * 21;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const F* a = sr + (5 * leg + 1 + s) * kSphereRec;
#pragma unroll
        for (int c = 0; c < 6; ++c)
            sm.cold[canch(s) + c][tid] = a[c];
        anch |= ((sphr[5 * leg + 1 + s] >> 16) & 1u) << s;
    }
    if (leg == 0) {
        const F* r = rec;  // torso, body 0
        for (int f = 0; f < 13; ++f)
            sm.torso[f][j] = r[f];
#pragma unroll
        for (int c = 0; c < 6; ++c)
            sm.cold[canch(5) + c][tid] = sr[c];
        anch |= ((sphr[0] >> 16) & 1u) << 5;
    }
    const TerrainView<F> T = terrain_of(W, wi);
    const StepK<F>& st = M.step;
    const BodyK<F>& K0 = M.body[0];
    __syncthreads();
    const BodyK<F> Kc = sm.body[b_c], Kf = sm.body[b_f], Kt = sm.body[b_t];

    // csrc/arc_phys.c:713-714
    if (active) {
        co.sync(Kc);
        fe.sync(Kf);
        ti.sync(Kt);
        if (leg == 0) {
            Body<true> to;
            to.q = Q{sm.torso[3][j], sm.torso[4][j], sm.torso[5][j], sm.torso[6][j]};
            to.sync(K0);
#pragma unroll
            for (int a = 0; a < 9; ++a)
                sm.torso[20 + a][j] = (&to.rot.m[0][0])[a];
        }
    }
    unsigned long long touches = 0;
    __syncthreads();

    // Only joint 3k of each leg touches a body another warp owns (the torso),
    // so the wavefront needs no CTA-wide barrier: warp k waits for warp k-1
    // to finish its torso joint (named barrier k, producer arrives, consumer
    // syncs), and warp 0 waits for warp 3 before the torso's own sphere and
    // contact velocities. Each barrier is re-armed only after its consumer
    // passed it: the arrivals form one ring per substep.
    // Contact lists can exceed the reference's cap of kMaxContacts only when
    // four lane lists can; then the leg-major prefix needs every count.
    const bool capped = kWarps * lane_cap > kMaxContacts;
    const int pos_wait = leg == 0 ? kWarps : leg, pos_done = leg + 1;  // barrier ids 1..4
    const int vel_wait = pos_wait + kWarps, vel_done = pos_done + kWarps;  // 5..8
    for (int sub = 0; sub < M.substeps; ++sub) {
        // integrate (csrc/arc_phys.c:658-672); warp 0 starts the wavefront,
        // so it integrates its femur and tibia after handing the torso on
        auto integrate_ft = [&]() {
            V v = cget(sm, cv(1), tid), w = cget(sm, cw(1), tid), xp;
            Q qp;
            integrate(fe, v, w, xp, qp, Kf, st);
            cset(sm, cv(1), tid, v); cset(sm, cw(1), tid, w); cset(sm, cxp(1), tid, xp); csetq(sm, cqp(1), tid, qp);
            v = cget(sm, cv(2), tid); w = cget(sm, cw(2), tid);
            integrate(ti, v, w, xp, qp, Kt, st);
            cset(sm, cv(2), tid, v); cset(sm, cw(2), tid, w); cset(sm, cxp(2), tid, xp); csetq(sm, cqp(2), tid, qp);
        };
        if (active) {
            V v, w, xp;
            Q qp;
            v = cget(sm, cv(0), tid); w = cget(sm, cw(0), tid);
            integrate(co, v, w, xp, qp, Kc, st);
            cset(sm, cv(0), tid, v); cset(sm, cw(0), tid, w); cset(sm, cxp(0), tid, xp); csetq(sm, cqp(0), tid, qp);
            if (leg == 0) {
                Body<true> to;
                load_torso(sm, j, to);
                V tv = tget(sm, 7, j), tw = tget(sm, 10, j), txp;
                Q tqp;
                integrate(to, tv, tw, txp, tqp, K0, st);
                store_torso(sm, j, to);
                tset(sm, 7, j, tv);
                tset(sm, 10, j, tw);
                tset(sm, 13, j, txp);
                sm.torso[16][j] = tqp.w; sm.torso[17][j] = tqp.x; sm.torso[18][j] = tqp.y; sm.torso[19][j] = tqp.z;
            }
        }
#pragma unroll 1
        for (int part = 0; part < 2; ++part) {
            if (part == (leg == 0 ? 1 : 0) && active)
                integrate_ft();
            if (part == 0) {
                // joint 3*leg: torso -> coxa (csrc/arc_phys.c:729-730)
                if (leg != 0)
                    bar_sync(pos_wait);
                if (active) {
                    Body<true> to;
                    load_torso(sm, j, to);
                    joint_positions(to, K0, co, Kc, sm.joint[j0], target[0], tacc[0], st.hh);
                    store_torso(sm, j, to);
                }
                bar_arrive(pos_done);
            }
        }
        if (active) {
            joint_positions(co, Kc, fe, Kf, sm.joint[j0 + 1], target[1], tacc[1], st.hh);
            joint_positions(fe, Kf, ti, Kt, sm.joint[j0 + 2], target[2], tacc[2], st.hh);
        }

        // sphere contacts (csrc/arc_phys.c:731-732) and velocities from
        // positions (csrc/arc_phys.c:674-687). The torso's sphere waits for
        // the last torso joint; when the cap can bind it also leads warp 0's
        // list, as sphere 0 leads the reference's.
        int nc = 0;
        auto record = [&](int body, V local, V n) {
            F* dst = nullptr;
            if (nc < kOnChip) {
                sm.con[nc * 7 + 0][tid] = local.x; sm.con[nc * 7 + 1][tid] = local.y; sm.con[nc * 7 + 2][tid] = local.z;
                sm.con[nc * 7 + 3][tid] = n.x; sm.con[nc * 7 + 4][tid] = n.y; sm.con[nc * 7 + 5][tid] = n.z;
                sm.con[nc * 7 + 6][tid] = (F)body;
            } else if (nc < lane_cap) {
                dst = spill + (((size_t)wi * kWarps + leg) * (size_t)spill_per_lane + (nc - kOnChip)) * 8;
                dst[0] = local.x; dst[1] = local.y; dst[2] = local.z;
                dst[3] = n.x; dst[4] = n.y; dst[5] = n.z;
                dst[6] = (F)body;
            }
            ++nc;
        };
#pragma unroll 1
        for (int part = 0; part < 2; ++part) {
            if ((part == 0) == capped) {
                if (leg != 0)
                    continue;
                bar_sync(pos_wait);
                if (!active)
                    continue;
                Body<true> to;
                load_torso(sm, j, to);
                SphereState<F> ss{cget(sm, canch(5), tid), cget(sm, canch(5) + 3, tid), (int)((anch >> 5) & 1u)};
                const V txp = tget(sm, 13, j);
                const Q tqp{sm.torso[16][j], sm.torso[17][j], sm.torso[18][j], sm.torso[19][j]};
                const int t = collide(to, K0, txp, tqp, sm.sphere[0], ss, T, st, [&](V l, V n) { record(0, l, n); });
                touches += (unsigned long long)t << 50;
                anch = (anch & ~(1u << 5)) | ((uint32_t)(ss.anchored != 0) << 5);
                cset(sm, canch(5), tid, ss.anchor);
                cset(sm, canch(5) + 3, tid, ss.anchor_n);
                V v, w;
                update_velocity(to.q, to.x, v, w, txp, tqp, st);
                store_torso(sm, j, to);
                tset(sm, 7, j, v);
                tset(sm, 10, j, w);
                continue;
            }
            if (!active)
                continue;
            {
                const int s = 5 * leg + 1;
                SphereState<F> ss{cget(sm, canch(0), tid), cget(sm, canch(0) + 3, tid), (int)(anch & 1u)};
                const int t = collide(fe, Kf, cget(sm, cxp(1), tid), cgetq(sm, cqp(1), tid), sm.sphere[s], ss, T, st,
                                      [&](V l, V n) { record(b_f, l, n); });
                touches += (unsigned long long)t;
                anch = (anch & ~1u) | (uint32_t)(ss.anchored != 0);
                cset(sm, canch(0), tid, ss.anchor);
                cset(sm, canch(0) + 3, tid, ss.anchor_n);
            }
            const V txp = cget(sm, cxp(2), tid);
            const Q tqp = cgetq(sm, cqp(2), tid);
#pragma unroll 1
            for (int it = 1; it < 5; ++it) {
                const int s = 5 * leg + 1 + it;
                SphereState<F> ss{cget(sm, canch(it), tid), cget(sm, canch(it) + 3, tid), (int)((anch >> it) & 1u)};
                const int t = collide(ti, Kt, txp, tqp, sm.sphere[s], ss, T, st, [&](V l, V n) { record(b_t, l, n); });
                touches += (unsigned long long)t << (10 * it);
                anch = (anch & ~(1u << it)) | ((uint32_t)(ss.anchored != 0) << it);
                cset(sm, canch(it), tid, ss.anchor);
                cset(sm, canch(it) + 3, tid, ss.anchor_n);
            }
            V v, w;
            update_velocity(co.q, co.x, v, w, cget(sm, cxp(0), tid), cgetq(sm, cqp(0), tid), st);
            cset(sm, cv(0), tid, v); cset(sm, cw(0), tid, w);
            update_velocity(fe.q, fe.x, v, w, cget(sm, cxp(1), tid), cgetq(sm, cqp(1), tid), st);
            cset(sm, cv(1), tid, v); cset(sm, cw(1), tid, w);
            update_velocity(ti.q, ti.x, v, w, cget(sm, cxp(2), tid), cgetq(sm, cqp(2), tid), st);
            cset(sm, cv(2), tid, v); cset(sm, cw(2), tid, w);
        }
        if (capped) {
            // double-buffered: a warp may record substep s+1 while another
            // still reads the counts of substep s
            sm.nc[sub & 1][leg][j] = nc;
            __syncthreads();
        }

        // drive damping, the same wavefront (csrc/arc_phys.c:700-705)
        if (leg != 0)
            bar_sync(vel_wait);
        if (active) {
            Body<true> to;
            load_torso(sm, j, to);
            V wp = tget(sm, 10, j), wc = cget(sm, cw(0), tid);
            joint_velocities(to, wp, co, wc, sm.joint[j0], st.h, tacc[0]);
            tset(sm, 10, j, wp);
            cset(sm, cw(0), tid, wc);
        }
        bar_arrive(vel_done);
        if (active) {
            V wp = cget(sm, cw(0), tid), wc = cget(sm, cw(1), tid);
            joint_velocities(co, wp, fe, wc, sm.joint[j0 + 1], st.h, tacc[1]);
            cset(sm, cw(0), tid, wp);
            wp = wc;
            wc = cget(sm, cw(2), tid);
            joint_velocities(fe, wp, ti, wc, sm.joint[j0 + 2], st.h, tacc[2]);
            cset(sm, cw(1), tid, wp);
            cset(sm, cw(2), tid, wc);
        }

        // contact velocities, in the reference's (leg-major) order under its
        // cap; the torso's after the last torso joint
        int base = 0;
        if (capped && active)
            for (int l = 0; l < leg; ++l)
                base += sm.nc[sub & 1][l][j];
        const int ncl = nc < lane_cap ? nc : lane_cap;
#pragma unroll 1
        for (int part = 0; part < 2; ++part) {
            if (part == 1) {
                if (leg != 0)
                    break;
                bar_sync(vel_wait);
            }
            if (!active)
                continue;
            for (int c = 0; c < ncl && base + c < kMaxContacts; ++c) {
                F rc[7];
                if (c < kOnChip) {
#pragma unroll
                    for (int f = 0; f < 7; ++f)
                        rc[f] = sm.con[c * 7 + f][tid];
                } else {
                    const F* src = spill + (((size_t)wi * kWarps + leg) * (size_t)spill_per_lane + (c - kOnChip)) * 8;
#pragma unroll
                    for (int f = 0; f < 7; ++f)
                        rc[f] = src[f];
                }
                const int b = (int)rc[6];
                if ((b == 0) != (part == 1))
                    continue;
                const ContactRec<F> cr{V{rc[0], rc[1], rc[2]}, V{rc[3], rc[4], rc[5]}};
                if (b == 0) {
                    V v = tget(sm, 7, j), w = tget(sm, 10, j);
                    Body<true> to;
                    load_torso(sm, j, to);
                    contact_velocity(to.rot, to.iw.s3(), K0.inv_mass, v, w, cr);
                    tset(sm, 7, j, v);
                    tset(sm, 10, j, w);
                } else if (b == b_f) {
                    V v = cget(sm, cv(1), tid), w = cget(sm, cw(1), tid);
                    contact_velocity(fe.rot, fe.iw.m, Kf.inv_mass, v, w, cr);
                    cset(sm, cv(1), tid, v);
                    cset(sm, cw(1), tid, w);
                } else {
                    V v = cget(sm, cv(2), tid), w = cget(sm, cw(2), tid);
                    contact_velocity(ti.rot, ti.iw.m, Kt.inv_mass, v, w, cr);
                    cset(sm, cv(2), tid, v);
                    cset(sm, cw(2), tid, w);
                }
            }
        }
    }
    __syncthreads();

    // epilogue (csrc/arc_phys.c:739-746)
    int bad = 0;
    if (active) {
        const Q tq{sm.torso[3][j], sm.torso[4][j], sm.torso[5][j], sm.torso[6][j]};
        const V tw = tget(sm, 10, j);
        const V wc0 = cget(sm, cw(0), tid), wc1 = cget(sm, cw(1), tid), wc2 = cget(sm, cw(2), tid);
        const JointK<F>& J0 = sm.joint[j0];
        const JointK<F>& J1 = sm.joint[j0 + 1];
        const JointK<F>& J2 = sm.joint[j0 + 2];
        jr[(j0 + 0) * kJointRec + 1] = joint_angle(tq, co.q, J0);
        jr[(j0 + 0) * kJointRec + 2] = joint_rate(tq, tw, wc0, J0);
        jr[(j0 + 1) * kJointRec + 1] = joint_angle(co.q, fe.q, J1);
        jr[(j0 + 1) * kJointRec + 2] = joint_rate(co.q, wc0, wc1, J1);
        jr[(j0 + 2) * kJointRec + 1] = joint_angle(fe.q, ti.q, J2);
        jr[(j0 + 2) * kJointRec + 2] = joint_rate(fe.q, wc1, wc2, J2);
#pragma unroll
        for (int c = 0; c < 3; ++c)
            jr[(j0 + c) * kJointRec + 3] = tacc[c] / F(M.substeps);
        bad |= body_unstable(co.x, cget(sm, cv(0), tid), wc0);
        bad |= body_unstable(fe.x, cget(sm, cv(1), tid), wc1);
        bad |= body_unstable(ti.x, cget(sm, cv(2), tid), wc2);
        if (leg == 0)
            bad |= body_unstable(tget(sm, 0, j), tget(sm, 7, j), tw);
        // write back the leg's bodies and spheres
        auto put = [&](int b, V x, Q q, V v, V w) {
            F* r = rec + b * kBodyRec;
            r[0] = x.x; r[1] = x.y; r[2] = x.z;
            r[3] = q.w; r[4] = q.x; r[5] = q.y; r[6] = q.z;
            r[7] = v.x; r[8] = v.y; r[9] = v.z;
            r[10] = w.x; r[11] = w.y; r[12] = w.z;
        };
        put(b_c, co.x, co.q, cget(sm, cv(0), tid), wc0);
        put(b_f, fe.x, fe.q, cget(sm, cv(1), tid), wc1);
        put(b_t, ti.x, ti.q, cget(sm, cv(2), tid), wc2);
        uint32_t* sphw = W.sph + (size_t)world * 21;
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            F* a = sr + (5 * leg + 1 + s) * kSphereRec;
#pragma unroll
            for (int c = 0; c < 6; ++c)
                a[c] = sm.cold[canch(s) + c][tid];
            sphw[5 * leg + 1 + s] = (uint32_t)((touches >> (10 * s)) & 1023u) | (((anch >> s) & 1u) << 16);
        }
        if (leg == 0) {
            for (int f = 0; f < 13; ++f)
                rec[f] = sm.torso[f][j];
#pragma unroll
            for (int c = 0; c < 6; ++c)
                sr[c] = sm.cold[canch(5) + c][tid];
            sphw[0] = (uint32_t)((touches >> 50) & 1023u) | (((anch >> 5) & 1u) << 16);
        }
    }
    sm.bad[leg][j] = bad;
    __syncthreads();
    if (active && leg == 0) {
        W.time[world] += M.step_dt;
        if (sm.bad[0][j] | sm.bad[1][j] | sm.bad[2][j] | sm.bad[3][j])
            W.unstable[world] = 1;
    }
}

}  // namespace wl

size_t warps_smem_bytes() { return sizeof(wl::Smem); }

cudaError_t launch_step_warps(const DevModel<float>& M, const Worlds<float>& W, const Actuation& A, float* spill,
                              int spill_per_lane, int lane_cap, cudaStream_t stream)
{
    if (W.n <= 0)
        return cudaSuccess;
    if (!M.leaper)
        return cudaErrorInvalidValue;
    static bool configured = false;
    const int smem = (int)sizeof(wl::Smem);
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(wl::k_step_warps, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             smem > 48 * 1024 ? smem : 48 * 1024);
        if (e != cudaSuccess)
            return e;
        configured = true;
    }
    const int grid = (W.n + wl::kWorlds - 1) / wl::kWorlds;
    wl::k_step_warps<<<grid, wl::kThreads, smem, stream>>>(M, W, A, spill, spill_per_lane, lane_cap);
    return cudaGetLastError();
}

}  // namespace arc
