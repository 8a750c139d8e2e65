// arc_step_warps.cuh - the warp-per-leg step (FP32): one group of 32 worlds.
//
// A CTA of four warps steps 32 worlds: lane j of warp k is leg k of world j.
// The reference's Gauss-Seidel order (csrc/arc_phys.c:729-735) couples the
// legs only through the torso: joint 3k (torso -> coxa of leg k) must see
// the torso as joint 3(k-1) left it. So warp k solves its torso joint after
// warp k-1 solved its own (a named barrier between the two warps, one
// arrive and one sync), and everything else of leg k - its two other
// joints, its five spheres, its three bodies' velocities - runs without
// waiting. Warp 0 also owns the torso's own work (its integration, its
// sphere, its contact velocities), so the torso sphere's contacts lead warp
// 0's list as sphere 0 leads the reference's, and the four warps' lists in
// warp order are the reference's contact list.
//
// Code size decides this kernel's speed. With 16 warps of 4 CTAs per SM in
// different phases of the step, a kernel whose code does not fit the SM's
// instruction cache spends most cycles waiting for instructions. Every
// phase is therefore one generic routine, run by a small interpreter over a
// per-warp list of operations (integrate bodies a..b, solve joints a..b,
// collide spheres a..b, ...): one copy of each routine, whatever the body.
// The bodies live in shared memory ([field][world], conflict-free); a
// routine loads the few it works on, recomputes their rotation and world
// inverse inertia from q (the same function of q as the reference's
// body_sync, so the same values), and stores them back.
//
// Rotations the reference leaves stale: update_velocities (csrc/arc_phys.c:
// 674-687) normalises q without re-syncing, so the velocity pass and the
// next substep's gyroscopic term use the rotation of the un-normalised q of
// the position pass. Each body therefore keeps two quaternions: field Q, the
// position-pass q the rotation comes from, and field QP, the substep-start
// q (and, after the velocity update, the normalised q the next substep
// starts from).
//
// This header holds the step of one group, `step_group`, which the control
// step kernel of arc_task.cu runs in FP32, alone (the physics step) or
// followed by the task layer on the group's worlds (the fused control step),
// and arc_step_warps64.cu's kernel runs in FP64 (ARC_WARPS_FP64). Everything
// here has internal linkage: each including translation unit has its own
// copy, its operation lists in its own constant bank.
#pragma once

#include "arc_kernels.cuh"

namespace arc {
namespace wl {
namespace {

constexpr int kWarps = 4;   // one per leg
constexpr int kWorlds = 32; // one per lane
constexpr int kThreads = kWarps * kWorlds;
constexpr int kOnChip = kWarpsOnChipContacts;

// the precision of the step: FP32 (arc_task.cu's control-step kernel) or,
// where the including file defines ARC_WARPS_FP64, FP64 (arc_step_warps64.cu)
#ifdef ARC_WARPS_FP64
using F = double;
#else
using F = float;
#endif
using V = V3<F>;
using Q = Q4<F>;
using P = Pose<F>;

// body fields: x, q (position pass), v, w, x_prev, q_prev / normalised q
constexpr int kX = 0, kQ = 3, kV = 7, kW = 10, kXP = 13, kQP = 16, kBodyF = 20;
constexpr int kTorso = 3;  // body slot of the torso; 0..2: the lane's coxa, femur, tibia

// The model constants stay in the kernel's parameter space: all lanes of a
// warp read the same body, joint or sphere, a broadcast from the constant
// cache.
struct Smem {
    F leg[kWarps][3 * kBodyF][kWorlds];   // the lane's three bodies
    F anch[kWarps][5 * 6][kWorlds];       // anchor, anchor normal of the lane's five spheres
    F con[kWarps][kOnChip * 7][kWorlds];  // on-chip contact records: local3 n3 body
    F torso[kBodyF + 6][kWorlds];     // each world's torso, then its sphere's anchor
    int nc[2][kWarps][kWorlds];       // contact counts (capped lists), by substep parity
    int bad[kWarps][kWorlds];
};

// A field array in shared memory: element f at p[f * kWorlds]. Every
// per-world array has the same row length, so fields are constant offsets
// from the pointer whichever body it points at.
struct Ref {
    F* p;
    __device__ __forceinline__ F& operator[](int f) const { return p[f * kWorlds]; }
};
__device__ __forceinline__ V getv(Ref r, int f) { return V{r[f], r[f + 1], r[f + 2]}; }
__device__ __forceinline__ void setv(Ref r, int f, V v)
{
    r[f] = v.x;
    r[f + 1] = v.y;
    r[f + 2] = v.z;
}
__device__ __forceinline__ Q getq(Ref r, int f) { return Q{r[f], r[f + 1], r[f + 2], r[f + 3]}; }
__device__ __forceinline__ void setq(Ref r, int f, Q q)
{
    r[f] = q.w;
    r[f + 1] = q.x;
    r[f + 2] = q.y;
    r[f + 3] = q.z;
}
__device__ __forceinline__ void load_pose(Ref r, const BodyK<F>& k, P& b)
{
    b.x = getv(r, kX);
    b.q = getq(r, kQ);
    body_sync(b, k);
}
__device__ __forceinline__ void store_pose(Ref r, const P& b)
{
    setv(r, kX, b.x);
    setq(r, kQ, b.q);
}

// named barriers between two warps (ids 1..8; 0 is __syncthreads). The
// producer's arrive orders its earlier shared-memory writes before the
// consumer's sync returns.
__device__ __forceinline__ void bar_arrive(int id) { asm volatile("bar.arrive %0, 64;" ::"r"(id) : "memory"); }
__device__ __forceinline__ void bar_sync(int id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }

// csrc/arc_phys.c:413-457 for a joint with a parent: the drive (solve_rot,
// :353-371), the limit and the axis alignment (solve_rot_block, :328-346)
// and the attachment (solve_point, :308-320), in that order, with one site
// that applies the impulse (+p on the parent, -p on the child, :196-211).
__device__ __forceinline__ void joint_positions(P& bp, const BodyK<F>& kp, P& bc, const BodyK<F>& kc,
                                                const JointK<F>& j, F target, F& torque_acc, F hh)
{
#pragma unroll 1
    for (int stage = 0; stage < 4; ++stage) {
        const V a1 = mul(bp.rot, j.a1);
        S3<F> K{F(0), F(0), F(0), F(0), F(0), F(0)};
        V rhs{F(0), F(0), F(0)}, p{F(0), F(0), F(0)}, r1{F(0), F(0), F(0)}, r2{F(0), F(0), F(0)};
        bool positional = false;
        if (stage < 2) {
            if (stage == 0 ? !(j.kp > F(0)) : !(j.lo <= j.hi))
                continue;
            const V b1 = mul(bp.rot, j.b1), b2 = mul(bc.rot, j.b2);
            const F s = dot(cross(b1, b2), a1), c = dot(b1, b2);
            // the limit needs the angle only outside [lo, hi]
            if (stage == 1 &&
                !(j.hi - j.lo > F(kPi) || s * j.lim[0] - c * j.lim[1] < F(0) || j.lim[3] * c - j.lim[2] * s < F(0)))
                continue;
            const F phi = r_atan2(s, c);
            if (stage == 0) {
                const V rot = scale(a1, phi - target);
                const F theta = len(rot);
                if (theta < F(1e-12))
                    continue;
                const V n = scale(rot, F(1) / theta);
                const F denom = dot(n, mul(bp.iiw, n)) + dot(n, mul(bc.iiw, n)) + j.alpha_hh;
                if (denom <= F(0))
                    continue;
                F dl = theta / denom;
                if (dl > j.max_dl)
                    dl = j.max_dl;
                p = scale(n, dl);
                torque_acc -= dot(p, a1) / hh;
            } else {
                if (phi < j.lo)
                    rhs = scale(a1, phi - j.lo);
                else if (phi > j.hi)
                    rhs = scale(a1, phi - j.hi);
                else
                    continue;
            }
        } else if (stage == 2) {
            rhs = cross(a1, mul(bc.rot, j.a2));
        } else {
            r1 = mul(bp.rot, j.r1);
            r2 = mul(bc.rot, j.r2);
            rhs = (bc.x + r2) - (bp.x + r1);
            positional = true;
        }
        if (stage > 0) {
            if (len2(rhs) < F(1e-24))
                continue;
            if (positional) {
                add_point_mass(K, bp.iiw, kp.inv_mass, r1);
                add_point_mass(K, bc.iiw, kc.inv_mass, r2);
            } else {
                K.xx = bp.iiw.xx + bc.iiw.xx; K.xy = bp.iiw.xy + bc.iiw.xy; K.xz = bp.iiw.xz + bc.iiw.xz;
                K.yy = bp.iiw.yy + bc.iiw.yy; K.yz = bp.iiw.yz + bc.iiw.yz; K.zz = bp.iiw.zz + bc.iiw.zz;
            }
            if (!solve3_sym(K, rhs, p))
                continue;
        }
        const V pn = -p;
        if (positional) {
            bp.x = madd(bp.x, p, kp.inv_mass);
            bc.x = madd(bc.x, pn, kc.inv_mass);
        }
        const V tp = mul(bp.iiw, positional ? cross(r1, p) : p);
        const V tc = mul(bc.iiw, positional ? cross(r2, pn) : pn);
        bp.q = q_turn(bp.q, tp);
        bc.q = q_turn(bc.q, tc);
        if (positional)  // the last stage: the caller keeps x and q only
            break;
        body_sync(bp, kp);
        body_sync(bc, kc);
    }
}

// One sphere against the column grid (csrc/arc_phys.c:542-610) with its
// contacts (solve_contact, :488-500) and the closing friction correction
// (solve_friction, :512-539). The scan and the friction share one site of
// the positional correction against the static world (solve_pos with no
// second body and alpha = 0, :226-242). Returns 1 when the sphere touched.
template <class Rec>
__device__ __forceinline__ int collide(P& b, const BodyK<F>& k, V xprev, Q qprev, const SphereK<F>& sk,
                                       SphereState<F>& ss, const TerrainView<F>& t, F inv_cell, const StepK<F>& st,
                                       Rec&& record)
{
    const F rad = sk.radius;
    V c = b.x + mul(b.rot, sk.pos);
    // a blown-up state must not reach the int conversions
    if (!(r_fabs(c.x) < F(1e6) && r_fabs(c.y) < F(1e6))) {
        ss.anchored = 0;
        return 0;
    }
    // the columns under the sphere's box (csrc/arc_phys.c:557-560), scaled by
    // 1/cell instead of divided by cell: the two differ only when a box edge
    // lies within an ulp of a column edge, where that column's face is the
    // sphere's radius away and cannot make a contact either way
    const int ix0 = (int)r_floor(((c.x - rad) - t.ox) * inv_cell);
    const int ix1 = (int)r_floor(((c.x + rad) - t.ox) * inv_cell);
    const int iy0 = (int)r_floor(((c.y - rad) - t.oy) * inv_cell);
    const int iy1 = (int)r_floor(((c.y + rad) - t.oy) * inv_cell);
    // the heights of the box's first 2 x 2 columns, loaded together: a
    // sphere narrower than a column spans at most that many, and the
    // buried-edge test's neighbours of one of them are the others
    F h00 = F(0), h10 = F(0), h01 = F(0), h11 = F(0);
    h00 = terrain_cell(t, ix0, iy0);
    if (ix1 > ix0)
        h10 = terrain_cell(t, ix0 + 1, iy0);
    if (iy1 > iy0) {
        h01 = terrain_cell(t, ix0, iy0 + 1);
        if (ix1 > ix0)
            h11 = terrain_cell(t, ix0 + 1, iy0 + 1);
    }
    auto height = [&](int cx, int cy) {
        const int dx = cx - ix0, dy = cy - iy0;
        if (dx >= 0 && dy >= 0 && dx < 2 && dy < 2 && cx <= ix1 && cy <= iy1)
            return dy ? (dx ? h11 : h01) : (dx ? h10 : h00);
        return terrain_cell(t, cx, cy);
    };
    F ln = F(0), depth_max = F(0);
    V n_max{F(0), F(0), F(1)};
    int touched = 0, ix = ix0, iy = iy0;
#pragma unroll 1
    for (;;) {
        V r, d, n{F(0), F(0), F(1)};
        F depth = F(0);
        bool contact = false;
#pragma unroll 1
        while (!contact && iy <= iy1) {
            const int cx = ix, cy = iy;
            if (++ix > ix1) {
                ix = ix0;
                ++iy;
            }
            const F top = height(cx, cy);
            if (c.z - rad >= top)
                continue;
            const F x0 = t.ox + F(cx) * t.cell, x1 = x0 + t.cell;
            const F y0 = t.oy + F(cy) * t.cell, y1 = y0 + t.cell;
            // edges and corners buried by an equal or higher neighbour
            const int sx = c.x > x1 ? 1 : (c.x < x0 ? -1 : 0);
            const int sy = c.y > y1 ? 1 : (c.y < y0 ? -1 : 0);
            bool buried = false;
#pragma unroll 1
            for (int m = 1; m < 4 && !buried; ++m) {
                if (((m & 1) && !sx) || ((m & 2) && !sy))
                    continue;
                buried = height(cx + ((m & 1) ? sx : 0), cy + ((m & 2) ? sy : 0)) >= top;
            }
            if (buried)
                continue;
            const V q{r_clamp(c.x, x0, x1), r_clamp(c.y, y0, y1), r_min(c.z, top)};
            const V diff = c - q;
            const F dist = len(diff);
            if (dist > F(1e-9)) {
                if (dist >= rad)
                    continue;
                n = scale(diff, F(1) / dist);
                depth = rad - dist;
            } else {
                depth = top - c.z + rad;  // centre inside the column: out through the top
            }
            r = madd(c, n, -rad) - b.x;
            d = scale(n, depth);
            contact = true;
        }
        if (!contact) {
            if (!touched)
                break;
            // friction, once, after the scan; c is the current centre
            const V p = madd(c, n_max, -rad);
            if (!ss.anchored || dot(n_max, ss.anchor_n) < F(0.9)) {
                const V c0 = xprev + qrotate(qprev, sk.pos);
                ss.anchor = madd(c0, n_max, -rad);
                ss.anchor_n = n_max;
                ss.anchored = 1;
            }
            V e = p - ss.anchor;
            e = madd(e, n_max, -dot(e, n_max));
            const F l = len(e);
            if (l < F(1e-12))
                break;
            r = p - b.x;
            const F lt = l / w_pos(b, k, r, scale(e, F(1) / l));
            F frac = F(1);
            if (lt > st.mu_s * ln) {
                frac = r_min(st.mu_d * ln / lt, F(1));
                ss.anchor = madd(ss.anchor, e, F(1) - frac);
            }
            d = scale(e, -frac);
        }
        F dl = F(0);
        const F cl = len(d);
        if (cl >= F(1e-12)) {
            const V nn = scale(d, F(1) / cl);
            const F denom = w_pos(b, k, r, nn);
            if (denom > F(0)) {
                dl = cl / denom;
                pos_impulse(b, k, r, scale(nn, dl));
            }
        }
        if (!contact)
            break;  // the friction correction closes the sphere
        ln += dl;
        record(tmul(b.rot, r), n);
        c = b.x + mul(b.rot, sk.pos);
        if (depth > depth_max) {
            depth_max = depth;
            n_max = n;
        }
        touched = 1;
    }
    if (!touched)
        ss.anchored = 0;
    return touched;
}

// per-warp operation lists: kind | a << 4 | b << 8 | wait << 12 | arrive << 16
// | flags. An op with a wait first syncs on that named barrier; one with an
// arrive arrives on it when done.
enum : uint32_t { OP_END = 0, OP_INT, OP_JNT, OP_COL, OP_UPD, OP_DMP, OP_CVL, OP_CNT };
// INT/UPD a..b: body ordinals (0 torso, 1..3 coxa, femur, tibia)
// JNT/DMP a..b: the leg's joints (0 torso->coxa, 1 coxa->femur, 2 femur->tibia)
// COL a..b: sphere ordinals on one body (0 torso sphere, 1 femur, 2..5 tibia)
// CVL a: contact velocities of the leg's bodies (0) or of the torso (1)
// CNT: publish the contact count, then __syncthreads (capped lists only)
#define ARC_OP(kind, a, b, w, r) ((kind) | (a) << 4 | (b) << 8 | (w) << 12 | (r) << 16)
// Uncapped lists. Warp 0 owns the torso's own work, and each substep's
// chain of torso hand-offs starts and ends in it: it integrates the torso
// and solves joint 0 at once (no hand-off), collides the torso's sphere
// after joint 9 (barrier 4), and applies the torso's contact velocities
// after joint 9's drive damping (barrier 8), before the next substep. Warp
// k > 0 solves joint 3k after warp k-1's (barrier k) and damping joint 3k
// after warp k-1's (barrier 4+k). Each warp solves what the next hand-off
// needs first (its coxa's velocity right after joint 3k+1, the only other
// joint that moves the coxa) and the rest of its leg while the chain runs
// elsewhere; work on different bodies commutes, so this is the reference's
// order. Warp 0 runs ahead of the others in issue priority: the torso's
// work there makes the step 5% faster than the same lists with the torso
// on warp 3.
#define ARC_LEG_OPS(k)                                                                                         \
    {ARC_OP(OP_INT, 1, 4, 0, 0), ARC_OP(OP_JNT, 0, 1, k, (k) + 1), ARC_OP(OP_JNT, 1, 2, 0, 0),                  \
     ARC_OP(OP_UPD, 1, 2, 0, 0), ARC_OP(OP_DMP, 0, 1, 4 + (k), 5 + (k)), ARC_OP(OP_JNT, 2, 3, 0, 0),            \
     ARC_OP(OP_COL, 1, 2, 0, 0), ARC_OP(OP_COL, 2, 6, 0, 0), ARC_OP(OP_UPD, 2, 4, 0, 0), ARC_OP(OP_DMP, 1, 3, 0, 0), \
     ARC_OP(OP_CVL, 0, 0, 0, 0), OP_END}
// Capped lists: warp 0 owns the torso, whose sphere's contacts lead the
// list as sphere 0 leads the reference's, and every lane's count is
// published before any contact velocity.
#define ARC_CAPPED_OPS(k)                                                                                           \
    {ARC_OP(OP_INT, 1, 4, 0, 0), ARC_OP(OP_JNT, 0, 1, k, k + 1), ARC_OP(OP_JNT, 1, 3, 0, 0),                        \
     ARC_OP(OP_COL, 1, 2, 0, 0), ARC_OP(OP_COL, 2, 6, 0, 0), ARC_OP(OP_UPD, 1, 4, 0, 0), ARC_OP(OP_CNT, 0, 0, 0, 0), \
     ARC_OP(OP_DMP, 0, 1, 4 + k, 5 + k), ARC_OP(OP_DMP, 1, 3, 0, 0), ARC_OP(OP_CVL, 0, 0, 0, 0), OP_END}

constexpr int kMaxOps = 20;
__constant__ uint32_t kOps[2][kWarps][kMaxOps] = {
    {{ARC_OP(OP_INT, 0, 4, 0, 0), ARC_OP(OP_JNT, 0, 1, 0, 1), ARC_OP(OP_JNT, 1, 2, 0, 0), ARC_OP(OP_UPD, 1, 2, 0, 0),
      ARC_OP(OP_COL, 0, 1, 4, 0), ARC_OP(OP_UPD, 0, 1, 0, 0), ARC_OP(OP_DMP, 0, 1, 0, 5), ARC_OP(OP_JNT, 2, 3, 0, 0),
      ARC_OP(OP_COL, 1, 2, 0, 0), ARC_OP(OP_COL, 2, 6, 0, 0), ARC_OP(OP_UPD, 2, 4, 0, 0), ARC_OP(OP_DMP, 1, 3, 0, 0),
      ARC_OP(OP_CVL, 0, 0, 0, 0), ARC_OP(OP_CVL, 1, 0, 8, 0), OP_END},
     ARC_LEG_OPS(1), ARC_LEG_OPS(2), ARC_LEG_OPS(3)},
    {{ARC_OP(OP_INT, 0, 2, 0, 0), ARC_OP(OP_JNT, 0, 1, 0, 1), ARC_OP(OP_INT, 2, 4, 0, 0), ARC_OP(OP_JNT, 1, 3, 0, 0),
      ARC_OP(OP_COL, 0, 1, 4, 0), ARC_OP(OP_UPD, 0, 1, 0, 0), ARC_OP(OP_COL, 1, 2, 0, 0), ARC_OP(OP_COL, 2, 6, 0, 0),
      ARC_OP(OP_UPD, 1, 4, 0, 0), ARC_OP(OP_CNT, 0, 0, 0, 0), ARC_OP(OP_DMP, 0, 1, 0, 5), ARC_OP(OP_DMP, 1, 3, 0, 0),
      ARC_OP(OP_CVL, 0, 0, 0, 0), ARC_OP(OP_CVL, 1, 0, 8, 0), OP_END},
     ARC_CAPPED_OPS(1), ARC_CAPPED_OPS(2), ARC_CAPPED_OPS(3)}};
#undef ARC_LEG_OPS
#undef ARC_CAPPED_OPS
#undef ARC_OP

// ---------------------------------------------------------------------------


// One control step of the 32 worlds of group `group` (items group * 32 ..
// group * 32 + 31: worlds ids[item], or item itself without ids) by a CTA of
// kThreads threads, thread tid = lane j of warp `leg`. On return the
// worlds' records, flags, time and unstable marks are written and every
// thread of the CTA has passed the group's last barrier.
//
// Substeps sub0 .. sub1 - 1 of the control step (0 .. M.substeps - 1: the
// whole step). A control step in several such tiles, one launch each, gives
// the worlds of one launch bit for bit: between tiles the record holds the
// bodies (with the normalised q), anchors, touch counts and the summed drive
// torques, and tile_q (13 x 4 floats per world) the position-pass q whose
// rotation the next substep's gyroscopic term uses; the joint outputs, time
// and stability come at the end of the last tile.
__device__ __forceinline__ void step_group(Smem& sm, const DevModel<F>& M, const Worlds<F>& W, const Actuation& A,
                                           F* __restrict__ spill, int spill_per_lane, int lane_cap,
                                           const int* __restrict__ ids, int n_items, int group, int tid, int leg,
                                           int j, int sub0, int sub1, F* __restrict__ tile_q)
{
    (void)tid;
    const bool first_tile = sub0 == 0, last_tile = sub1 >= M.substeps;
    const int item = group * kWorlds + j;
    const int world = item < n_items ? (ids ? ids[item] : item) : -1;
    const bool valid = world >= 0 && world < W.n;
    const int wi = valid ? world : 0;

    F* rec = W.rec + (size_t)wi * W.stride;
    F* sr = rec + W.off_sphere;
    F* jr = rec + W.off_joint;
    const int b_c = 1 + 3 * leg, b_f = 2 + 3 * leg, b_t = 3 + 3 * leg;  // coxa, femur, tibia
    const int j0 = 3 * leg;
    const Ref torso{&sm.torso[0][j]};
    auto body_ref = [&](int slot) {
        return slot == kTorso ? torso : Ref{&sm.leg[leg][slot * kBodyF][j]};
    };
    // actuation (csrc/arc_sim.c:132-136)
    F target0 = F(0), target1 = F(0), target2 = F(0);
    if (valid) {
        target0 = actuate(M, A, world, j0);
        target1 = actuate(M, A, world, j0 + 1);
        target2 = actuate(M, A, world, j0 + 2);
        jr[j0 * kJointRec] = target0;
        jr[(j0 + 1) * kJointRec] = target1;
        jr[(j0 + 2) * kJointRec] = target2;
    }
    F tacc0 = F(0), tacc1 = F(0), tacc2 = F(0);
    if (!first_tile) {
        tacc0 = jr[j0 * kJointRec + 3];
        tacc1 = jr[(j0 + 1) * kJointRec + 3];
        tacc2 = jr[(j0 + 2) * kJointRec + 3];
    }
    const bool active = valid && W.unstable[wi] == 0;
    auto stage_body = [&](Ref r, const F* src) {
        setv(r, kX, V{src[0], src[1], src[2]});
        setq(r, kQ, Q{src[3], src[4], src[5], src[6]});
        setq(r, kQP, Q{src[3], src[4], src[5], src[6]});
        setv(r, kV, V{src[7], src[8], src[9]});
        setv(r, kW, V{src[10], src[11], src[12]});
    };
    // the position-pass q of a tile's predecessor
    auto stage_q = [&](Ref r, int body) {
        const F* tq = tile_q + ((size_t)wi * 13 + body) * 4;
        setq(r, kQ, Q{tq[0], tq[1], tq[2], tq[3]});
    };
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        stage_body(body_ref(i), rec + (b_c + i) * kBodyRec);
        if (!first_tile)
            stage_q(body_ref(i), b_c + i);
    }
    uint32_t anch = 0;
    const uint32_t* sphr = W.sph + (size_t)wi * 21;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const F* a = sr + (5 * leg + 1 + s) * kSphereRec;
#pragma unroll
        for (int c = 0; c < 6; ++c)
            sm.anch[leg][6 * s + c][j] = a[c];
        anch |= ((sphr[5 * leg + 1 + s] >> 16) & 1u) << s;
    }
    // warp 0 collides the torso's sphere and keeps its flags
    const bool capped = kWarps * lane_cap > kMaxContacts;
    if (leg == 0) {
        stage_body(torso, rec);
        if (!first_tile)
            stage_q(torso, 0);
#pragma unroll
        for (int c = 0; c < 6; ++c)
            torso[kBodyF + c] = sr[c];
        anch |= ((sphr[0] >> 16) & 1u) << 5;
    }
    const TerrainView<F> T = terrain_of(W, wi);
    const F inv_cell = F(1) / T.cell;
    const StepK<F>& st = M.step;
    unsigned long long touches = 0;  // 10 bits per sphere: leg spheres 0..4, torso sphere at 50
    if (!first_tile) {
#pragma unroll
        for (int s = 0; s < 5; ++s)
            touches |= (unsigned long long)(sphr[5 * leg + 1 + s] & 1023u) << (10 * s);
        if (leg == 0)
            touches |= (unsigned long long)(sphr[0] & 1023u) << 50;
    }
    const uint32_t* ops = &kOps[capped ? 1 : 0][leg][0];
    int last_nc = 0;  // this lane's contact records in the last substep
    __syncthreads();

    for (int sub = sub0; sub < sub1; ++sub) {
        int nc = 0;
        auto record = [&](int body, V local, V n) {
            if (nc < kOnChip) {
                const Ref d{&sm.con[leg][nc * 7][j]};
                setv(d, 0, local);
                setv(d, 3, n);
                d[6] = (F)body;
            } else if (nc < lane_cap && ARC_IN_BOUNDS(nc - kOnChip, spill_per_lane, kCheckSpillWrite)) {
                F* d = spill + (((size_t)wi * kWarps + leg) * (size_t)spill_per_lane + (nc - kOnChip)) * 8;
                d[0] = local.x; d[1] = local.y; d[2] = local.z;
                d[3] = n.x; d[4] = n.y; d[5] = n.z;
                d[6] = (F)body;
            }
            ++nc;
        };
#pragma unroll 1
        for (int i = 0;; ++i) {
            const uint32_t op = ops[i];
            const uint32_t kind = op & 15u;
            if (kind == OP_END)
                break;
            const int a = (op >> 4) & 15, b = (op >> 8) & 15, wait = (op >> 12) & 15, arrive = (op >> 16) & 15;
            if (wait)
                bar_sync(wait);
            if (kind == OP_CNT) {
                // double-buffered: a warp may record substep s+1 while
                // another still reads the counts of substep s
                sm.nc[sub & 1][leg][j] = nc;
                __syncthreads();
            } else if (active) {
                switch (kind) {
                case OP_INT:
                    // csrc/arc_phys.c:658-672
#pragma unroll 1
                    for (int o = a; o < b; ++o) {
                        const Ref r = body_ref(o == 0 ? kTorso : o - 1);
                        const BodyK<F>& k = M.body[o == 0 ? 0 : b_c + o - 1];
                        V x = getv(r, kX), v = getv(r, kV), w = getv(r, kW);
                        const Q q0 = getq(r, kQP);
                        setv(r, kXP, x);
                        v = madd(v, st.gravity, st.h);
                        x = madd(x, v, st.h);
                        if (!k.iso) {
                            const M3<F> rot = m3_from_quat(getq(r, kQ));
                            w = mul(rot, gyroscopic(k, tmul(rot, w), st.h));
                        }
                        setv(r, kX, x);
                        setq(r, kQ, q_turn(q0, scale(w, st.h)));
                        setv(r, kV, v);
                        setv(r, kW, w);
                    }
                    break;
                case OP_JNT:
#pragma unroll 1
                    for (int c = a; c < b; ++c) {
                        const Ref rp = body_ref(c == 0 ? kTorso : c - 1), rc = body_ref(c);
                        const BodyK<F>& kp = M.body[c == 0 ? 0 : b_c + c - 1];
                        const BodyK<F>& kc = M.body[b_c + c];
                        P bp, bc;
                        load_pose(rp, kp, bp);
                        load_pose(rc, kc, bc);
                        F acc = c == 0 ? tacc0 : (c == 1 ? tacc1 : tacc2);
                        const F tgt = c == 0 ? target0 : (c == 1 ? target1 : target2);
                        joint_positions(bp, kp, bc, kc, M.joint[j0 + c], tgt, acc, st.hh);
                        if (c == 0)
                            tacc0 = acc;
                        else if (c == 1)
                            tacc1 = acc;
                        else
                            tacc2 = acc;
                        store_pose(rp, bp);
                        store_pose(rc, bc);
                    }
                    break;
                case OP_COL: {
                    // csrc/arc_phys.c:542-610, spheres a..b-1 of one body
                    const int slot = a == 0 ? kTorso : (a == 1 ? 1 : 2);
                    const int bid = a == 0 ? 0 : (a == 1 ? b_f : b_t);
                    const Ref r = body_ref(slot);
                    const BodyK<F>& k = M.body[bid];
                    P pose;
                    load_pose(r, k, pose);
                    const V xp = getv(r, kXP);
                    const Q qp = getq(r, kQP);
#pragma unroll 1
                    for (int s = a; s < b; ++s) {
                        const int bit = s == 0 ? 5 : s - 1;
                        const Ref ra{s == 0 ? &sm.torso[kBodyF][j] : &sm.anch[leg][6 * (s - 1)][j]};
                        SphereState<F> ss{getv(ra, 0), getv(ra, 3), (int)((anch >> bit) & 1u)};
                        const int t = collide(pose, k, xp, qp, M.sphere[s == 0 ? 0 : 5 * leg + s], ss, T, inv_cell, st,
                                                     [&](V l, V n) { record(bid, l, n); });
                        touches += (unsigned long long)t << (10 * bit);
                        anch = (anch & ~(1u << bit)) | ((uint32_t)(ss.anchored != 0) << bit);
                        setv(ra, 0, ss.anchor);
                        setv(ra, 3, ss.anchor_n);
                    }
                    store_pose(r, pose);
                    break;
                }
                case OP_UPD:
                    // csrc/arc_phys.c:674-687; the rotation stays that of the
                    // un-normalised q (field Q)
#pragma unroll 1
                    for (int o = a; o < b; ++o) {
                        const Ref r = body_ref(o == 0 ? kTorso : o - 1);
                        Q q = getq(r, kQ);
                        V v, w;
                        update_velocity(q, getv(r, kX), v, w, getv(r, kXP), getq(r, kQP), st);
                        setq(r, kQP, q);
                        setv(r, kV, v);
                        setv(r, kW, w);
                    }
                    break;
                case OP_DMP: {
                    // csrc/arc_phys.c:459-481; the child of joint c is the
                    // parent of joint c+1 (rotation of the position pass)
                    P bp, bc;
                    Ref rp = body_ref(a == 0 ? kTorso : a - 1);
                    bp.q = getq(rp, kQ);
                    body_sync(bp, M.body[a == 0 ? 0 : b_c + a - 1]);
                    V wp = getv(rp, kW);
#pragma unroll 1
                    for (int c = a; c < b; ++c) {
                        const Ref rc = body_ref(c);
                        bc.q = getq(rc, kQ);
                        body_sync(bc, M.body[b_c + c]);
                        V wc = getv(rc, kW);
                        const JointK<F>& J = M.joint[j0 + c];
                        F acc = c == 0 ? tacc0 : (c == 1 ? tacc1 : tacc2);
                        joint_velocities<F, true>(bp.rot, bp.iiw, wp, bc.iiw, wc, J, joint_step_k(J, st), st.h,
                                                  acc);
                        if (c == 0)
                            tacc0 = acc;
                        else if (c == 1)
                            tacc1 = acc;
                        else
                            tacc2 = acc;
                        setv(rp, kW, wp);
                        rp = rc;
                        bp = bc;
                        wp = wc;
                    }
                    setv(rp, kW, wp);
                    break;
                }
                case OP_CVL: {
                    // csrc/arc_phys.c:612-626, the reference's (sphere-major)
                    // list order under its cap
                    int base = 0;
                    if (capped)
                        for (int l = 0; l < leg; ++l)
                            base += sm.nc[sub & 1][l][j];
                    const int ncl = nc < lane_cap ? nc : lane_cap;
#pragma unroll 1
                    for (int c = 0; c < ncl && base + c < kMaxContacts; ++c) {
                        F rc[7];
                        if (c < kOnChip) {
#pragma unroll
                            for (int f = 0; f < 7; ++f)
                                rc[f] = sm.con[leg][c * 7 + f][j];
                        } else {
                            if (!ARC_IN_BOUNDS(c - kOnChip, spill_per_lane, kCheckSpillRead))
                                continue;
                            const F* src =
                                spill + (((size_t)wi * kWarps + leg) * (size_t)spill_per_lane + (c - kOnChip)) * 8;
#pragma unroll
                            for (int f = 0; f < 7; ++f)
                                rc[f] = src[f];
                        }
                        const int bid = (int)rc[6];
                        if ((bid == 0) != (a == 1))
                            continue;
                        const Ref r = body_ref(bid == 0 ? kTorso : (bid == b_f ? 1 : 2));
                        const BodyK<F>& k = M.body[bid];
                        P pose;
                        pose.q = getq(r, kQ);
                        body_sync(pose, k);
                        V v = getv(r, kV), w = getv(r, kW);
                        contact_velocity(pose.rot, pose.iiw, k.inv_mass, v, w,
                                         ContactRec<F>{V{rc[0], rc[1], rc[2]}, V{rc[3], rc[4], rc[5]}});
                        setv(r, kV, v);
                        setv(r, kW, w);
                    }
                    break;
                }
                default:
                    break;
                }
            }
            if (arrive)
                bar_arrive(arrive);
        }
        last_nc = nc;
    }
    __syncthreads();

    if (last_tile && W.lastc) {
        // the last substep's contact list in the reference's order
        // (csrc/arc_phys.c:493-499): sphere by sphere, the torso's first,
        // which is the four warps' lists in warp order (the torso's records
        // lead warp 0's). Counts go through the (now free) count array.
        sm.nc[0][leg][j] = last_nc < lane_cap ? last_nc : lane_cap;
        __syncthreads();
        if (active) {
            int before = 0, total = 0;  // records of the warps listed ahead of this one; of all
            for (int l = 0; l < kWarps; ++l) {
                total += sm.nc[0][l][j];
                if (l < leg)
                    before += sm.nc[0][l][j];
            }
            const int mine = sm.nc[0][leg][j];
            F* dst = W.lastc + (size_t)world * kMaxContacts * kContactRec;
#pragma unroll 1
            for (int c = 0; c < mine; ++c) {
                const int at = before + c;
                if (at >= kMaxContacts)
                    continue;
                F rc[7];
                if (c < kOnChip) {
#pragma unroll
                    for (int f = 0; f < 7; ++f)
                        rc[f] = sm.con[leg][c * 7 + f][j];
                } else {
                    if (!ARC_IN_BOUNDS(c - kOnChip, spill_per_lane, kCheckSpillRead))
                        continue;
                    const F* src = spill + (((size_t)wi * kWarps + leg) * (size_t)spill_per_lane + (c - kOnChip)) * 8;
#pragma unroll
                    for (int f = 0; f < 7; ++f)
                        rc[f] = src[f];
                }
                F* d = dst + (size_t)at * kContactRec;
                d[0] = rc[6];
                for (int f = 0; f < 6; ++f)
                    d[1 + f] = rc[f];
            }
            if (leg == 0)
                W.lastn[world] = total < kMaxContacts ? total : kMaxContacts;
        }
    }

    if (!last_tile) {
        // hand the state to the next tile
        if (active) {
            auto keep = [&](Ref r, int body) {
                F* d = rec + body * kBodyRec;
                const V x = getv(r, kX), v = getv(r, kV), w = getv(r, kW);
                const Q q = getq(r, kQP), qa = getq(r, kQ);
                d[0] = x.x; d[1] = x.y; d[2] = x.z;
                d[3] = q.w; d[4] = q.x; d[5] = q.y; d[6] = q.z;
                d[7] = v.x; d[8] = v.y; d[9] = v.z;
                d[10] = w.x; d[11] = w.y; d[12] = w.z;
                F* tq = tile_q + ((size_t)wi * 13 + body) * 4;
                tq[0] = qa.w; tq[1] = qa.x; tq[2] = qa.y; tq[3] = qa.z;
            };
#pragma unroll 1
            for (int i = 0; i < 3; ++i)
                keep(body_ref(i), b_c + i);
            if (leg == 0)
                keep(torso, 0);
            jr[j0 * kJointRec + 3] = tacc0;
            jr[(j0 + 1) * kJointRec + 3] = tacc1;
            jr[(j0 + 2) * kJointRec + 3] = tacc2;
            uint32_t* sphw = W.sph + (size_t)world * 21;
#pragma unroll
            for (int s = 0; s < 5; ++s) {
                F* a = sr + (5 * leg + 1 + s) * kSphereRec;
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    a[c] = sm.anch[leg][6 * s + c][j];
                sphw[5 * leg + 1 + s] = (uint32_t)((touches >> (10 * s)) & 1023u) | (((anch >> s) & 1u) << 16);
            }
            if (leg == 0) {
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    sr[c] = torso[kBodyF + c];
                sphw[0] = (uint32_t)((touches >> 50) & 1023u) | (((anch >> 5) & 1u) << 16);
            }
        }
        __syncthreads();
        return;
    }

    // epilogue (csrc/arc_phys.c:739-746), from the normalised quaternions
    int bad = 0;
    if (active) {
        const Ref r0 = body_ref(0), r1 = body_ref(1), r2 = body_ref(2);
        const Q tq = getq(torso, kQP), q0 = getq(r0, kQP), q1 = getq(r1, kQP), q2 = getq(r2, kQP);
        const V tw = getv(torso, kW), w0 = getv(r0, kW), w1 = getv(r1, kW), w2 = getv(r2, kW);
        const JointK<F>& J0 = M.joint[j0];
        const JointK<F>& J1 = M.joint[j0 + 1];
        const JointK<F>& J2 = M.joint[j0 + 2];
        jr[(j0 + 0) * kJointRec + 1] = joint_angle(tq, q0, J0);
        jr[(j0 + 0) * kJointRec + 2] = joint_rate(tq, tw, w0, J0);
        jr[(j0 + 1) * kJointRec + 1] = joint_angle(q0, q1, J1);
        jr[(j0 + 1) * kJointRec + 2] = joint_rate(q0, w0, w1, J1);
        jr[(j0 + 2) * kJointRec + 1] = joint_angle(q1, q2, J2);
        jr[(j0 + 2) * kJointRec + 2] = joint_rate(q1, w1, w2, J2);
        jr[(j0 + 0) * kJointRec + 3] = tacc0 / F(M.substeps);
        jr[(j0 + 1) * kJointRec + 3] = tacc1 / F(M.substeps);
        jr[(j0 + 2) * kJointRec + 3] = tacc2 / F(M.substeps);
        auto put = [&](Ref r, F* d) {
            const V x = getv(r, kX), v = getv(r, kV), w = getv(r, kW);
            const Q q = getq(r, kQP);
            bad |= body_unstable(x, v, w);
            d[0] = x.x; d[1] = x.y; d[2] = x.z;
            d[3] = q.w; d[4] = q.x; d[5] = q.y; d[6] = q.z;
            d[7] = v.x; d[8] = v.y; d[9] = v.z;
            d[10] = w.x; d[11] = w.y; d[12] = w.z;
        };
#pragma unroll 1
        for (int i = 0; i < 3; ++i)
            put(body_ref(i), rec + (b_c + i) * kBodyRec);
        uint32_t* sphw = W.sph + (size_t)world * 21;
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            F* a = sr + (5 * leg + 1 + s) * kSphereRec;
#pragma unroll
            for (int c = 0; c < 6; ++c)
                a[c] = sm.anch[leg][6 * s + c][j];
            sphw[5 * leg + 1 + s] = (uint32_t)((touches >> (10 * s)) & 1023u) | (((anch >> s) & 1u) << 16);
        }
        if (leg == 0)
            put(torso, rec);
        if (leg == 0) {
#pragma unroll
            for (int c = 0; c < 6; ++c)
                sr[c] = torso[kBodyF + c];
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

}  // namespace
}  // namespace wl
}  // namespace arc
