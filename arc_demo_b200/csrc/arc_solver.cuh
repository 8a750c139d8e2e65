// arc_solver.cuh - XPBD solver primitives for one world, on register-held
// bodies, templated on the step precision R (float or double).
//
// This is the physics of the reference's csrc/arc_phys.c restated for the
// GPU: every helper keeps the reference's evaluation order (so an FP64 build
// differs from the reference only by FMA contraction and libm ulps), but the
// data live in small value structs that the kernels load from shared or
// global memory, update in registers and store back:
//   Pose   - what the position pass reads and writes: x, q and the derived
//            rotation / world inverse inertia (csrc/arc_phys.h:25-36)
//   BodyK  - per-body constants of the model (mass terms, inertia)
//   JointK - per-joint constants (frames, limits, drive gains)
#pragma once

#include <cstdint>
#include <cmath>

#include "arc_checks.cuh"

#ifdef __CUDACC__
#define ARC_HD __host__ __device__ __forceinline__
#else
#define ARC_HD inline
#endif

namespace arc {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// scalar helpers (csrc/arc_math.h:139-145)

template <class R> ARC_HD R r_min(R a, R b) { return a < b ? a : b; }
template <class R> ARC_HD R r_max(R a, R b) { return a > b ? a : b; }
template <class R> ARC_HD R r_clamp(R v, R lo, R hi) { return v < lo ? lo : (v > hi ? hi : v); }

ARC_HD float r_sqrt(float v) { return sqrtf(v); }
ARC_HD double r_sqrt(double v) { return sqrt(v); }
ARC_HD float r_atan2(float y, float x) { return atan2f(y, x); }
ARC_HD double r_atan2(double y, double x) { return atan2(y, x); }
ARC_HD float r_fabs(float v) { return fabsf(v); }
ARC_HD double r_fabs(double v) { return fabs(v); }
ARC_HD float r_floor(float v) { return floorf(v); }
ARC_HD double r_floor(double v) { return floor(v); }

// Singular-matrix threshold of the 3x3 solvers: the reference's 1e-300
// (csrc/arc_phys.c:252,270) underflows in FP32, so FP32 uses 1e-30.
template <class R> struct Tiny;
template <> struct Tiny<float> { static ARC_HD float det() { return 1e-30f; } };
template <> struct Tiny<double> { static ARC_HD double det() { return 1e-300; } };

// ---------------------------------------------------------------------------
// vectors, quaternions, matrices (csrc/arc_math.h:20-137)

template <class R> struct V3 { R x, y, z; };
template <class R> struct Q4 { R w, x, y, z; };
template <class R> struct M3 { R m[3][3]; };
// symmetric 3x3 (the world inverse inertia), m[i][j] == m[j][i] bitwise
template <class R> struct S3 { R xx, xy, xz, yy, yz, zz; };

template <class R> ARC_HD V3<R> v3(R x, R y, R z) { return V3<R>{x, y, z}; }
template <class R> ARC_HD V3<R> operator+(V3<R> a, V3<R> b) { return V3<R>{a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> ARC_HD V3<R> operator-(V3<R> a, V3<R> b) { return V3<R>{a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> ARC_HD V3<R> operator-(V3<R> a) { return V3<R>{-a.x, -a.y, -a.z}; }
template <class R> ARC_HD V3<R> scale(V3<R> a, R s) { return V3<R>{a.x * s, a.y * s, a.z * s}; }
template <class R> ARC_HD V3<R> vmul(V3<R> a, V3<R> b) { return V3<R>{a.x * b.x, a.y * b.y, a.z * b.z}; }
// a + b * s
template <class R> ARC_HD V3<R> madd(V3<R> a, V3<R> b, R s) { return V3<R>{a.x + b.x * s, a.y + b.y * s, a.z + b.z * s}; }
template <class R> ARC_HD R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> ARC_HD V3<R> cross(V3<R> a, V3<R> b)
{
    return V3<R>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> ARC_HD R len2(V3<R> a) { return dot(a, a); }
template <class R> ARC_HD R len(V3<R> a) { return r_sqrt(dot(a, a)); }
template <class R> ARC_HD V3<R> normalize(V3<R> a)
{
    R l = len(a);
    return l > R(1e-15) ? scale(a, R(1) / l) : V3<R>{R(0), R(0), R(0)};
}
template <class R> ARC_HD V3<R> perp(V3<R> n)
{
    V3<R> t = r_fabs(n.x) < R(0.57) ? V3<R>{R(1), R(0), R(0)} : V3<R>{R(0), R(1), R(0)};
    return normalize(cross(n, t));
}

template <class R> ARC_HD Q4<R> q_identity() { return Q4<R>{R(1), R(0), R(0), R(0)}; }
template <class R> ARC_HD Q4<R> conj(Q4<R> a) { return Q4<R>{a.w, -a.x, -a.y, -a.z}; }
template <class R> ARC_HD Q4<R> qmul(Q4<R> a, Q4<R> b)
{
    return Q4<R>{a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
                 a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
                 a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                 a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
template <class R> ARC_HD Q4<R> qnormalize(Q4<R> a)
{
    R l = r_sqrt(a.w * a.w + a.x * a.x + a.y * a.y + a.z * a.z);
    if (l < R(1e-15))
        return q_identity<R>();
    l = R(1) / l;
    return Q4<R>{a.w * l, a.x * l, a.y * l, a.z * l};
}
template <class R> ARC_HD V3<R> qrotate(Q4<R> q, V3<R> v)
{
    // v + 2w (u x v) + 2 u x (u x v)
    V3<R> u{q.x, q.y, q.z};
    V3<R> t = scale(cross(u, v), R(2));
    return madd(v, t, q.w) + cross(u, t);
}
template <class R> ARC_HD V3<R> qinv_rotate(Q4<R> q, V3<R> v) { return qrotate(conj(q), v); }

// rotation matrix of q / |q| (csrc/arc_math.h:112-122)
template <class R> ARC_HD M3<R> m3_from_quat(Q4<R> q)
{
    R k = R(2) / (q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    R x2 = q.x * k, y2 = q.y * k, z2 = q.z * k;
    R xx = q.x * x2, yy = q.y * y2, zz = q.z * z2;
    R xy = q.x * y2, xz = q.x * z2, yz = q.y * z2;
    R wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
    M3<R> r;
    r.m[0][0] = R(1) - (yy + zz); r.m[0][1] = xy - wz;           r.m[0][2] = xz + wy;
    r.m[1][0] = xy + wz;           r.m[1][1] = R(1) - (xx + zz); r.m[1][2] = yz - wx;
    r.m[2][0] = xz - wy;           r.m[2][1] = yz + wx;           r.m[2][2] = R(1) - (xx + yy);
    return r;
}
template <class R> ARC_HD V3<R> mul(const M3<R>& a, V3<R> v)
{
    return V3<R>{a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z,
                 a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
                 a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}
template <class R> ARC_HD V3<R> tmul(const M3<R>& a, V3<R> v)
{
    return V3<R>{a.m[0][0] * v.x + a.m[1][0] * v.y + a.m[2][0] * v.z,
                 a.m[0][1] * v.x + a.m[1][1] * v.y + a.m[2][1] * v.z,
                 a.m[0][2] * v.x + a.m[1][2] * v.y + a.m[2][2] * v.z};
}
template <class R> ARC_HD V3<R> mul(const S3<R>& a, V3<R> v)
{
    return V3<R>{a.xx * v.x + a.xy * v.y + a.xz * v.z,
                 a.xy * v.x + a.yy * v.y + a.yz * v.z,
                 a.xz * v.x + a.yz * v.y + a.zz * v.z};
}

// ---------------------------------------------------------------------------
// model constants

template <class R> struct BodyK {
    R inv_mass;
    V3<R> inertia, inv_inertia;
    int iso;  // inertia.x == inertia.y == inertia.z (csrc/arc_phys.c:41-44)
};

template <class R> struct JointK {
    int parent, child;
    V3<R> r1, r2, a1, a2, b1, b2;
    R lo, hi, kp, kd, max_torque;
    R lim[4];   // cos lo, sin lo, cos hi, sin hi (FP64, rounded once)
    R alpha;    // 1 / kp, the drive compliance (csrc/arc_phys.c:427)
    // per-step constants, the same operations as the reference's inline
    // expressions: alpha / (h*h), max_torque*h*h, max_torque*h
    R alpha_hh, max_dl, max_th;
};

template <class R> struct SphereK {
    int body;
    V3<R> pos;
    R radius;
};

// Per-step constants derived from h = dt / substeps. Each equals the value
// the reference recomputes inline, bit for bit (same operations, same inputs).
template <class R> struct StepK {
    R h, hh;        // h, h * h
    R inv_h, two_h; // 1 / h, 2 / h
    R mu_s, mu_d;
    V3<R> gravity;
};

// ---------------------------------------------------------------------------
// body working set of the position pass

template <class R> struct Pose {
    V3<R> x;
    Q4<R> q;
    M3<R> rot;
    S3<R> iiw;
};

// csrc/arc_phys.c:64-82
template <class R> ARC_HD void body_sync(Pose<R>& b, const BodyK<R>& k)
{
    b.rot = m3_from_quat(b.q);
    V3<R> d = k.inv_inertia;
    if (k.iso) {
        b.iiw = S3<R>{d.x, R(0), R(0), d.x, R(0), d.x};
        return;
    }
    const M3<R>& r = b.rot;
    V3<R> r0{r.m[0][0] * d.x, r.m[0][1] * d.y, r.m[0][2] * d.z};
    V3<R> r1{r.m[1][0] * d.x, r.m[1][1] * d.y, r.m[1][2] * d.z};
    V3<R> r2{r.m[2][0] * d.x, r.m[2][1] * d.y, r.m[2][2] * d.z};
    b.iiw.xx = r0.x * r.m[0][0] + r0.y * r.m[0][1] + r0.z * r.m[0][2];
    b.iiw.xy = r0.x * r.m[1][0] + r0.y * r.m[1][1] + r0.z * r.m[1][2];
    b.iiw.xz = r0.x * r.m[2][0] + r0.y * r.m[2][1] + r0.z * r.m[2][2];
    b.iiw.yy = r1.x * r.m[1][0] + r1.y * r.m[1][1] + r1.z * r.m[1][2];
    b.iiw.yz = r1.x * r.m[2][0] + r1.y * r.m[2][1] + r1.z * r.m[2][2];
    b.iiw.zz = r2.x * r.m[2][0] + r2.y * r.m[2][1] + r2.z * r.m[2][2];
}

// q + 0.5 [w, 0] q without renormalising (csrc/arc_phys.c:54-61)
template <class R> ARC_HD Q4<R> q_turn(Q4<R> q, V3<R> w)
{
    R hx = R(0.5) * w.x, hy = R(0.5) * w.y, hz = R(0.5) * w.z;
    return Q4<R>{q.w - hx * q.x - hy * q.y - hz * q.z,
                 q.x + hx * q.w + hy * q.z - hz * q.y,
                 q.y - hx * q.z + hy * q.w + hz * q.x,
                 q.z + hx * q.y - hy * q.x + hz * q.w};
}

// csrc/arc_phys.c:182-194
template <class R> ARC_HD R w_pos(const Pose<R>& b, const BodyK<R>& k, V3<R> r, V3<R> n)
{
    V3<R> rn = cross(r, n);
    return k.inv_mass + dot(rn, mul(b.iiw, rn));
}
template <class R> ARC_HD R w_rot(const Pose<R>& b, V3<R> n) { return dot(n, mul(b.iiw, n)); }

// csrc/arc_phys.c:196-211
template <class R> ARC_HD void pos_impulse(Pose<R>& b, const BodyK<R>& k, V3<R> r, V3<R> p)
{
    b.x = madd(b.x, p, k.inv_mass);
    b.q = q_turn(b.q, mul(b.iiw, cross(r, p)));
    body_sync(b, k);
}
template <class R> ARC_HD void rot_impulse(Pose<R>& b, const BodyK<R>& k, V3<R> p)
{
    b.q = q_turn(b.q, mul(b.iiw, p));
    body_sync(b, k);
}

// Positional correction of one body against the static world (the only form
// the solver uses: csrc/arc_phys.c:226-242 with b2 = NULL, alpha = 0).
template <class R>
ARC_HD R solve_pos_static(Pose<R>& b, const BodyK<R>& k, V3<R> r, V3<R> d, R hh)
{
    R c = len(d);
    if (c < R(1e-12))
        return R(0);
    V3<R> n = scale(d, R(1) / c);
    // the reference adds w_pos(NULL) = 0 and alpha / (h*h) = 0 here; both
    // are exact no-ops for the value and for the sign test below
    (void)hh;
    R denom = w_pos(b, k, r, n);
    if (denom <= R(0))
        return R(0);
    R dl = c / denom;
    pos_impulse(b, k, r, scale(n, dl));
    return dl;
}

// Cramer's rule (csrc/arc_phys.c:245-262)
template <class R> ARC_HD bool solve3(const M3<R>& K, V3<R> d, V3<R>& x)
{
    R c00 = K.m[1][1] * K.m[2][2] - K.m[1][2] * K.m[2][1];
    R c01 = K.m[1][2] * K.m[2][0] - K.m[1][0] * K.m[2][2];
    R c02 = K.m[1][0] * K.m[2][1] - K.m[1][1] * K.m[2][0];
    R det = K.m[0][0] * c00 + K.m[0][1] * c01 + K.m[0][2] * c02;
    if (r_fabs(det) < Tiny<R>::det())
        return false;
    R inv = R(1) / det;
    V3<R> c0{K.m[0][0], K.m[1][0], K.m[2][0]};
    V3<R> c1{K.m[0][1], K.m[1][1], K.m[2][1]};
    V3<R> c2{K.m[0][2], K.m[1][2], K.m[2][2]};
    x.x = dot(d, cross(c1, c2)) * inv;
    x.y = dot(c0, cross(d, c2)) * inv;
    x.z = dot(c0, cross(c1, d)) * inv;
    return true;
}

// symmetric adjugate solve (csrc/arc_phys.c:265-280)
template <class R> ARC_HD bool solve3_sym(const S3<R>& K, V3<R> d, V3<R>& x)
{
    R a = K.xx, b = K.xy, c = K.xz, e = K.yy, f = K.yz, g = K.zz;
    R A = e * g - f * f, B = c * f - b * g, C = b * f - c * e;
    R det = a * A + b * B + c * C;
    if (r_fabs(det) < Tiny<R>::det())
        return false;
    R inv = R(1) / det;
    R D = a * g - c * c;
    R E = b * c - a * f;
    R F = a * e - b * b;
    x.x = (A * d.x + B * d.y + C * d.z) * inv;
    x.y = (B * d.x + D * d.y + E * d.z) * inv;
    x.z = (C * d.x + E * d.y + F * d.z) * inv;
    return true;
}

// K += point mass matrix of a body at offset r (csrc/arc_phys.c:284-300)
template <class R> ARC_HD void add_point_mass(S3<R>& K, const S3<R>& a, R inv_mass, V3<R> r)
{
    R x = r.x, y = r.y, z = r.z;
    K.xx += inv_mass + a.yy * z * z - R(2) * a.yz * y * z + a.zz * y * y;
    K.yy += inv_mass + a.zz * x * x - R(2) * a.xz * x * z + a.xx * z * z;
    K.zz += inv_mass + a.xx * y * y - R(2) * a.xy * x * y + a.yy * x * x;
    R k01 = a.yz * x * z + a.xz * y * z - a.xy * z * z - a.zz * x * y;
    R k02 = a.xy * y * z + a.yz * x * y - a.yy * x * z - a.xz * y * y;
    R k12 = a.xz * x * y + a.xy * x * z - a.xx * y * z - a.yz * x * x;
    K.xy += k01;
    K.xz += k02;
    K.yz += k12;
}

// ---------------------------------------------------------------------------
// joints. P: the joint has a parent body (false: attached to the static world)

// body-frame vector in world frame; the static world is the identity
template <class R, bool P> ARC_HD V3<R> brot(const Pose<R>& b, V3<R> v)
{
    if (P)
        return mul(b.rot, v);
    return v;
}

// csrc/arc_phys.c:308-320
template <class R, bool P>
ARC_HD void solve_point(Pose<R>& b1, const BodyK<R>& k1, V3<R> r1, Pose<R>& b2, const BodyK<R>& k2,
                        V3<R> r2, V3<R> d)
{
    if (len2(d) < R(1e-24))
        return;
    S3<R> K{R(0), R(0), R(0), R(0), R(0), R(0)};
    if (P)
        add_point_mass(K, b1.iiw, k1.inv_mass, r1);
    add_point_mass(K, b2.iiw, k2.inv_mass, r2);
    V3<R> p;
    if (!solve3_sym(K, d, p))
        return;
    if (P)
        pos_impulse(b1, k1, r1, p);
    pos_impulse(b2, k2, r2, -p);
}

// csrc/arc_phys.c:328-346
template <class R, bool P>
ARC_HD void solve_rot_block(Pose<R>& b1, const BodyK<R>& k1, Pose<R>& b2, const BodyK<R>& k2, V3<R> rot)
{
    if (len2(rot) < R(1e-24))
        return;
    S3<R> K{R(0), R(0), R(0), R(0), R(0), R(0)};
    if (P) {
        K.xx += b1.iiw.xx; K.xy += b1.iiw.xy; K.xz += b1.iiw.xz;
        K.yy += b1.iiw.yy; K.yz += b1.iiw.yz; K.zz += b1.iiw.zz;
    }
    K.xx += b2.iiw.xx; K.xy += b2.iiw.xy; K.xz += b2.iiw.xz;
    K.yy += b2.iiw.yy; K.yz += b2.iiw.yz; K.zz += b2.iiw.zz;
    V3<R> p;
    if (!solve3_sym(K, rot, p))
        return;
    if (P)
        rot_impulse(b1, k1, p);
    rot_impulse(b2, k2, -p);
}

// csrc/arc_phys.c:353-371; alpha_hh = alpha / (h * h)
template <class R, bool P>
ARC_HD V3<R> solve_rot(Pose<R>& b1, const BodyK<R>& k1, Pose<R>& b2, const BodyK<R>& k2, V3<R> rot,
                       R alpha_hh, R max_dl)
{
    R theta = len(rot);
    if (theta < R(1e-12))
        return V3<R>{R(0), R(0), R(0)};
    V3<R> n = scale(rot, R(1) / theta);
    R denom = (P ? w_rot(b1, n) : R(0)) + w_rot(b2, n) + alpha_hh;
    if (denom <= R(0))
        return V3<R>{R(0), R(0), R(0)};
    R dl = theta / denom;
    if (dl > max_dl)
        dl = max_dl;
    V3<R> p = scale(n, dl);
    if (P)
        rot_impulse(b1, k1, p);
    rot_impulse(b2, k2, -p);
    return p;
}

// Per-joint per-step constants: alpha / (h*h) and max_torque * h * h, each
// the same operations as the reference's inline expressions.
template <class R> struct JointStepK {
    R alpha_hh, max_dl, max_th;  // alpha/(h*h), max_torque*h*h, max_torque*h
};

template <class R> ARC_HD JointStepK<R> joint_step_k(const JointK<R>& j, const StepK<R>& s)
{
    (void)s;
    JointStepK<R> o;
    o.alpha_hh = j.alpha_hh;
    o.max_dl = j.max_dl;
    o.max_th = j.max_th;
    return o;
}

// csrc/arc_phys.c:413-457: drive, limits, axis alignment, attachment.
template <class R, bool P>
ARC_HD void joint_positions(Pose<R>& bp, const BodyK<R>& kp, Pose<R>& bc, const BodyK<R>& kc,
                            const JointK<R>& j, const JointStepK<R>& js, R target, R& torque_acc,
                            R hh)
{
    V3<R> a1;
    R s, c;
    if (j.kp > R(0)) {
        a1 = brot<R, P>(bp, j.a1);
        V3<R> b1 = brot<R, P>(bp, j.b1), b2 = mul(bc.rot, j.b2);
        s = dot(cross(b1, b2), a1);
        c = dot(b1, b2);
        R phi = r_atan2(s, c);
        V3<R> p = solve_rot<R, P>(bp, kp, bc, kc, scale(a1, phi - target), js.alpha_hh, js.max_dl);
        torque_acc -= dot(p, a1) / hh;
    }
    if (j.lo <= j.hi) {
        a1 = brot<R, P>(bp, j.a1);
        V3<R> b1 = brot<R, P>(bp, j.b1), b2 = mul(bc.rot, j.b2);
        s = dot(cross(b1, b2), a1);
        c = dot(b1, b2);
        if (j.hi - j.lo > R(kPi) || s * j.lim[0] - c * j.lim[1] < R(0) || j.lim[3] * c - j.lim[2] * s < R(0)) {
            R phi = r_atan2(s, c);
            if (phi < j.lo)
                solve_rot_block<R, P>(bp, kp, bc, kc, scale(a1, phi - j.lo));
            else if (phi > j.hi)
                solve_rot_block<R, P>(bp, kp, bc, kc, scale(a1, phi - j.hi));
        }
    }
    a1 = brot<R, P>(bp, j.a1);
    solve_rot_block<R, P>(bp, kp, bc, kc, cross(a1, mul(bc.rot, j.a2)));
    V3<R> r1 = brot<R, P>(bp, j.r1);
    V3<R> r2 = mul(bc.rot, j.r2);
    V3<R> p1 = P ? bp.x + r1 : r1;
    V3<R> p2 = bc.x + r2;
    solve_point<R, P>(bp, kp, r1, bc, kc, r2, p2 - p1);
}

// csrc/arc_phys.c:459-481: drive damping; rot and iiw of both bodies are
// those left by the position pass.
template <class R, bool P>
ARC_HD void joint_velocities(const M3<R>& rotp, const S3<R>& iiwp, V3<R>& wp, const S3<R>& iiwc, V3<R>& wc,
                             const JointK<R>& j, const JointStepK<R>& js, R h, R& torque_acc)
{
    if (j.kd <= R(0))
        return;
    V3<R> a = P ? mul(rotp, j.a1) : j.a1;
    V3<R> wpar = P ? wp : V3<R>{R(0), R(0), R(0)};
    R rel = dot(wc - wpar, a);
    R wsum = (P ? dot(a, mul(iiwp, a)) : R(0)) + dot(a, mul(iiwc, a));
    if (wsum <= R(0))
        return;
    R impulse = -j.kd * rel * h;
    R cap = r_min(r_fabs(rel) / wsum, js.max_th);
    impulse = r_clamp(impulse, -cap, cap);
    if (P)
        wp = wp - mul(iiwp, scale(a, impulse));
    wc = wc + mul(iiwc, scale(a, impulse));
    torque_acc += impulse / h;
}

// csrc/arc_phys.c:386-400, from normalised quaternions (end of step)
template <class R>
ARC_HD R joint_angle(Q4<R> qp, Q4<R> qc, const JointK<R>& j)
{
    V3<R> a = qrotate(qp, j.a1);
    V3<R> b1 = qrotate(qp, j.b1);
    V3<R> b2 = qrotate(qc, j.b2);
    return r_atan2(dot(cross(b1, b2), a), dot(b1, b2));
}
template <class R>
ARC_HD R joint_rate(Q4<R> qp, V3<R> wp, V3<R> wc, const JointK<R>& j)
{
    V3<R> a = qrotate(qp, j.a1);
    return dot(wc - wp, a);
}

// ---------------------------------------------------------------------------
// integration and velocity update (csrc/arc_phys.c:636-687)

template <class R> ARC_HD V3<R> gyroscopic(const BodyK<R>& k, V3<R> w0, R h)
{
    M3<R> J;
    V3<R> iw = vmul(w0, k.inertia), f = scale(cross(w0, iw), h), dw;
    R in[3] = {k.inertia.x, k.inertia.y, k.inertia.z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        V3<R> e{R(c == 0), R(c == 1), R(c == 2)};
        V3<R> col = scale(e, in[c]) + scale(scale(cross(w0, e), in[c]) - cross(iw, e), h);
        J.m[0][c] = col.x;
        J.m[1][c] = col.y;
        J.m[2][c] = col.z;
    }
    if (!solve3(J, f, dw))
        return w0;
    return w0 - dw;
}

// One body's integrate step (csrc/arc_phys.c:661-671): x_prev/q_prev are
// returned through xp/qp; rot of the incoming pose must be current.
template <class R>
ARC_HD void integrate_body(Pose<R>& b, V3<R>& v, V3<R>& w, V3<R>& xp, Q4<R>& qp, const BodyK<R>& k,
                           const StepK<R>& s)
{
    xp = b.x;
    qp = b.q;
    v = madd(v, s.gravity, s.h);
    b.x = madd(b.x, v, s.h);
    if (!k.iso)
        w = mul(b.rot, gyroscopic(k, tmul(b.rot, w), s.h));
    b.q = q_turn(b.q, scale(w, s.h));
    body_sync(b, k);
}

template <class R>
ARC_HD void update_velocity(Q4<R>& q, V3<R> x, V3<R>& v, V3<R>& w, V3<R> xp, Q4<R> qp, const StepK<R>& s)
{
    q = qnormalize(q);
    Q4<R> dq = qmul(q, conj(qp));
    v = scale(x - xp, s.inv_h);
    w = scale(V3<R>{dq.x, dq.y, dq.z}, s.two_h);
    if (dq.w < R(0))
        w = -w;
}

// csrc/arc_phys.c:689-705: true when the body makes the world unstable
template <class R> ARC_HD bool is_finite_r(R v) { return v == v && v < R(1e300) && v > R(-1e300); }
template <class R> ARC_HD bool body_unstable(V3<R> x, V3<R> v, V3<R> w)
{
    R v2 = len2(v), w2 = len2(w);
    return !is_finite_r(v2) || !is_finite_r(w2) || !(len2(x) < R(1e6) * R(1e6)) || v2 > R(60) * R(60) ||
           w2 > R(400) * R(400);
}

// ---------------------------------------------------------------------------
// terrain (csrc/arc_terrain.h:13-50): heights h[ix + iy * nx]

template <class R> struct TerrainView {
    const R* h;
    int nx, ny;
    R cell, ox, oy, outside;
#ifdef ARC_DEVICE_CHECKS
    long long cap = -1;  // columns of the world's slice of the pool (< 0: unchecked)
#endif
};

template <class R> ARC_HD R terrain_cell(const TerrainView<R>& t, int ix, int iy)
{
    if (ix < 0 || iy < 0 || ix >= t.nx || iy >= t.ny)
        return t.outside;
#ifdef ARC_DEVICE_CHECKS
    if (t.cap >= 0 && !ARC_IN_BOUNDS(ix + (long long)iy * t.nx, t.cap, kCheckTerrainRead))
        return t.outside;
#endif
#ifdef __CUDA_ARCH__
    return __ldg(t.h + ix + iy * t.nx);
#else
    return t.h[ix + iy * t.nx];
#endif
}

// ---------------------------------------------------------------------------
// contacts

template <class R> struct ContactRec {
    V3<R> local, n;
};

// Per-sphere friction state (csrc/arc_phys.h:38-46)
template <class R> struct SphereState {
    V3<R> anchor, anchor_n;
    int anchored;
};

// csrc/arc_phys.c:512-539. xprev/qprev: the body pose at the substep start.
template <class R>
ARC_HD void solve_friction(Pose<R>& b, const BodyK<R>& k, V3<R> xprev, Q4<R> qprev, const SphereK<R>& sk,
                           SphereState<R>& ss, V3<R> n, R ln, const StepK<R>& st)
{
    V3<R> c = b.x + mul(b.rot, sk.pos);
    V3<R> p = madd(c, n, -sk.radius);
    R frac = R(1);
    if (!ss.anchored || dot(n, ss.anchor_n) < R(0.9)) {
        V3<R> c0 = xprev + qrotate(qprev, sk.pos);
        ss.anchor = madd(c0, n, -sk.radius);
        ss.anchor_n = n;
        ss.anchored = 1;
    }
    V3<R> e = p - ss.anchor;
    e = madd(e, n, -dot(e, n));
    R l = len(e);
    if (l < R(1e-12))
        return;
    V3<R> r = p - b.x;
    R wt = w_pos(b, k, r, scale(e, R(1) / l));
    R lt = l / wt;
    if (lt > st.mu_s * ln) {
        frac = r_min(st.mu_d * ln / lt, R(1));
        ss.anchor = madd(ss.anchor, e, R(1) - frac);
    }
    solve_pos_static(b, k, r, scale(e, -frac), st.hh);
}

// Sphere vs the column grid (csrc/arc_phys.c:542-610). Each contact is
// solved at once and handed to `record(local, n)` for the velocity pass.
// Returns 1 when the sphere touched.
template <class R, class Rec>
ARC_HD int collide_sphere(Pose<R>& b, const BodyK<R>& k, V3<R> xprev, Q4<R> qprev, const SphereK<R>& sk,
                          SphereState<R>& ss, const TerrainView<R>& t, const StepK<R>& st, Rec&& record)
{
    R rad = sk.radius, ln = R(0);
    V3<R> c = b.x + mul(b.rot, sk.pos), n_max{R(0), R(0), R(1)};
    R depth_max = R(0);
    int touched = 0;
    if (!(r_fabs(c.x) < R(1e6) && r_fabs(c.y) < R(1e6))) {
        ss.anchored = 0;
        return 0;
    }
    int ix0 = (int)r_floor((c.x - rad - t.ox) / t.cell);
    int ix1 = (int)r_floor((c.x + rad - t.ox) / t.cell);
    int iy0 = (int)r_floor((c.y - rad - t.oy) / t.cell);
    int iy1 = (int)r_floor((c.y + rad - t.oy) / t.cell);
    for (int iy = iy0; iy <= iy1; ++iy) {
        for (int ix = ix0; ix <= ix1; ++ix) {
            R top = terrain_cell(t, ix, iy);
            if (c.z - rad >= top)
                continue;
            R x0 = t.ox + R(ix) * t.cell, x1 = x0 + t.cell;
            R y0 = t.oy + R(iy) * t.cell, y1 = y0 + t.cell;
            int sx = c.x > x1 ? 1 : (c.x < x0 ? -1 : 0);
            int sy = c.y > y1 ? 1 : (c.y < y0 ? -1 : 0);
            if (sx && terrain_cell(t, ix + sx, iy) >= top)
                continue;
            if (sy && terrain_cell(t, ix, iy + sy) >= top)
                continue;
            if (sx && sy && terrain_cell(t, ix + sx, iy + sy) >= top)
                continue;
            V3<R> q{r_clamp(c.x, x0, x1), r_clamp(c.y, y0, y1), r_min(c.z, top)};
            V3<R> diff = c - q;
            R dist = len(diff), depth;
            V3<R> n;
            if (dist > R(1e-9)) {
                if (dist >= rad)
                    continue;
                n = scale(diff, R(1) / dist);
                depth = rad - dist;
            } else {
                n = V3<R>{R(0), R(0), R(1)};
                depth = top - c.z + rad;
            }
            // csrc/arc_phys.c:488-500
            V3<R> point = madd(c, n, -rad);
            V3<R> r = point - b.x;
            ln += solve_pos_static(b, k, r, scale(n, depth), st.hh);
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
        solve_friction(b, k, xprev, qprev, sk, ss, n_max, ln, st);
    else
        ss.anchored = 0;
    return touched;
}

// Removes the normal velocity at one recorded contact (csrc/arc_phys.c:612-626).
template <class R>
ARC_HD void contact_velocity(const M3<R>& rot, const S3<R>& iiw, R inv_mass, V3<R>& v, V3<R>& w,
                             const ContactRec<R>& c)
{
    V3<R> r = mul(rot, c.local);
    V3<R> vc = v + cross(w, r);
    R vn = dot(c.n, vc);
    V3<R> rn = cross(r, c.n);
    R wp = inv_mass + dot(rn, mul(iiw, rn));
    V3<R> p = scale(c.n, -vn / wp);
    v = madd(v, p, inv_mass);
    w = w + mul(iiw, cross(r, p));
}

}  // namespace arc
