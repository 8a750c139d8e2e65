// arc_model.cu - host construction of the robot template (FP64).
#include <algorithm>
#include <cmath>
#include <cstring>
#include "arc_model.h"

namespace arc {

// csrc/arc_phys.c:801-821
V3<double> inertia_box(double mass, V3<double> he)
{
    double k = mass / 3.0;
    return V3<double>{k * (he.y * he.y + he.z * he.z), k * (he.x * he.x + he.z * he.z),
                      k * (he.x * he.x + he.y * he.y)};
}

V3<double> inertia_capsule_z(double mass, double radius, double half_length)
{
    double len_ = 2.0 * (half_length + radius);
    double ixx = mass * (3.0 * radius * radius + len_ * len_) / 12.0;
    return V3<double>{ixx, ixx, 0.5 * mass * radius * radius};
}

V3<double> inertia_sphere(double mass, double r)
{
    double i = 0.4 * mass * r * r;
    return V3<double>{i, i, i};
}

int ModelHost::add_body(double mass, V3<double> inertia, V3<double> pos, Q4<double> q)
{
    if (nb >= kMaxBodies)
        return -1;
    Body& bd = b[nb];
    bd.x = pos;
    bd.q = qnormalize(q);
    bd.mass = mass;
    bd.inv_mass = 1.0 / mass;
    bd.inertia = inertia;
    bd.inv_inertia = V3<double>{1.0 / inertia.x, 1.0 / inertia.y, 1.0 / inertia.z};
    return nb++;
}

int ModelHost::add_sphere(int body, V3<double> pos, double radius)
{
    if (ns >= kMaxSpheres)
        return -1;
    s[ns] = Sphere{body, pos, radius};
    channel[ns] = 0;
    return ns++;
}

int ModelHost::add_visual(int type, int body, V3<double> p0, V3<double> p1, double radius, double radius2,
                          int material, const float* rgb)
{
    if (nv >= kMaxVisuals)
        return -1;
    v[nv] = Visual{type, body, material, p0, p1, radius, radius2, 1.0, {rgb[0], rgb[1], rgb[2]}};
    return nv++;
}

int ModelHost::add_hinge(int parent, int child, V3<double> anchor, V3<double> axis_world)
{
    if (nj >= kMaxJoints || child <= parent)
        return -1;
    Q4<double> qp = q_identity<double>();
    V3<double> xp{0.0, 0.0, 0.0};
    if (parent >= 0) {
        xp = b[parent].x;
        qp = b[parent].q;
    }
    Q4<double> qc = b[child].q;
    V3<double> axis = normalize(axis_world);
    V3<double> ref = perp(axis);
    Joint& jt = j[nj];
    jt.parent = parent;
    jt.child = child;
    jt.r1 = qinv_rotate(qp, anchor - xp);
    jt.r2 = qinv_rotate(qc, anchor - b[child].x);
    jt.a1 = qinv_rotate(qp, axis);
    jt.a2 = qinv_rotate(qc, axis);
    jt.b1 = qinv_rotate(qp, ref);
    jt.b2 = qinv_rotate(qc, ref);
    jt.q_rel0 = qmul(conj(qp), qc);
    jt.lo = 1.0;  // lo > hi: limits off
    jt.hi = -1.0;
    jt.kp = jt.kd = jt.max_torque = 0.0;
    return nj++;
}

static Q4<double> axis_angle(V3<double> axis, double angle)
{
    double s = sin(0.5 * angle);
    return Q4<double>{cos(0.5 * angle), axis.x * s, axis.y * s, axis.z * s};
}

void ModelHost::pose(V3<double> root_x, Q4<double> root_q, const double* angles, V3<double>* xs,
                     Q4<double>* qs) const
{
    for (int i = 0; i < nb; ++i) {
        xs[i] = b[i].x;
        qs[i] = b[i].q;
    }
    xs[0] = root_x;
    qs[0] = qnormalize(root_q);
    for (int i = 0; i < nj; ++i) {
        const Joint& jt = j[i];
        V3<double> xp = jt.parent >= 0 ? xs[jt.parent] : V3<double>{0.0, 0.0, 0.0};
        Q4<double> qp = jt.parent >= 0 ? qs[jt.parent] : q_identity<double>();
        V3<double> anchor = xp + qrotate(qp, jt.r1);
        qs[jt.child] = qnormalize(qmul(qp, qmul(axis_angle(jt.a1, angles[i]), jt.q_rel0)));
        xs[jt.child] = anchor - qrotate(qs[jt.child], jt.r2);
    }
}

// Leg geometry, masses and drive gains of csrc/arc_robot.c:16-36.
namespace leaper {
constexpr double kBodyMass = 8.0, kBodyR = 0.2;
constexpr double kCoxaMass = 0.4, kCoxaInertia = 0.02;
constexpr double kFemurMass = 1.5, kTibiaMass = 1.0;
constexpr double kLegAngle = 0.785, kHipElevation = 0.785;
constexpr double kCoxaLen = 0.06, kFemurLen = 0.50, kTibiaLen = 0.95, kFootR = 0.045;
constexpr double kKp = 250.0, kKd = 6.0, kMaxTorque = 80.0;
}  // namespace leaper

// Surface colours (sRGB) of csrc/arc_robot.c:38-47.
namespace paint {
constexpr float kArmor[3] = {0.40f, 0.41f, 0.43f}, kHull[3] = {0.34f, 0.345f, 0.36f};
constexpr float kDark[3] = {0.17f, 0.17f, 0.18f}, kSteel[3] = {0.52f, 0.53f, 0.55f};
constexpr float kBezel[3] = {0.72f, 0.73f, 0.74f}, kCable[3] = {0.30f, 0.30f, 0.31f};
constexpr float kBlack[3] = {0.06f, 0.06f, 0.065f}, kGlow[3] = {1.00f, 0.10f, 0.06f};
constexpr float kDimGlow[3] = {0.62f, 0.05f, 0.03f};
}  // namespace paint

// A faceted armour plate along body z (csrc/arc_robot.c:55-61).
static void add_plate(ModelHost& m, int body, V3<double> p0, V3<double> p1, double r0, double r1, double aspect)
{
    int i = m.add_visual(kVisTaper, body, p0, p1, r0, r1, kMatPaint, paint::kArmor);
    if (i >= 0)
        m.v[i].aspect = aspect;
}

// The visuals of one leg, in the order of csrc/arc_robot.c:114-142: hip
// hinge and collar on the coxa; knee axle, armour plate, cable sleeve, knee
// block, knee hinge and its two lights on the femur; two plates, a sleeve,
// the ankle, its collars and the rubber foot on the tibia.
static void add_leg_visuals(ModelHost& m, int bc, int bf, int bt, V3<double> d, double fl, double tl)
{
    using V = V3<double>;
    using namespace paint;
    m.add_visual(kVisCylinder, bc, scale(d, -0.05), scale(d, 0.035), 0.062, 0.0, kMatMetal, kDark);
    m.add_visual(kVisRing, bc, scale(d, 0.02), d, 0.062, 0.012, kMatMetal, kSteel);
    m.add_visual(kVisCylinder, bf, V{0, -0.07, -fl}, V{0, 0.07, -fl}, 0.045, 0.0, kMatMetal, kDark);
    add_plate(m, bf, V{-0.012, 0, -fl + 0.02}, V{-0.012, 0, fl - 0.02}, 0.055, 0.08, 0.8);
    m.add_visual(kVisCylinder, bf, V{0.055, 0, -fl + 0.06}, V{0.07, 0, fl - 0.07}, 0.022, 0.0, kMatRibs, kCable);
    m.add_visual(kVisBox, bf, V{0, 0, fl}, V{0.085, 0.07, 0.075}, 0.0, 0.0, kMatPaint, kDark);
    m.add_visual(kVisCylinder, bf, V{0, -0.085, fl}, V{0, 0.085, fl}, 0.048, 0.0, kMatMetal, kSteel);
    m.add_visual(kVisCylinder, bf, V{0, 0.085, fl}, V{0, 0.089, fl}, 0.02, 0.0, kMatGlow, kGlow);
    m.add_visual(kVisCylinder, bf, V{0, -0.089, fl}, V{0, -0.085, fl}, 0.02, 0.0, kMatGlow, kGlow);
    add_plate(m, bt, V{-0.01, 0, -tl + 0.03}, V{-0.01, 0, -0.05}, 0.068, 0.082, 0.8);
    add_plate(m, bt, V{-0.01, 0, -0.05}, V{-0.004, 0, tl - 0.11}, 0.082, 0.03, 0.85);
    m.add_visual(kVisCylinder, bt, V{0.065, 0, -tl + 0.08}, V{0.045, 0, 0.25 * tl}, 0.02, 0.0, kMatRibs, kCable);
    m.add_visual(kVisCylinder, bt, V{0, 0, tl - 0.12}, V{0, 0, tl - 0.035}, 0.026, 0.0, kMatMetal, kSteel);
    m.add_visual(kVisRing, bt, V{0, 0, tl - 0.09}, V{0, 0, 1}, 0.03, 0.01, kMatMetal, kDark);
    m.add_visual(kVisSphere, bt, V{0, 0, tl}, V{0, 0, 0}, leaper::kFootR, 0.0, kMatRubber, kBlack);
    m.add_visual(kVisRing, bt, V{0, 0, tl - 0.02}, V{0, 0, 1}, 0.036, 0.011, kMatMetal, kSteel);
}

// The torso's visuals (csrc/arc_robot.c:158-170): panelled hull, two collars,
// a bottom hatch, two side knobs, and the eye (glow ring, bezel, lens, inner
// glow ring). The renderer's eye light is the first glowing ring on body 0.
static void add_torso_visuals(ModelHost& m)
{
    using V = V3<double>;
    using namespace paint;
    m.add_visual(kVisSphere, 0, V{0, 0, 0}, V{0, 0, 0}, leaper::kBodyR, 0.0, kMatPanels, kHull);
    m.add_visual(kVisRing, 0, V{0, 0, 0.135}, V{0, 0, 1}, 0.148, 0.02, kMatMetal, kDark);
    m.add_visual(kVisRing, 0, V{0, 0, -0.125}, V{0, 0, 1}, 0.156, 0.024, kMatPaint, kDark);
    m.add_visual(kVisCylinder, 0, V{0, 0, -0.2}, V{0, 0, -0.17}, 0.07, 0.0, kMatMetal, kDark);
    for (int side = -1; side <= 1; side += 2) {
        V k = normalize(V{0.45, 0.62 * side, -0.64});
        m.add_visual(kVisCylinder, 0, scale(k, 0.17), scale(k, 0.215), 0.028, 0.0, kMatMetal, kSteel);
    }
    m.add_visual(kVisRing, 0, V{0.18, 0, 0}, V{1, 0, 0}, 0.08, 0.013, kMatGlow, kGlow);
    m.add_visual(kVisRing, 0, V{0.168, 0, 0}, V{1, 0, 0}, 0.112, 0.02, kMatMetal, kBezel);
    m.add_visual(kVisCylinder, 0, V{0.11, 0, 0}, V{0.178, 0, 0}, 0.095, 0.0, kMatLens, kBlack);
    m.add_visual(kVisRing, 0, V{0.181, 0, 0}, V{1, 0, 0}, 0.032, 0.006, kMatGlow, kDimGlow);
}

static void set_drive(ModelHost::Joint& jt, double lo, double hi)
{
    jt.lo = lo;
    jt.hi = hi;
    jt.kp = leaper::kKp;
    jt.kd = leaper::kKd;
    jt.max_torque = leaper::kMaxTorque;
}

// csrc/arc_robot.c:88-142: bodies, hinges, collision spheres, then the
// render-only visuals
static void build_leg(ModelHost& m, int leg, double sx, double sy)
{
    using namespace leaper;
    double psi = sx > 0.0 ? sy * kLegAngle : sy * (kPi - kLegAngle);
    V3<double> d{cos(psi), sin(psi), 0.0};
    V3<double> up{0.0, 0.0, 1.0};
    V3<double> lift = cross(d, up);
    Q4<double> along = axis_angle(normalize(cross(up, d)), 0.5 * kPi);
    V3<double> hip = scale(d, kBodyR * cos(kHipElevation)) + V3<double>{0.0, 0.0, kBodyR * sin(kHipElevation)};
    V3<double> p1 = madd(hip, d, kCoxaLen);
    V3<double> p2 = madd(p1, d, kFemurLen);
    double fl = 0.5 * kFemurLen, tl = 0.5 * kTibiaLen;
    int bc = m.add_body(kCoxaMass, V3<double>{kCoxaInertia, kCoxaInertia, kCoxaInertia}, madd(hip, d, 0.5 * kCoxaLen),
                        q_identity<double>());
    int bf = m.add_body(kFemurMass, inertia_capsule_z(kFemurMass, 0.06, fl), madd(p1, d, fl), along);
    int bt = m.add_body(kTibiaMass, inertia_capsule_z(kTibiaMass, 0.05, tl), madd(p2, d, tl), along);
    int j = m.add_hinge(0, bc, hip, V3<double>{0.0, 0.0, -sy});
    set_drive(m.j[j], -0.8, 0.8);
    j = m.add_hinge(bc, bf, p1, lift);
    set_drive(m.j[j], -0.4, 1.5);
    j = m.add_hinge(bf, bt, p2, lift);
    set_drive(m.j[j], -2.8, -0.5);
    m.default_angles[3 * leg + 0] = 0.0;
    m.default_angles[3 * leg + 1] = 0.6;
    m.default_angles[3 * leg + 2] = -1.95;
    m.add_sphere(bf, V3<double>{0.0, 0.0, 0.0}, 0.06);
    m.add_sphere(bt, V3<double>{0.0, 0.0, -tl}, 0.07);
    m.add_sphere(bt, V3<double>{0.0, 0.0, -0.3 * tl}, 0.055);
    m.add_sphere(bt, V3<double>{0.0, 0.0, 0.4 * tl}, 0.035);
    m.foot_sphere[leg] = m.add_sphere(bt, V3<double>{0.0, 0.0, tl}, kFootR);
    add_leg_visuals(m, bc, bf, bt, d, fl, tl);
}

void build_leaper(ModelHost& m)
{
    using namespace leaper;
    static const double SX[kNumLegs] = {1.0, 1.0, -1.0, -1.0};
    static const double SY[kNumLegs] = {1.0, -1.0, 1.0, -1.0};
    m = ModelHost();
    m.add_body(kBodyMass, inertia_sphere(kBodyMass, kBodyR), V3<double>{0, 0, 0}, q_identity<double>());
    m.add_sphere(0, V3<double>{0, 0, 0}, kBodyR);
    m.n_torso_spheres = m.ns;
    add_torso_visuals(m);
    for (int leg = 0; leg < kNumLegs; ++leg)
        build_leg(m, leg, SX[leg], SY[leg]);
    m.total_mass = 0.0;
    for (int i = 0; i < m.nb; ++i)
        m.total_mass += m.b[i].mass;
    // contact channels: foot k -> k, torso -> 4, other leg parts -> 5 (csrc/arc_sim.c:47-50)
    for (int i = 0; i < m.ns; ++i)
        m.channel[i] = i < m.n_torso_spheres ? kNumLegs : kNumLegs + 1;
    for (int k = 0; k < kNumLegs; ++k)
        m.channel[m.foot_sphere[k]] = k;
    m.n_channels = kNumLegs + 2;
    // stand height: feet on z = 0 in the default stance (csrc/arc_robot.c:183-194)
    V3<double> xs[kMaxBodies];
    Q4<double> qs[kMaxBodies];
    m.pose(V3<double>{0, 0, 0}, q_identity<double>(), m.default_angles, xs, qs);
    double lowest = 1e30;
    m.footprint = 0.0;
    for (int leg = 0; leg < kNumLegs; ++leg) {
        const ModelHost::Sphere& s = m.s[m.foot_sphere[leg]];
        V3<double> c = xs[s.body] + qrotate(qs[s.body], s.pos);
        lowest = lowest < c.z - s.radius ? lowest : c.z - s.radius;
        m.footprint += sqrt(c.x * c.x + c.y * c.y) / kNumLegs;
    }
    m.stand_height = -lowest;
    m.pose(V3<double>{0, 0, m.stand_height}, q_identity<double>(), m.default_angles, xs, qs);
    for (int i = 0; i < m.nb; ++i) {
        m.b[i].x = xs[i];
        m.b[i].q = qs[i];
    }
    m.leaper = is_leaper_topology(m);
}

bool is_leaper_topology(const ModelHost& m)
{
    if (m.nb != 13 || m.nj != 12 || m.ns != 21)
        return false;
    for (int k = 0; k < kNumLegs; ++k) {
        const int coxa = 1 + 3 * k, femur = 2 + 3 * k, tibia = 3 + 3 * k;
        if (m.j[3 * k].parent != 0 || m.j[3 * k].child != coxa)
            return false;
        if (m.j[3 * k + 1].parent != coxa || m.j[3 * k + 1].child != femur)
            return false;
        if (m.j[3 * k + 2].parent != femur || m.j[3 * k + 2].child != tibia)
            return false;
        if (m.s[1 + 5 * k].body != femur)
            return false;
        for (int c = 2; c <= 5; ++c)
            if (m.s[c + 5 * k].body != tibia)
                return false;
    }
    return m.s[0].body == 0;
}

template <class R> static V3<R> rv(V3<double> a) { return V3<R>{(R)a.x, (R)a.y, (R)a.z}; }

template <class R> DevModel<R> make_dev_model(const ModelHost& m, double dt, int substeps, double action_scale)
{
    DevModel<R> d;
    std::memset(&d, 0, sizeof(d));
    d.nb = m.nb;
    d.nj = m.nj;
    d.ns = m.ns;
    d.n_channels = m.n_channels;
    d.substeps = substeps;
    d.step_dt = dt;
    d.leaper = m.leaper ? 1 : 0;
    for (int i = 0; i < m.nb; ++i) {
        BodyK<R>& b = d.body[i];
        b.inv_mass = (R)m.b[i].inv_mass;
        b.inertia = rv<R>(m.b[i].inertia);
        b.inv_inertia = rv<R>(m.b[i].inv_inertia);
        b.iso = b.inertia.x == b.inertia.y && b.inertia.y == b.inertia.z && b.inv_inertia.x == b.inv_inertia.y &&
                b.inv_inertia.y == b.inv_inertia.z;
    }
    for (int i = 0; i < m.nj; ++i) {
        JointK<R>& j = d.joint[i];
        const ModelHost::Joint& t = m.j[i];
        j.parent = t.parent;
        j.child = t.child;
        j.r1 = rv<R>(t.r1); j.r2 = rv<R>(t.r2);
        j.a1 = rv<R>(t.a1); j.a2 = rv<R>(t.a2);
        j.b1 = rv<R>(t.b1); j.b2 = rv<R>(t.b2);
        j.lo = (R)t.lo; j.hi = (R)t.hi;
        j.kp = (R)t.kp; j.kd = (R)t.kd; j.max_torque = (R)t.max_torque;
        j.lim[0] = (R)cos(t.lo);
        j.lim[1] = (R)sin(t.lo);
        j.lim[2] = (R)cos(t.hi);
        j.lim[3] = (R)sin(t.hi);
        j.alpha = j.kp > R(0) ? R(1) / j.kp : R(0);
        d.lo[i] = j.lo;
        d.hi[i] = j.hi;
        d.default_angles[i] = m.default_angles[i];
    }
    for (int i = 0; i < m.ns; ++i) {
        d.sphere[i].body = m.s[i].body;
        d.sphere[i].pos = rv<R>(m.s[i].pos);
        d.sphere[i].radius = (R)m.s[i].radius;
        d.channel[i] = m.channel[i];
    }
    StepK<R>& s = d.step;
    s.h = (R)(dt / substeps);
    s.hh = s.h * s.h;
    s.inv_h = R(1) / s.h;
    s.two_h = R(2) / s.h;
    for (int i = 0; i < m.nj; ++i) {
        JointK<R>& j = d.joint[i];
        j.alpha_hh = j.alpha / s.hh;
        j.max_dl = j.max_torque * s.h * s.h;
        j.max_th = j.max_torque * s.h;
    }
    s.mu_s = (R)m.mu_s;
    s.mu_d = (R)m.mu_d;
    s.gravity = rv<R>(m.gravity);
    d.action_scale = action_scale;
    return d;
}

ResetModel make_reset_model(const ModelHost& m)
{
    ResetModel r;
    std::memset(&r, 0, sizeof(r));
    r.nb = m.nb;
    r.nj = m.nj;
    r.ns = m.ns;
    for (int i = 0; i < m.nj; ++i) {
        r.parent[i] = m.j[i].parent;
        r.child[i] = m.j[i].child;
        r.r1[i] = m.j[i].r1;
        r.r2[i] = m.j[i].r2;
        r.a1[i] = m.j[i].a1;
        r.q_rel0[i] = m.j[i].q_rel0;
        r.default_angles[i] = m.default_angles[i];
        r.lo[i] = m.j[i].lo;
        r.hi[i] = m.j[i].hi;
    }
    r.stand_height = m.stand_height;
    r.footprint = m.footprint;
    return r;
}

template DevModel<float> make_dev_model<float>(const ModelHost&, double, int, double);
template DevModel<double> make_dev_model<double>(const ModelHost&, double, int, double);

// Upper bound of the contacts one lane of the leg-parallel kernel records in
// a substep: a sphere of radius r touches at most (floor(2r/cell)+2)^2
// columns, one contact each.
int lane_contact_bound(const ModelHost& m, double cell)
{
    if (!m.leaper)
        return 0;
    int worst = 0;
    for (int leg = 0; leg < kNumLegs; ++leg) {
        long long sum = 0;
        for (int it = 0; it < 6; ++it) {
            int s = it == 0 ? (leg == 0 ? 0 : -1) : 5 * leg + it;
            if (s < 0)
                continue;
            long long per = (long long)std::floor(2.0 * m.s[s].radius / cell) + 2;
            sum += per * per;
        }
        worst = (int)std::max<long long>(worst, std::min<long long>(sum, kMaxContacts));
    }
    return worst;
}

}  // namespace arc
